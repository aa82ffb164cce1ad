// launch_state.h - host-side one-time launch state, kept per device.
//
// Kernel attributes (the dynamic shared-memory limit) and device properties
// (the SM count, residency) belong to a device, not to the process: a caller
// that launches on two devices in one process needs each set up on each.
// These helpers key that state by the current device ordinal, are safe to call
// from several host threads, never lower a limit another thread relies on, and
// do not remember failures (a failed query is retried on the next call).
#pragma once

#include <cuda_runtime.h>

namespace hsi_b200 {

// Multiprocessors of the current device (148 when the query fails).
int device_sm_count();

// Raise `func`'s dynamic shared-memory limit on the current device to at least
// `bytes`.  The limit only ever grows, so a launch prepared by one host thread
// cannot be undercut by another thread that configures a smaller layout.
cudaError_t raise_smem_limit(const void* func, int bytes);

// Blocks of `func` resident per SM of the current device at `threads` threads
// and `smem` bytes of dynamic shared memory (0 if the query fails; callers
// choose their own floor).  Calls raise_smem_limit(func, smem) first.
int device_residency(const void* func, int threads, size_t smem);

template <typename K>
cudaError_t raise_smem_limit(K* func, int bytes) {
  return raise_smem_limit(reinterpret_cast<const void*>(func), bytes);
}

template <typename K>
int device_residency(K* func, int threads, size_t smem) {
  return device_residency(reinterpret_cast<const void*>(func), threads, smem);
}

}  // namespace hsi_b200
