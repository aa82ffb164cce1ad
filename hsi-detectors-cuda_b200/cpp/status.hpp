// Status translation between the C ABI and the cudaError_t the hsi C++ API
// returns (the reference's launchers return cudaError_t).
#pragma once

#include <cuda_runtime.h>

#include "hsi_b200.h"

namespace hsi {
namespace detail {

// 0 -> cudaSuccess; CUDA runtime codes pass through; the library's own codes
// map to the nearest runtime meaning.
inline cudaError_t to_cuda(int status) {
  if (status == HSI_OK) return cudaSuccess;
  if (status < 10000) return static_cast<cudaError_t>(status);
  switch (status) {
    case HSI_E_TIMEOUT: return cudaErrorLaunchTimeout;
    case HSI_E_NO_DEVICE: return cudaErrorNoDevice;
    default: return cudaErrorInvalidValue;
  }
}

inline hsi_stream_t as_stream(cudaStream_t s) { return reinterpret_cast<hsi_stream_t>(s); }

}  // namespace detail
}  // namespace hsi
