// capi.cu - library-wide C entry points: status text, version, plane stride.
#include <mutex>
#include <vector>

#include "common.cuh"
#include "launch_state.h"

extern "C" HSI_API const char* hsi_status_string(int status) {
  switch (status) {
    case HSI_OK: return "success";
    case HSI_E_NOT_POSITIVE_DEFINITE:
      return "matrix is not positive definite; hyperspectral bands are strongly correlated, so try a larger "
             "diagonal loading";
    case HSI_E_TIMEOUT: return "a bounded device-side wait gave up (pipeline stalled)";
    case HSI_E_WORKSPACE: return "workspace missing or smaller than required";
    case HSI_E_CAPACITY: return "a size exceeds a documented maximum";
    case HSI_E_NO_DEVICE: return "no CUDA device";
    default:
      if (status > 0 && status < 10000) return cudaGetErrorString(static_cast<cudaError_t>(status));
      return "unknown status";
  }
}

extern "C" HSI_API int hsi_version(void) { return 100; }

extern "C" HSI_API int64_t hsi_plane_stride(int height, int width) {
  if (height <= 0 || width <= 0) return 0;
  const int64_t pixels = static_cast<int64_t>(height) * width;
  return (pixels + 31) / 32 * 32;
}

// ---- per-device launch state (launch_state.h) ---------------------------------
namespace hsi_b200 {
namespace {

constexpr int kMaxDevices = 64;

std::mutex g_state_mutex;
int g_sm_count[kMaxDevices];  // 0 = not read yet

struct Limit {
  int device;
  const void* func;
  int bytes;
};
struct Residency {
  int device;
  const void* func;
  int threads;
  size_t smem;
  int blocks;
};
std::vector<Limit> g_limits;
std::vector<Residency> g_residency;

int current_device() {
  int dev = 0;
  return cudaGetDevice(&dev) == cudaSuccess ? dev : -1;
}

}  // namespace

int device_sm_count() {
  const int dev = current_device();
  if (dev < 0) return 148;
  if (dev < kMaxDevices) {
    std::lock_guard<std::mutex> lock(g_state_mutex);
    if (g_sm_count[dev] > 0) return g_sm_count[dev];
  }
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) return 148;
  if (dev < kMaxDevices) {
    std::lock_guard<std::mutex> lock(g_state_mutex);
    g_sm_count[dev] = v;
  }
  return v;
}

cudaError_t raise_smem_limit(const void* func, int bytes) {
  const int dev = current_device();
  std::lock_guard<std::mutex> lock(g_state_mutex);
  for (Limit& l : g_limits) {
    if (l.device != dev || l.func != func) continue;
    if (l.bytes >= bytes) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) l.bytes = bytes;
    return e;
  }
  const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) g_limits.push_back(Limit{dev, func, bytes});
  return e;
}

int device_residency(const void* func, int threads, size_t smem) {
  if (raise_smem_limit(func, static_cast<int>(smem)) != cudaSuccess) return 0;
  const int dev = current_device();
  {
    std::lock_guard<std::mutex> lock(g_state_mutex);
    for (const Residency& r : g_residency)
      if (r.device == dev && r.func == func && r.threads == threads && r.smem == smem) return r.blocks;
  }
  int v = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, func, threads, smem) != cudaSuccess || v <= 0) return 0;
  std::lock_guard<std::mutex> lock(g_state_mutex);
  g_residency.push_back(Residency{dev, func, threads, smem, v});
  return v;
}

}  // namespace hsi_b200
