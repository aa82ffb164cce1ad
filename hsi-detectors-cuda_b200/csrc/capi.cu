// capi.cu - library-wide C entry points: status text, version, plane stride.
#include "common.cuh"

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
