// generate.cu - device generator for the synthetic scenes of synth.h.
//
// One thread per pixel: the band-independent draws (abundances, gain, implant)
// are made once, then the thread walks the bands, so consecutive threads write
// consecutive addresses of every band plane.
#include <cuda_fp16.h>

#include "common.cuh"
#include "launch_state.h"
#include "synth.h"

namespace hsi_b200 {
namespace {

hsi_scene_spec to_spec(const hsi_scene& s) {
  hsi_scene_spec out;
  out.bands = s.bands;
  out.n_end = s.n_end;
  out.n_targets = s.n_targets;
  out.target_frac = s.target_frac;
  out.anomaly_frac = s.anomaly_frac;
  out.noise_sigma = s.noise_sigma;
  out.library_seed = s.library_seed;
  out.frame_seed = s.frame_seed;
  return out;
}

template <typename T>
__device__ __forceinline__ T from_float(float v);
template <>
__device__ __forceinline__ float from_float<float>(float v) {
  return v;
}
template <>
__device__ __forceinline__ __half from_float<__half>(float v) {
  return __float2half_rn(v);
}

template <typename T>
__global__ void __launch_bounds__(256) generate_kernel(hsi_scene_spec spec, const float* __restrict__ spectra,
                                                       int64_t pixels, int64_t pixel0, T* __restrict__ cube,
                                                       int64_t stride, uint8_t* __restrict__ truth) {
  extern __shared__ float s_spectra[];  // [bands][n_spectra], band-major
  const int B = spec.bands;
  const int n_spectra = spec.n_end + spec.n_targets + 1;
  for (int i = threadIdx.x; i < n_spectra * B; i += blockDim.x) {
    const int k = i / B, b = i % B;
    s_spectra[b * n_spectra + k] = spectra[i];
  }
  __syncthreads();

  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < pixels;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint64_t id = static_cast<uint64_t>(pixel0 + p);
    const hsi_pixel_draw d = hsi_draw_pixel(&spec, id);
    const int implant_col = d.implant >= 0 ? spec.n_end + d.implant : 0;
    for (int b = 0; b < B; ++b) {
      const float* col = s_spectra + b * n_spectra;
      const float v = hsi_pixel_value(&spec, &d, id, b, col, col[implant_col]);
      cube[static_cast<int64_t>(b) * stride + p] = from_float<T>(v);
    }
    if (truth) truth[p] = static_cast<uint8_t>(d.truth);
  }
}

}  // namespace
}  // namespace hsi_b200

using namespace hsi_b200;

extern "C" HSI_API int hsi_scene_spectra(const hsi_scene* scene, float* out) {
  if (!scene || !out || scene->bands <= 0 || scene->bands > HSI_MAX_BANDS || scene->n_end < 1 ||
      scene->n_end > 8 || scene->n_targets < 0 || scene->n_targets > 64)
    return HSI_E_INVALID;
  const int B = scene->bands;
  int k = 0;
  for (int e = 0; e < scene->n_end; ++e, ++k)
    hsi_spectrum(scene->library_seed, HSI_SPECTRUM_ENDMEMBER(e), B, out + static_cast<int64_t>(k) * B);
  for (int t = 0; t < scene->n_targets; ++t, ++k)
    hsi_spectrum(scene->library_seed, HSI_SPECTRUM_TARGET(t), B, out + static_cast<int64_t>(k) * B);
  hsi_spectrum(scene->library_seed, HSI_SPECTRUM_ANOMALY, B, out + static_cast<int64_t>(k) * B);
  return HSI_OK;
}

extern "C" HSI_API int hsi_generate(const hsi_scene* scene, const float* d_spectra, int height, int width,
                                    int64_t pixel0, void* d_cube, int dtype, int64_t plane_stride,
                                    uint8_t* d_truth, hsi_stream_t stream) {
  if (!scene || !d_spectra || !d_cube || height <= 0 || width <= 0) return HSI_E_INVALID;
  if (scene->bands <= 0 || scene->bands > HSI_MAX_BANDS || scene->n_end < 1 || scene->n_end > 8 ||
      scene->n_targets < 0 || scene->n_targets > 64)
    return HSI_E_INVALID;
  const int64_t pixels = static_cast<int64_t>(height) * width;
  if (plane_stride < pixels) return HSI_E_INVALID;
  const hsi_scene_spec spec = to_spec(*scene);
  const size_t smem = sizeof(float) * static_cast<size_t>(scene->bands) *
                      static_cast<size_t>(scene->n_end + scene->n_targets + 1);
  int blocks = static_cast<int>(div_up<int64_t>(pixels, 256));
  if (blocks > 148 * 16) blocks = 148 * 16;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (dtype == HSI_F32) {
    const cudaError_t e = raise_smem_limit(generate_kernel<float>, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    generate_kernel<float><<<blocks, 256, smem, s>>>(spec, d_spectra, pixels, pixel0,
                                                     static_cast<float*>(d_cube), plane_stride, d_truth);
  } else if (dtype == HSI_F16) {
    const cudaError_t e = raise_smem_limit(generate_kernel<__half>, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    generate_kernel<__half><<<blocks, 256, smem, s>>>(spec, d_spectra, pixels, pixel0,
                                                      static_cast<__half*>(d_cube), plane_stride, d_truth);
  } else {
    return HSI_E_INVALID;
  }
  return static_cast<int>(cudaGetLastError());
}
