// hsi/sam_cuda.hpp and hsi/detect_cuda.hpp over the C ABI.
#include "hsi/sam_cuda.hpp"

#include <cstring>

#include "hsi/detect_cuda.hpp"
#include "status.hpp"
#include "workspace.hpp"

namespace hsi {

using detail::as_stream;
using detail::to_cuda;

namespace {
constexpr int kMaxTargets = 64;
}

const char* to_string(SamVariant variant) {
  switch (variant) {
    case SamVariant::Baseline: return "baseline";
    case SamVariant::Optimized: return "optimized";
    case SamVariant::Half: return "half";
    case SamVariant::BipDirect: return "bip";
  }
  return "unknown";
}

// The reference's names and aliases (src/sam.cu:330-336): "opt" and "fp16"
// are accepted beside the names to_string gives.
bool parse_sam_variant(const std::string& name, SamVariant* out) {
  for (SamVariant v : {SamVariant::Baseline, SamVariant::Optimized, SamVariant::Half, SamVariant::BipDirect}) {
    if (name == to_string(v)) {
      *out = v;
      return true;
    }
  }
  if (name == "opt" || name == "fp16") {
    *out = name == "opt" ? SamVariant::Optimized : SamVariant::Half;
    return true;
  }
  return false;
}

std::size_t bsq_plane_stride(CubeShape shape) {
  if (!shape.valid()) return 0;
  return static_cast<std::size_t>(hsi_plane_stride(shape.height, shape.width));
}

int max_constant_target_elements() { return kMaxTargets * HSI_MAX_BANDS; }

cudaError_t upload_targets(const float* values, const float* norms, int num_targets, int bands) {
  if (!values || !norms || num_targets <= 0 || num_targets > kMaxTargets || bands <= 0 || bands > HSI_MAX_BANDS)
    return cudaErrorInvalidValue;
  return cudaSuccess;
}

namespace {

hsi_frame frame_of(const void* d_cube, CubeShape shape, int dtype, std::size_t stride) {
  hsi_frame f;
  std::memset(&f, 0, sizeof(f));
  f.cube = d_cube;
  f.plane_stride = static_cast<int64_t>(stride);
  f.height = shape.height;
  f.width = shape.width;
  f.bands = shape.bands;
  f.dtype = dtype;
  f.map_stride = static_cast<int64_t>(shape.pixels());
  return f;
}

}  // namespace

cudaError_t launch_sam_best(SamVariant variant, const void* d_cube, CubeShape shape, const float* d_targets,
                            const float* d_target_norms, int num_targets, float* d_score,
                            std::int32_t* d_target_id, cudaStream_t stream, int /*opt_pixels_per_thread*/) {
  if (!d_cube || !shape.valid() || !d_targets || !d_target_norms || num_targets <= 0 || !d_score)
    return cudaErrorInvalidValue;
  const std::size_t stride = bsq_plane_stride(shape);
  int dtype = HSI_F32;
  if (variant == SamVariant::Half) {
    dtype = HSI_F16;
  } else if (variant == SamVariant::BipDirect) {
    // one pass over the BIP cube, the transpose fused into the scorer
    return to_cuda(hsi_sam_bip(static_cast<const float*>(d_cube), shape.height, shape.width, shape.bands, d_targets,
                               d_target_norms, num_targets, nullptr, 0, d_score, d_target_id, as_stream(stream)));
  }
  hsi_frame f = frame_of(d_cube, shape, dtype, stride);
  f.sam_targets = d_targets;
  f.sam_norms = d_target_norms;
  f.num_sam = num_targets;
  f.sam_best = d_score;
  f.sam_best_target = d_target_id;
  return to_cuda(hsi_score_frames(&f, 1, as_stream(stream)));
}

cudaError_t launch_sam_maps(const void* d_cube, CubeShape shape, bool half, const float* d_targets,
                            const float* d_target_norms, int num_targets, float* d_maps, std::size_t map_stride,
                            cudaStream_t stream) {
  if (!d_cube || !shape.valid() || !d_targets || !d_target_norms || num_targets <= 0 || !d_maps ||
      map_stride < shape.pixels())
    return cudaErrorInvalidValue;
  hsi_frame f = frame_of(d_cube, shape, half ? HSI_F16 : HSI_F32, bsq_plane_stride(shape));
  f.sam_targets = d_targets;
  f.sam_norms = d_target_norms;
  f.num_sam = num_targets;
  f.sam_maps = d_maps;
  f.map_stride = static_cast<int64_t>(map_stride);
  return to_cuda(hsi_score_frames(&f, 1, as_stream(stream)));
}

cudaError_t launch_transpose_bip_to_bsq(const float* d_src, float* d_dst, CubeShape shape, cudaStream_t stream) {
  if (!shape.valid()) return cudaErrorInvalidValue;
  return to_cuda(hsi_transpose_bip_to_bsq(d_src, d_dst, shape.height, shape.width, shape.bands,
                                          static_cast<int64_t>(bsq_plane_stride(shape)), as_stream(stream)));
}

cudaError_t launch_narrow_to_half(const float* d_src, void* d_dst, std::size_t count, cudaStream_t stream) {
  return to_cuda(hsi_narrow_to_half(d_src, d_dst, static_cast<int64_t>(count), as_stream(stream)));
}

cudaError_t launch_detect(const float* d_score, const std::int32_t* d_target_id, CubeShape shape,
                          DetectionParams params, Detection* d_out, unsigned int* d_count, cudaStream_t stream) {
  static_assert(sizeof(Detection) == sizeof(hsi_detection), "Detection must match hsi_detection");
  if (!d_score || !d_count || shape.height <= 0 || shape.width <= 0 || params.max_detections < 0 ||
      (params.max_detections > 0 && !d_out))
    return cudaErrorInvalidValue;
  const std::size_t bytes = hsi_detect_workspace_bytes(shape.height, shape.width);
  if (bytes == 0) return cudaErrorInvalidValue;  // beyond the detection kernels' segment limit
  void* ws = nullptr;
  const cudaError_t e = detail::stream_scratch(stream, bytes, &ws);
  if (e != cudaSuccess) return e;
  const int st = hsi_detect(d_score, d_target_id, shape.height, shape.width, params.threshold, params.nms_radius,
                            params.polarity == ScorePolarity::HigherIsBetter ? HSI_HIGHER_IS_BETTER
                                                                             : HSI_LOWER_IS_BETTER,
                            params.max_detections, reinterpret_cast<hsi_detection*>(d_out), d_count, ws, bytes,
                            as_stream(stream));
  return to_cuda(st);
}

}  // namespace hsi
