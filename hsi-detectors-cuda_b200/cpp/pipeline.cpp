// hsi::Pipeline over the C ABI: slots of pinned host + device buffers, one
// stream each; per frame: upload, [narrow to fp16], score (hsi_score_frames),
// detect (hsi_detect), download; results harvested in submission order.
#include "hsi/pipeline.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <sstream>

#include "hsi/detect_cuda.hpp"
#include "hsi_b200.h"

namespace hsi {

const char* to_string(MemoryMode mode) { return mode == MemoryMode::ZeroCopy ? "zerocopy" : "copy"; }

bool parse_memory_mode(const std::string& name, MemoryMode* out) {
  if (name == "copy") {
    *out = MemoryMode::Copy;
    return true;
  }
  if (name == "zerocopy" || name == "zero-copy") {  // the reference's alias (src/pipeline.cu:452-456)
    *out = MemoryMode::ZeroCopy;
    return true;
  }
  return false;
}

namespace {

using Clock = std::chrono::steady_clock;

float ms_since(Clock::time_point t0) { return std::chrono::duration<float, std::milli>(Clock::now() - t0).count(); }

float quantile(std::vector<float> v, double q) {
  if (v.empty()) return 0.0f;
  std::sort(v.begin(), v.end());
  const double pos = q * (static_cast<double>(v.size()) - 1.0);
  const std::size_t lo = static_cast<std::size_t>(pos), hi = std::min(lo + 1, v.size() - 1);
  const double f = pos - static_cast<double>(lo);
  return static_cast<float>(v[lo] * (1.0 - f) + v[hi] * f);
}

float mean_of(const std::vector<float>& v) {
  double s = 0.0;
  for (float x : v) s += x;
  return v.empty() ? 0.0f : static_cast<float>(s / static_cast<double>(v.size()));
}

struct Slot {
  cudaStream_t stream = nullptr;
  float* host_cube = nullptr;    // pinned
  float* device_cube = nullptr;
  void* half_cube = nullptr;     // SamVariant::Half only
  float* d_score = nullptr;
  std::int32_t* d_target = nullptr;
  hsi_detection* d_dets = nullptr;
  unsigned* d_count = nullptr;
  void* d_workspace = nullptr;
  hsi_detection* h_dets = nullptr;  // pinned
  unsigned* h_count = nullptr;      // pinned
  float* h_score = nullptr;         // pinned, return_score_map only
  cudaEvent_t ev[5] = {};           // begin, uploaded, scored, detected, done
  FrameMeta meta;
  float ms_source = 0;
  Clock::time_point submitted;
  bool busy = false;
};

#define HSI_TRY(expr, what)                                                        \
  do {                                                                             \
    const cudaError_t e_ = (expr);                                                 \
    if (e_ != cudaSuccess) {                                                       \
      if (error) *error = std::string(what) + ": " + cudaGetErrorString(e_);       \
      return false;                                                                \
    }                                                                              \
  } while (0)

#define HSI_TRY_ABI(expr, what)                                                    \
  do {                                                                             \
    const int s_ = (expr);                                                         \
    if (s_ != HSI_OK) {                                                            \
      if (error) *error = std::string(what) + ": " + hsi_status_string(s_);        \
      return false;                                                                \
    }                                                                              \
  } while (0)

class PipelineImpl final : public Pipeline {
 public:
  PipelineImpl(FrameSource* source, const SpectralLibrary& library, const PipelineOptions& opt)
      : source_(source), library_(library), opt_(opt), shape_(source->shape()) {}

  ~PipelineImpl() override {
    for (Slot& s : slots_) {
      if (s.stream) cudaStreamSynchronize(s.stream);
      for (cudaEvent_t e : s.ev)
        if (e) cudaEventDestroy(e);
      cudaFreeHost(s.host_cube);
      cudaFreeHost(s.h_dets);
      cudaFreeHost(s.h_count);
      cudaFreeHost(s.h_score);
      cudaFree(s.device_cube);
      cudaFree(s.half_cube);
      cudaFree(s.d_score);
      cudaFree(s.d_target);
      cudaFree(s.d_dets);
      cudaFree(s.d_count);
      cudaFree(s.d_workspace);
      if (s.stream) cudaStreamDestroy(s.stream);
    }
    cudaFree(d_targets_);
    cudaFree(d_norms_);
  }

  bool init(std::string* error) {
    const int T = library_.size();
    if (opt_.memory == MemoryMode::ZeroCopy) {
      if (error) *error = "MemoryMode::ZeroCopy is not supported: frames are uploaded to device memory";
      return false;
    }
    if (opt_.variant == SamVariant::BipDirect && source_->interleave() != Interleave::Bip) {
      if (error) *error = "SamVariant::BipDirect needs a BIP source";
      return false;
    }
    if (opt_.variant != SamVariant::BipDirect && source_->interleave() != Interleave::Bsq) {
      if (error) *error = "the source must deliver BSQ frames for this variant";
      return false;
    }
    const std::vector<float> flat = library_.flatten();
    const std::vector<float> norms = library_.norms();
    HSI_TRY(upload_targets(flat.data(), norms.data(), T, library_.bands()), "library");
    if (library_.bands() != shape_.bands) {
      if (error) *error = "library has " + std::to_string(library_.bands()) + " bands, the source " +
                          std::to_string(shape_.bands);
      return false;
    }
    if (opt_.num_streams < 1 || opt_.detection.max_detections < 0) {
      if (error) *error = "num_streams must be >= 1 and max_detections >= 0";
      return false;
    }
    stride_ = bsq_plane_stride(shape_);
    const std::size_t elems = bsq_device_elements(shape_);
    const std::size_t P = shape_.pixels();
    const std::size_t cap = static_cast<std::size_t>(std::max(opt_.detection.max_detections, 1));
    ws_bytes_ = hsi_detect_workspace_bytes(shape_.height, shape_.width);
    HSI_TRY(cudaMalloc(&d_targets_, sizeof(float) * flat.size()), "allocate library");
    HSI_TRY(cudaMalloc(&d_norms_, sizeof(float) * norms.size()), "allocate library");
    HSI_TRY(cudaMemcpy(d_targets_, flat.data(), sizeof(float) * flat.size(), cudaMemcpyHostToDevice), "library");
    HSI_TRY(cudaMemcpy(d_norms_, norms.data(), sizeof(float) * norms.size(), cudaMemcpyHostToDevice), "library");
    slots_.resize(static_cast<std::size_t>(opt_.num_streams));
    const unsigned flags = opt_.time_stages ? cudaEventDefault : cudaEventDisableTiming;
    for (Slot& s : slots_) {
      HSI_TRY(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "create stream");
      HSI_TRY(cudaMallocHost(&s.host_cube, sizeof(float) * elems), "pinned cube");
      HSI_TRY(cudaMalloc(&s.device_cube, sizeof(float) * elems), "device cube");
      if (opt_.variant == SamVariant::Half) HSI_TRY(cudaMalloc(&s.half_cube, 2 * elems), "fp16 cube");
      HSI_TRY(cudaMalloc(&s.d_score, sizeof(float) * P), "score map");
      HSI_TRY(cudaMalloc(&s.d_target, sizeof(std::int32_t) * P), "target map");
      HSI_TRY(cudaMalloc(&s.d_dets, sizeof(hsi_detection) * cap), "detections");
      HSI_TRY(cudaMalloc(&s.d_count, sizeof(unsigned)), "count");
      HSI_TRY(cudaMalloc(&s.d_workspace, ws_bytes_), "detection workspace");
      HSI_TRY(cudaMallocHost(&s.h_dets, sizeof(hsi_detection) * cap), "pinned detections");
      HSI_TRY(cudaMallocHost(&s.h_count, sizeof(unsigned)), "pinned count");
      if (opt_.return_score_map) HSI_TRY(cudaMallocHost(&s.h_score, sizeof(float) * P), "pinned score map");
      for (cudaEvent_t& e : s.ev) HSI_TRY(cudaEventCreateWithFlags(&e, flags), "create event");
    }
    if (opt_.prefill > 0) {
      prefilled_ = true;
      for (Slot& s : slots_)
        if (!source_->read_into(s.host_cube, stride_, &s.meta)) {
          if (error) *error = "source ended while prefilling";
          return false;
        }
    }
    return true;
  }

  bool run(std::uint64_t frames, const std::function<void(const FrameResult&)>& on_frame,
           std::string* error) override {
    stats_ = PipelineStats{};
    lat_.clear();
    src_.clear();
    up_.clear();
    sc_.clear();
    de_.clear();
    dn_.clear();
    gpu_.clear();
    const auto t0 = Clock::now();
    std::deque<Slot*> pending;
    std::uint64_t submitted = 0;
    bool dry = false;
    while (!dry && (frames == 0 || submitted < frames)) {
      Slot& s = slots_[submitted % slots_.size()];
      if (s.busy) {
        // the oldest pending frame is this slot's (round robin)
        if (!harvest(*pending.front(), on_frame, error)) return false;
        pending.pop_front();
      }
      const auto ts = Clock::now();
      if (!prefilled_) {
        if (!source_->read_into(s.host_cube, stride_, &s.meta)) {
          dry = true;
          break;
        }
      } else {
        s.meta.index = submitted;
        s.meta.timestamp_s = static_cast<double>(submitted) / 30.0;
      }
      s.ms_source = ms_since(ts);
      s.submitted = Clock::now();
      if (!submit(s, error)) return false;
      pending.push_back(&s);
      ++submitted;
    }
    while (!pending.empty()) {
      if (!harvest(*pending.front(), on_frame, error)) return false;
      pending.pop_front();
    }
    const double wall = std::chrono::duration<double>(Clock::now() - t0).count();
    stats_.wall_s = wall;
    if (wall > 0) {
      stats_.fps = static_cast<double>(stats_.frames) / wall;
      stats_.mpixel_per_s = static_cast<double>(stats_.frames) * shape_.pixels() / wall / 1e6;
      stats_.cube_gb_per_s = static_cast<double>(stats_.frames) * shape_.bytes_f32() / wall / 1e9;
    }
    stats_.ms_p50 = quantile(lat_, 0.50);
    stats_.ms_p95 = quantile(lat_, 0.95);
    stats_.ms_p99 = quantile(lat_, 0.99);
    stats_.ms_max = lat_.empty() ? 0.0f : *std::max_element(lat_.begin(), lat_.end());
    stats_.mean_source = mean_of(src_);
    stats_.mean_upload = mean_of(up_);
    stats_.mean_score = mean_of(sc_);
    stats_.mean_detect = mean_of(de_);
    stats_.mean_download = mean_of(dn_);
    stats_.mean_gpu = mean_of(gpu_);
    return true;
  }

  PipelineStats stats() const override { return stats_; }

  std::string describe() const override {
    std::ostringstream o;
    o << "hsi-b200 pipeline: " << shape_.height << "x" << shape_.width << "x" << shape_.bands << ", "
      << library_.size() << " targets, variant " << to_string(opt_.variant) << ", " << slots_.size()
      << " streams, threshold " << opt_.detection.threshold << ", nms radius " << opt_.detection.nms_radius
      << ", capacity " << opt_.detection.max_detections << (prefilled_ ? ", prefilled" : "") << "; source: "
      << source_->describe();
    return o.str();
  }

 private:
  bool submit(Slot& s, std::string* error) {
    const std::size_t elems = bsq_device_elements(shape_);
    HSI_TRY(cudaEventRecord(s.ev[0], s.stream), "record");
    const bool bip = opt_.variant == SamVariant::BipDirect;
    // a BIP frame arrives packed (pixels * bands floats)
    const std::size_t bytes = sizeof(float) * (bip ? shape_.elements() : elems);
    HSI_TRY(cudaMemcpyAsync(s.device_cube, s.host_cube, bytes, cudaMemcpyHostToDevice, s.stream), "upload cube");
    HSI_TRY(cudaEventRecord(s.ev[1], s.stream), "record");
    const void* cube = s.device_cube;
    if (opt_.variant == SamVariant::Half) {
      HSI_TRY(launch_narrow_to_half(s.device_cube, s.half_cube, elems, s.stream), "narrow to fp16");
      cube = s.half_cube;
    }
    HSI_TRY(launch_sam_best(opt_.variant, cube, shape_, d_targets_, d_norms_, library_.size(), s.d_score, s.d_target,
                            s.stream),
            "score");
    HSI_TRY(cudaEventRecord(s.ev[2], s.stream), "record");
    HSI_TRY(cudaMemsetAsync(s.d_count, 0, sizeof(unsigned), s.stream), "zero count");
    const DetectionParams& p = opt_.detection;
    HSI_TRY_ABI(hsi_detect(s.d_score, s.d_target, shape_.height, shape_.width, p.threshold, p.nms_radius,
                           p.polarity == ScorePolarity::HigherIsBetter ? HSI_HIGHER_IS_BETTER : HSI_LOWER_IS_BETTER,
                           p.max_detections, s.d_dets, s.d_count, s.d_workspace, ws_bytes_,
                           reinterpret_cast<hsi_stream_t>(s.stream)),
                "detect");
    HSI_TRY(cudaEventRecord(s.ev[3], s.stream), "record");
    HSI_TRY(cudaMemcpyAsync(s.h_count, s.d_count, sizeof(unsigned), cudaMemcpyDeviceToHost, s.stream), "download");
    if (p.max_detections > 0)
      HSI_TRY(cudaMemcpyAsync(s.h_dets, s.d_dets, sizeof(hsi_detection) * p.max_detections, cudaMemcpyDeviceToHost,
                              s.stream),
              "download");
    if (opt_.return_score_map)
      HSI_TRY(cudaMemcpyAsync(s.h_score, s.d_score, sizeof(float) * shape_.pixels(), cudaMemcpyDeviceToHost,
                              s.stream),
              "download");
    HSI_TRY(cudaEventRecord(s.ev[4], s.stream), "record");
    s.busy = true;
    return true;
  }

  bool harvest(Slot& s, const std::function<void(const FrameResult&)>& on_frame, std::string* error) {
    HSI_TRY(cudaEventSynchronize(s.ev[4]), "wait for frame");
    s.busy = false;
    FrameResult r;
    r.meta = s.meta;
    r.detections_found = *s.h_count;
    const unsigned kept = std::min<unsigned>(r.detections_found, static_cast<unsigned>(opt_.detection.max_detections));
    r.detections.resize(kept);
    if (kept) std::memcpy(static_cast<void*>(r.detections.data()), s.h_dets, sizeof(Detection) * kept);
    if (opt_.return_score_map) r.score_map.assign(s.h_score, s.h_score + shape_.pixels());
    r.ms_source = s.ms_source;
    if (opt_.time_stages) {
      cudaEventElapsedTime(&r.ms_upload, s.ev[0], s.ev[1]);
      cudaEventElapsedTime(&r.ms_score, s.ev[1], s.ev[2]);
      cudaEventElapsedTime(&r.ms_detect, s.ev[2], s.ev[3]);
      cudaEventElapsedTime(&r.ms_download, s.ev[3], s.ev[4]);
      cudaEventElapsedTime(&r.ms_gpu, s.ev[0], s.ev[4]);
    }
    r.ms_wall = ms_since(s.submitted) + s.ms_source;
    ++stats_.frames;
    stats_.total_detections += r.detections_found;
    lat_.push_back(r.ms_wall);
    src_.push_back(r.ms_source);
    up_.push_back(r.ms_upload);
    sc_.push_back(r.ms_score);
    de_.push_back(r.ms_detect);
    dn_.push_back(r.ms_download);
    gpu_.push_back(r.ms_gpu);
    if (on_frame) on_frame(r);
    return true;
  }

  FrameSource* source_;
  SpectralLibrary library_;
  PipelineOptions opt_;
  CubeShape shape_;
  std::size_t stride_ = 0, ws_bytes_ = 0;
  float* d_targets_ = nullptr;
  float* d_norms_ = nullptr;
  std::vector<Slot> slots_;
  bool prefilled_ = false;
  PipelineStats stats_;
  std::vector<float> lat_, src_, up_, sc_, de_, dn_, gpu_;
};

}  // namespace

std::unique_ptr<Pipeline> Pipeline::create(FrameSource* source, const SpectralLibrary& library,
                                           const PipelineOptions& options, std::string* error) {
  if (!source) {
    if (error) *error = "no frame source";
    return nullptr;
  }
  if (library.size() <= 0) {
    if (error) *error = "the target library is empty";
    return nullptr;
  }
  std::unique_ptr<PipelineImpl> p(new PipelineImpl(source, library, options));
  if (!p->init(error)) return nullptr;
  return p;
}

}  // namespace hsi
