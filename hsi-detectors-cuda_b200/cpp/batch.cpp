// The batched frame runner behind include/hsi_batch.h: a fixed plan of
// launches over frames of uneven sizes and band counts, run eagerly or
// replayed as one CUDA graph, with an autotuner that times the plan's
// tunable choices on the batch itself.
#include "hsi_batch.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "hsi/detectors.hpp"

namespace {

struct Frame {
  hsi_batch_frame spec{};
  int64_t P = 0, stride = 0;
  void* cube = nullptr;
  float* targets = nullptr;
  float* norms = nullptr;
  double* moments = nullptr;
  double* stats64 = nullptr;
  int32_t* status = nullptr;
  float* sam_best = nullptr;
  int32_t* sam_target = nullptr;
  float* rx = nullptr;
  float* ace_best = nullptr;
  int32_t* ace_target = nullptr;
  hsi_detection* dets[3] = {nullptr, nullptr, nullptr};
  uint32_t* counts = nullptr;
  float rx_threshold = 0.0f;
  bool tensor_core_rx = false;
};

}  // namespace

struct hsi_batch {
  // Per-frame chains (factor, then RX/ACE) run on kLanes streams forked from
  // the caller's stream, and the SAM scorer on one more, so frames overlap:
  // a frame's FP64 factor occupies two SMs and a small frame's RX/ACE only
  // part of the GPU.  Each lane has its own factor and RX/ACE workspace.
  static constexpr int kLanes = 4;
  std::vector<Frame> frames;
  hsi_batch_options opt{};
  std::vector<void*> allocations;
  void* stats_ws = nullptr;
  size_t stats_bytes = 0;
  void* factor_ws[kLanes] = {};
  size_t factor_bytes = 0;
  void* rx_ws[kLanes] = {};
  size_t rx_bytes = 0;
  std::vector<int> lane_of;            // lane of each frame's chain
  cudaStream_t lanes[kLanes + 1] = {};  // [kLanes]: the scorer's
  cudaEvent_t ev_cubes = nullptr, ev_moments = nullptr, ev_done[kLanes + 1] = {};
  void* det_ws = nullptr;
  size_t det_bytes = 0;
  uint32_t* all_counts = nullptr;
  std::vector<hsi_detect_job> jobs;
  std::vector<hsi_moments_job> moment_jobs;  // every frame's moments in one batched call
  hsi_frame* table[2] = {nullptr, nullptr};
  int table_n[2] = {0, 0}, table_bands[2] = {0, 0}, table_targets[2] = {0, 0};
  int32_t* score_status = nullptr;
  int score_ctas_per_sm = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  float tuning_ms = 0.0f;

  ~hsi_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (cudaStream_t l : lanes)
      if (l) cudaStreamDestroy(l);
    for (cudaEvent_t e : ev_done)
      if (e) cudaEventDestroy(e);
    if (ev_cubes) cudaEventDestroy(ev_cubes);
    if (ev_moments) cudaEventDestroy(ev_moments);
    for (void* p : allocations) cudaFree(p);
  }

  int make_lanes() {
    for (cudaStream_t& l : lanes)
      if (cudaStreamCreateWithFlags(&l, cudaStreamNonBlocking) != cudaSuccess) return HSI_E_INVALID;
    for (cudaEvent_t& e : ev_done)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return HSI_E_INVALID;
    if (cudaEventCreateWithFlags(&ev_cubes, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_moments, cudaEventDisableTiming) != cudaSuccess)
      return HSI_E_INVALID;
    return HSI_OK;
  }

  template <typename T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 256));
    if (e != cudaSuccess) return static_cast<int>(e);
    allocations.push_back(q);
    *p = static_cast<T*>(q);
    return HSI_OK;
  }

  int rx_ace(Frame& f, bool tensor_core, int lane, cudaStream_t s) {
    const hsi_batch_frame& sp = f.spec;
    const hsi_stream_t hs = reinterpret_cast<hsi_stream_t>(s);
    if (tensor_core)
      return hsi_rx_ace(f.cube, sp.height, sp.width, sp.bands, sp.dtype, f.stride, f.stats64, sp.num_targets, f.rx,
                        f.ace_best, f.ace_target, nullptr, f.P, rx_ws[lane], rx_bytes, hs);
    return hsi_rx_ace_simt(f.cube, sp.height, sp.width, sp.bands, sp.dtype, f.stride, f.stats64, sp.num_targets, f.rx,
                           f.ace_best, f.ace_target, nullptr, f.P, rx_ws[lane], rx_bytes, hs);
  }

  int score(int cps, cudaStream_t s) {
    for (int d = 0; d < 2; ++d) {
      if (!table_n[d]) continue;
      const int rc = hsi_score_frames_device_grid(table[d], table_n[d], d, table_bands[d], table_targets[d], 0,
                                                  score_status, cps, reinterpret_cast<hsi_stream_t>(s));
      if (rc != HSI_OK) return rc;
    }
    return HSI_OK;
  }

  // The plan on the caller's stream s: demosaic; then the scorer on its lane
  // (it needs only the cubes) while s runs the batched moments; then each
  // frame's factor and RX/ACE on the frame's lane; s waits for every lane and
  // runs the detection launches.  Every fork is joined before return (also on
  // errors), so a capture of s records the whole plan.
  int run(cudaStream_t s) {
    const hsi_stream_t hs = reinterpret_cast<hsi_stream_t>(s);
    for (Frame& f : frames) {
      const hsi_batch_frame& sp = f.spec;
      if (!sp.raw) continue;
      const int rc = hsi_demosaic(sp.raw, sp.raw_height, sp.raw_width, sp.period, sp.bands, nullptr, f.cube, HSI_F32,
                                  f.stride, hs);
      if (rc != HSI_OK) return rc;
    }
    cudaError_t e = cudaEventRecord(ev_cubes, s);
    if (e != cudaSuccess) return static_cast<int>(e);
    int rc = HSI_OK;
    bool forked[kLanes + 1] = {};
    if ((e = cudaStreamWaitEvent(lanes[kLanes], ev_cubes, 0)) == cudaSuccess) {
      forked[kLanes] = true;
      rc = score(score_ctas_per_sm, lanes[kLanes]);
    }
    if (rc == HSI_OK && e == cudaSuccess)
      rc = hsi_scene_moments_batch(moment_jobs.data(), static_cast<int>(moment_jobs.size()), stats_ws, stats_bytes, hs);
    if (rc == HSI_OK && e == cudaSuccess) e = cudaEventRecord(ev_moments, s);
    for (int l = 0; l < kLanes && rc == HSI_OK && e == cudaSuccess; ++l) {
      if ((e = cudaStreamWaitEvent(lanes[l], ev_moments, 0)) != cudaSuccess) break;
      forked[l] = true;
      const hsi_stream_t hl = reinterpret_cast<hsi_stream_t>(lanes[l]);
      for (size_t i = 0; i < frames.size() && rc == HSI_OK; ++i) {
        if (lane_of[i] != l) continue;
        Frame& f = frames[i];
        const hsi_batch_frame& sp = f.spec;
        rc = hsi_build_statistics(1, sp.bands, sp.num_targets, opt.loading, f.moments, f.targets, 0, f.stats64,
                                  nullptr, nullptr, f.status, factor_ws[l], factor_bytes, hl);
        if (rc == HSI_OK) rc = rx_ace(f, f.tensor_core_rx, l, lanes[l]);
      }
    }
    // join every lane that was forked
    for (int l = 0; l <= kLanes; ++l) {
      if (!forked[l]) continue;
      cudaError_t j = cudaEventRecord(ev_done[l], lanes[l]);
      if (j == cudaSuccess) j = cudaStreamWaitEvent(s, ev_done[l], 0);
      if (e == cudaSuccess) e = j;
    }
    if (rc != HSI_OK) return rc;
    if (e != cudaSuccess) return static_cast<int>(e);
    e = cudaMemsetAsync(all_counts, 0, sizeof(uint32_t) * 3 * frames.size(), s);
    if (e != cudaSuccess) return static_cast<int>(e);
    for (size_t j0 = 0; j0 < jobs.size(); j0 += HSI_MAX_DETECT_JOBS) {
      const int n = static_cast<int>(std::min<size_t>(HSI_MAX_DETECT_JOBS, jobs.size() - j0));
      rc = hsi_detect_batch(&jobs[j0], n, det_ws, det_bytes, hs);
      if (rc != HSI_OK) return rc;
    }
    return HSI_OK;
  }
};

namespace {

// Mean device time of `reps` calls of fn on `s`.
template <typename F>
float time_ms(F&& fn, int reps, cudaStream_t s, int* rc) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, s);
  for (int i = 0; i < reps && *rc == HSI_OK; ++i) *rc = fn();
  cudaEventRecord(b, s);
  cudaEventSynchronize(b);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / reps;
}

int build(hsi_batch* bt, const hsi_batch_frame* frames, int n) {
  const hsi_batch_options& o = bt->opt;
  std::vector<hsi_frame> tables[2];
  bt->frames.resize(n);
  size_t rx_bytes = 0;
  for (int i = 0; i < n; ++i) {
    Frame& f = bt->frames[i];
    f.spec = frames[i];
    hsi_batch_frame& sp = f.spec;
    if (sp.raw) {
      if (sp.period <= 0 || sp.bands <= 0 || sp.bands > sp.period * sp.period) return HSI_E_INVALID;
      sp.height = sp.raw_height / sp.period;
      sp.width = sp.raw_width / sp.period;
      sp.dtype = HSI_F32;
    }
    if (sp.height <= 0 || sp.width <= 0 || sp.bands <= 0 || sp.bands > HSI_MAX_BANDS) return HSI_E_INVALID;
    if (sp.dtype != HSI_F32 && sp.dtype != HSI_F16) return HSI_E_INVALID;
    if (!sp.targets || sp.num_targets < 1 || sp.num_targets > HSI_MAX_FILTERS_PER_PASS) return HSI_E_INVALID;
    if (!sp.raw && !sp.cube) return HSI_E_INVALID;
    f.P = static_cast<int64_t>(sp.height) * sp.width;
    f.stride = hsi_plane_stride(sp.height, sp.width);
    const int B = sp.bands, T = sp.num_targets;
    int rc = HSI_OK;
    if (sp.raw) {
      float* c = nullptr;
      rc = bt->alloc(&c, static_cast<size_t>(f.stride) * B);
      f.cube = c;
    } else {
      f.cube = const_cast<void*>(sp.cube);
    }
    if (rc == HSI_OK) rc = bt->alloc(&f.targets, static_cast<size_t>(T) * B);
    if (rc == HSI_OK) rc = bt->alloc(&f.norms, T);
    if (rc == HSI_OK) rc = bt->alloc(&f.moments, B + static_cast<size_t>(B) * B + 1);
    if (rc == HSI_OK) rc = bt->alloc(&f.stats64, hsi_statistics_elements(B, T));
    if (rc == HSI_OK) rc = bt->alloc(&f.status, 1);
    if (rc == HSI_OK) rc = bt->alloc(&f.sam_best, f.P);
    if (rc == HSI_OK) rc = bt->alloc(&f.sam_target, f.P);
    if (rc == HSI_OK) rc = bt->alloc(&f.rx, f.P);
    if (rc == HSI_OK) rc = bt->alloc(&f.ace_best, f.P);
    if (rc == HSI_OK) rc = bt->alloc(&f.ace_target, f.P);
    for (int k = 0; k < 3 && rc == HSI_OK; ++k) rc = bt->alloc(&f.dets[k], std::max(o.capacity, 1));
    if (rc != HSI_OK) return rc;
    // library and its norms (FP64 accumulation, as the reference's SpectralLibrary::norms)
    std::vector<float> norms(T);
    for (int t = 0; t < T; ++t) {
      double s = 0.0;
      for (int b = 0; b < B; ++b) s += static_cast<double>(sp.targets[t * B + b]) * sp.targets[t * B + b];
      norms[t] = static_cast<float>(std::sqrt(s));
    }
    cudaError_t e = cudaMemcpy(f.targets, sp.targets, sizeof(float) * T * B, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(f.norms, norms.data(), sizeof(float) * T, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return static_cast<int>(e);
    f.rx_threshold = static_cast<float>(hsi::rx_threshold_for_false_alarm_rate(B, o.rx_false_alarm_rate));
    f.tensor_core_rx = B <= 127;
    hsi_moments_job mj;
    std::memset(&mj, 0, sizeof(mj));
    mj.cube = f.cube;
    mj.plane_stride = f.stride;
    mj.moments = f.moments;
    mj.height = sp.height;
    mj.width = sp.width;
    mj.bands = B;
    mj.dtype = sp.dtype;
    bt->moment_jobs.push_back(mj);
    bt->factor_bytes = std::max(bt->factor_bytes, hsi_factor_workspace_bytes(1, B));
    rx_bytes = std::max(rx_bytes, std::max(hsi_rx_ace_workspace_bytes(B, T), hsi_rx_ace_simt_workspace_bytes(B, T)));
    hsi_frame hf;
    std::memset(&hf, 0, sizeof(hf));
    hf.cube = f.cube;
    hf.plane_stride = f.stride;
    hf.height = sp.height;
    hf.width = sp.width;
    hf.bands = B;
    hf.dtype = sp.dtype;
    hf.sam_targets = f.targets;
    hf.sam_norms = f.norms;
    hf.num_sam = T;
    hf.sam_best = f.sam_best;
    hf.sam_best_target = f.sam_target;
    hf.map_stride = f.P;
    tables[sp.dtype].push_back(hf);
    bt->table_bands[sp.dtype] = std::max(bt->table_bands[sp.dtype], B);
    bt->table_targets[sp.dtype] = std::max(bt->table_targets[sp.dtype], T);
  }
  int rc = bt->alloc(&bt->all_counts, 3 * static_cast<size_t>(n));
  if (rc == HSI_OK) rc = bt->alloc(&bt->score_status, 1);
  for (int d = 0; d < 2 && rc == HSI_OK; ++d) {
    bt->table_n[d] = static_cast<int>(tables[d].size());
    if (!bt->table_n[d]) continue;
    if (bt->table_n[d] > HSI_MAX_TABLE_FRAMES) return HSI_E_CAPACITY;
    rc = bt->alloc(&bt->table[d], tables[d].size());
    if (rc == HSI_OK)
      rc = static_cast<int>(
          cudaMemcpy(bt->table[d], tables[d].data(), sizeof(hsi_frame) * tables[d].size(), cudaMemcpyHostToDevice));
  }
  if (rc != HSI_OK) return rc;
  // detection jobs: SAM (lower is better), ACE, RX (higher is better)
  for (int i = 0; i < n; ++i) {
    Frame& f = bt->frames[i];
    f.counts = bt->all_counts + 3 * i;
    const float* maps[3] = {f.sam_best, f.ace_best, f.rx};
    const int32_t* ids[3] = {f.sam_target, f.ace_target, nullptr};
    const float thr[3] = {o.sam_threshold, o.ace_threshold, f.rx_threshold};
    for (int k = 0; k < 3; ++k) {
      hsi_detect_job j;
      j.score = maps[k];
      j.target = ids[k];
      j.height = f.spec.height;
      j.width = f.spec.width;
      j.threshold = thr[k];
      j.nms_radius = o.nms_radius;
      j.polarity = k == 0 ? HSI_LOWER_IS_BETTER : HSI_HIGHER_IS_BETTER;
      j.capacity = o.capacity;
      j.out = f.dets[k];
      j.count = f.counts + k;
      bt->jobs.push_back(j);
    }
  }
  for (size_t j0 = 0; j0 < bt->jobs.size(); j0 += HSI_MAX_DETECT_JOBS) {
    const int m = static_cast<int>(std::min<size_t>(HSI_MAX_DETECT_JOBS, bt->jobs.size() - j0));
    bt->det_bytes = std::max(bt->det_bytes, hsi_detect_batch_workspace_bytes(&bt->jobs[j0], m));
  }
  bt->rx_bytes = rx_bytes;
  bt->stats_bytes = hsi_scene_moments_batch_workspace_bytes(bt->moment_jobs.data(), n);
  unsigned char* p = nullptr;
  rc = bt->alloc(&p, std::max<size_t>(bt->stats_bytes, 256));
  bt->stats_ws = p;
  for (int l = 0; l < hsi_batch::kLanes && rc == HSI_OK; ++l) {
    rc = bt->alloc(&p, std::max<size_t>(bt->factor_bytes, 256));
    bt->factor_ws[l] = p;
    if (rc == HSI_OK) rc = bt->alloc(&p, std::max<size_t>(bt->rx_bytes, 256));
    bt->rx_ws[l] = p;
  }
  if (rc == HSI_OK) rc = bt->alloc(&p, std::max<size_t>(bt->det_bytes, 256));
  bt->det_ws = p;
  if (rc == HSI_OK) rc = bt->make_lanes();
  // Frames to lanes, largest chain first onto the least loaded lane; the cost
  // of a chain is its RX/ACE arithmetic, pixels x bands x (bands + targets).
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  auto cost = [&](int i) {
    const hsi_batch_frame& sp = bt->frames[i].spec;
    return static_cast<double>(bt->frames[i].P) * sp.bands * (sp.bands + sp.num_targets);
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
  bt->lane_of.assign(n, 0);
  double load[hsi_batch::kLanes] = {};
  for (int i : order) {
    int l = 0;
    for (int k = 1; k < hsi_batch::kLanes; ++k)
      if (load[k] < load[l]) l = k;
    bt->lane_of[i] = l;
    load[l] += cost(i);
  }
  return rc;
}

// Time the tunable choices on the batch: the persistent scorer's CTAs per SM
// and, for frames the tensor-core path can take, tensor-core vs plain RX/ACE.
int autotune(hsi_batch* bt) {
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return HSI_E_INVALID;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, s);
  int rc = bt->run(s);  // warm-up: first-use set-up of every kernel, statistics for the RX timings
  float best = 1e30f;
  const int candidates[] = {1, 2, 3, 0};
  for (int c : candidates) {
    if (rc != HSI_OK) break;
    const float ms = time_ms([&] { return bt->score(c, s); }, 3, s, &rc);
    if (rc == HSI_OK && ms < best) {
      best = ms;
      bt->score_ctas_per_sm = c;
    }
  }
  for (Frame& f : bt->frames) {
    if (rc != HSI_OK || f.spec.bands > 127) continue;
    rc = bt->rx_ace(f, true, 0, s);  // warm
    const float tc = time_ms([&] { return bt->rx_ace(f, true, 0, s); }, 2, s, &rc);
    const float plain = time_ms([&] { return bt->rx_ace(f, false, 0, s); }, 2, s, &rc);
    f.tensor_core_rx = tc <= plain;
  }
  cudaEventRecord(b, s);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(&bt->tuning_ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamDestroy(s);
  return rc;
}

}  // namespace

extern "C" HSI_API hsi_batch* hsi_batch_create(const hsi_batch_frame* frames, int num_frames,
                                               const hsi_batch_options* options, int* status) {
  int rc = HSI_OK;
  hsi_batch* bt = nullptr;
  if (!frames || num_frames <= 0 || !options || options->capacity < 0 || options->nms_radius < 0 ||
      !(options->rx_false_alarm_rate > 0.0 && options->rx_false_alarm_rate < 1.0) || !(options->loading >= 0.0)) {
    rc = HSI_E_INVALID;
  } else {
    bt = new (std::nothrow) hsi_batch();
    if (!bt) rc = HSI_E_INVALID;
  }
  if (bt) {
    bt->opt = *options;
    rc = build(bt, frames, num_frames);
    if (rc == HSI_OK && options->autotune) rc = autotune(bt);
    if (rc != HSI_OK) {
      delete bt;
      bt = nullptr;
    }
  }
  if (status) *status = rc;
  return bt;
}

extern "C" HSI_API int hsi_batch_run(hsi_batch* batch, hsi_stream_t stream) {
  if (!batch) return HSI_E_INVALID;
  return batch->run(reinterpret_cast<cudaStream_t>(stream));
}

extern "C" HSI_API int hsi_batch_capture(hsi_batch* batch, hsi_stream_t stream) {
  if (!batch || !stream) return HSI_E_INVALID;  // the legacy default stream cannot be captured
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (batch->exec) {
    cudaGraphExecDestroy(batch->exec);
    batch->exec = nullptr;
  }
  if (batch->graph) {
    cudaGraphDestroy(batch->graph);
    batch->graph = nullptr;
  }
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return static_cast<int>(e);
  const int rc = batch->run(s);
  e = cudaStreamEndCapture(s, &batch->graph);
  if (rc != HSI_OK) return rc;
  if (e != cudaSuccess) return static_cast<int>(e);
  e = cudaGraphInstantiate(&batch->exec, batch->graph, 0);
  return static_cast<int>(e);
}

extern "C" HSI_API int hsi_batch_launch(hsi_batch* batch, hsi_stream_t stream) {
  if (!batch || !batch->exec) return HSI_E_INVALID;
  return static_cast<int>(cudaGraphLaunch(batch->exec, reinterpret_cast<cudaStream_t>(stream)));
}

extern "C" HSI_API int hsi_batch_outputs_of(const hsi_batch* batch, int frame, hsi_batch_outputs* out) {
  if (!batch || !out || frame < 0 || frame >= static_cast<int>(batch->frames.size())) return HSI_E_INVALID;
  const Frame& f = batch->frames[frame];
  out->sam_best = f.sam_best;
  out->sam_target = f.sam_target;
  out->rx = f.rx;
  out->ace_best = f.ace_best;
  out->ace_target = f.ace_target;
  for (int k = 0; k < 3; ++k) out->detections[k] = f.dets[k];
  out->counts = f.counts;
  out->status = f.status;
  out->rx_threshold = f.rx_threshold;
  return HSI_OK;
}

extern "C" HSI_API int hsi_batch_tuning_of(const hsi_batch* batch, hsi_batch_tuning* out) {
  if (!batch || !out) return HSI_E_INVALID;
  out->score_ctas_per_sm = batch->score_ctas_per_sm;
  out->tensor_core_rx_frames = 0;
  out->plain_rx_frames = 0;
  for (const Frame& f : batch->frames) (f.tensor_core_rx ? out->tensor_core_rx_frames : out->plain_rx_frames)++;
  out->tuning_ms = batch->tuning_ms;
  return HSI_OK;
}

extern "C" HSI_API void hsi_batch_destroy(hsi_batch* batch) { delete batch; }
