// The lagged-statistics video runner behind include/hsi_lagged.h: frame k is
// scored with frame k-1's statistics on the caller's stream while frame k's
// own moments and FP64 statistics are built on an internal stream.
#include "hsi_lagged.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "hsi/detectors.hpp"

struct hsi_lagged {
  hsi_lagged_options opt{};
  std::vector<float> host_targets;
  int64_t P = 0, stride = 0;
  size_t stats_elems = 0;
  cudaStream_t side = nullptr;  // moments + factorisation of the frame being scored
  cudaEvent_t cube_ready = nullptr, moments_read = nullptr;
  cudaEvent_t stats_done[2] = {nullptr, nullptr}, score_done[2] = {nullptr, nullptr};
  std::vector<void*> allocations;
  float* targets = nullptr;
  float* norms = nullptr;
  // two statistics buffers: the one scoring the current frame, the one being built
  double* moments[2] = {nullptr, nullptr};
  double* stats64[2] = {nullptr, nullptr};
  float* stats32[2] = {nullptr, nullptr};
  float* cem[2] = {nullptr, nullptr};
  int32_t* status[2] = {nullptr, nullptr};
  void* stats_ws = nullptr;
  size_t stats_bytes = 0;
  void* factor_ws = nullptr;
  size_t factor_bytes = 0;
  void* rx_ws = nullptr;
  size_t rx_bytes = 0;
  void* det_ws = nullptr;
  size_t det_bytes = 0;
  float *sam_maps = nullptr, *sam_best = nullptr, *cem_maps = nullptr, *cem_best = nullptr;
  int32_t *sam_target = nullptr, *cem_target = nullptr, *ace_target = nullptr;
  float *rx = nullptr, *ace_maps = nullptr, *ace_best = nullptr;
  hsi_detection* dets[4] = {nullptr, nullptr, nullptr, nullptr};
  uint32_t* counts = nullptr;
  std::vector<hsi_detect_job> jobs;
  float rx_threshold = 0.0f;
  bool tensor_rx = false;
  int64_t pushed = 0;
  int cur = 0;  // statistics buffer that scores the next frame

  ~hsi_lagged() {
    if (side) cudaStreamSynchronize(side);
    for (void* p : allocations) cudaFree(p);
    for (cudaEvent_t e : {cube_ready, moments_read, stats_done[0], stats_done[1], score_done[0], score_done[1]})
      if (e) cudaEventDestroy(e);
    if (side) cudaStreamDestroy(side);
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

  bool sam_cem() const { return (opt.detectors & HSI_LAGGED_SAM_CEM) != 0; }
  bool rx_ace() const { return (opt.detectors & HSI_LAGGED_RX_ACE) != 0; }

  // Moments of `cube` (shifted by `reference`, nullable) and its FP64
  // statistics into buffer b, on stream s.
  int statistics(const void* cube, const float* reference, int b, cudaStream_t s) {
    const hsi_stream_t hs = reinterpret_cast<hsi_stream_t>(s);
    int rc = hsi_scene_moments(cube, opt.height, opt.width, opt.bands, opt.dtype, stride, moments[b], reference,
                               stats_ws, stats_bytes, hs);
    if (rc != HSI_OK) return rc;
    if (s == side && cudaEventRecord(moments_read, s) != cudaSuccess) return HSI_E_INVALID;
    rc = hsi_build_statistics(1, opt.bands, opt.num_targets, opt.loading, moments[b], targets, 0, stats64[b],
                              stats32[b], cem[b], status[b], factor_ws, factor_bytes, hs);
    return rc;
  }

  // Maps and lists of `cube` from statistics buffer b, on stream s.
  int score(const void* cube, int b, cudaStream_t s) {
    const hsi_stream_t hs = reinterpret_cast<hsi_stream_t>(s);
    if (sam_cem()) {
      hsi_frame f;
      std::memset(&f, 0, sizeof(f));
      f.cube = cube;
      f.plane_stride = stride;
      f.height = opt.height;
      f.width = opt.width;
      f.bands = opt.bands;
      f.dtype = opt.dtype;
      f.sam_targets = targets;
      f.sam_norms = norms;
      f.num_sam = opt.num_targets;
      f.cem_weights = cem[b];
      f.num_cem = opt.num_targets;
      f.sam_maps = sam_maps;
      f.sam_best = sam_best;
      f.sam_best_target = sam_target;
      f.cem_maps = cem_maps;
      f.cem_best = cem_best;
      f.cem_best_target = cem_target;
      f.map_stride = P;
      const int rc = hsi_score_frames(&f, 1, hs);
      if (rc != HSI_OK) return rc;
    }
    if (rx_ace()) {
      const auto fn = tensor_rx ? hsi_rx_ace : hsi_rx_ace_simt;
      const int rc = fn(cube, opt.height, opt.width, opt.bands, opt.dtype, stride, stats64[b], opt.num_targets, rx,
                        ace_best, ace_target, ace_maps, P, rx_ws, rx_bytes, hs);
      if (rc != HSI_OK) return rc;
    }
    if (cudaMemsetAsync(counts, 0, 4 * sizeof(uint32_t), s) != cudaSuccess) return HSI_E_INVALID;
    return hsi_detect_batch(jobs.data(), static_cast<int>(jobs.size()), det_ws, det_bytes, hs);
  }

  int push(const void* cube, cudaStream_t s) {
    if (pushed == 0) {
      // frame 0: its own statistics, then its maps
      int rc = statistics(cube, nullptr, 0, s);
      if (rc == HSI_OK) rc = score(cube, 0, s);
      if (rc != HSI_OK) return rc;
      if (cudaEventRecord(score_done[0], s) != cudaSuccess) return HSI_E_INVALID;
      cur = 0;
      ++pushed;
      return HSI_OK;
    }
    const int nb = 1 - cur;
    // side stream: frame k's moments shifted by frame k-1's mean, and its statistics
    cudaError_t e = cudaEventRecord(cube_ready, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side, cube_ready, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side, score_done[nb], 0);  // buffer nb's last reader
    if (e != cudaSuccess) return static_cast<int>(e);
    // the tensor-core moments take a caller's shift at up to 127 bands; wider
    // frames keep their own (their moments are exact either way)
    const float* shift = opt.bands <= 127 ? stats32[cur] : nullptr;
    int rc = statistics(cube, shift, nb, side);
    if (rc != HSI_OK) return rc;
    e = cudaEventRecord(stats_done[nb], side);
    // caller's stream: frame k's maps and lists from frame k-1's statistics
    if (e == cudaSuccess && pushed >= 2) e = cudaStreamWaitEvent(s, stats_done[cur], 0);
    if (e != cudaSuccess) return static_cast<int>(e);
    rc = score(cube, cur, s);
    if (rc != HSI_OK) return rc;
    e = cudaEventRecord(score_done[cur], s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, moments_read, 0);  // the cube is read on both streams
    if (e != cudaSuccess) return static_cast<int>(e);
    cur = nb;
    ++pushed;
    return HSI_OK;
  }

  int create(const hsi_lagged_options& o) {
    opt = o;
    P = static_cast<int64_t>(o.height) * o.width;
    stride = hsi_plane_stride(o.height, o.width);
    const int B = o.bands, T = o.num_targets;
    host_targets.assign(o.targets, o.targets + static_cast<size_t>(T) * B);
    hsi::SpectralLibrary lib;
    for (int t = 0; t < T; ++t) {
      hsi::Spectrum sp;
      sp.values.assign(host_targets.begin() + static_cast<size_t>(t) * B,
                       host_targets.begin() + static_cast<size_t>(t + 1) * B);
      lib.targets.push_back(sp);
    }
    const std::vector<float> n = lib.norms();
    stats_elems = hsi_statistics_elements(B, T);
    int rc;
    if ((rc = alloc(&targets, static_cast<size_t>(T) * B)) != HSI_OK) return rc;
    if ((rc = alloc(&norms, T)) != HSI_OK) return rc;
    for (int b = 0; b < 2; ++b) {
      if ((rc = alloc(&moments[b], B + static_cast<size_t>(B) * B + 1)) != HSI_OK) return rc;
      if ((rc = alloc(&stats64[b], stats_elems)) != HSI_OK) return rc;
      if ((rc = alloc(&stats32[b], stats_elems)) != HSI_OK) return rc;
      if ((rc = alloc(&cem[b], static_cast<size_t>(T) * B)) != HSI_OK) return rc;
      if ((rc = alloc(&status[b], 1)) != HSI_OK) return rc;
    }
    if (cudaMemcpy(targets, host_targets.data(), sizeof(float) * T * B, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(norms, n.data(), sizeof(float) * T, cudaMemcpyHostToDevice) != cudaSuccess)
      return HSI_E_INVALID;
    stats_bytes = hsi_stats_workspace_bytes(o.height, o.width, B);
    factor_bytes = hsi_factor_workspace_bytes(1, B);
    unsigned char* w = nullptr;
    if ((rc = alloc(&w, stats_bytes)) != HSI_OK) return rc;
    stats_ws = w;
    if ((rc = alloc(&w, factor_bytes)) != HSI_OK) return rc;
    factor_ws = w;
    const size_t mp = static_cast<size_t>(T) * P;
    if (sam_cem()) {
      if ((rc = alloc(&sam_maps, mp)) != HSI_OK || (rc = alloc(&sam_best, P)) != HSI_OK ||
          (rc = alloc(&sam_target, P)) != HSI_OK || (rc = alloc(&cem_maps, mp)) != HSI_OK ||
          (rc = alloc(&cem_best, P)) != HSI_OK || (rc = alloc(&cem_target, P)) != HSI_OK)
        return rc;
    }
    if (rx_ace()) {
      tensor_rx = B <= 127;
      rx_bytes = tensor_rx ? hsi_rx_ace_workspace_bytes(B, T) : hsi_rx_ace_simt_workspace_bytes(B, T);
      if ((rc = alloc(&w, rx_bytes)) != HSI_OK) return rc;
      rx_ws = w;
      if ((rc = alloc(&rx, P)) != HSI_OK || (rc = alloc(&ace_maps, mp)) != HSI_OK ||
          (rc = alloc(&ace_best, P)) != HSI_OK || (rc = alloc(&ace_target, P)) != HSI_OK)
        return rc;
      rx_threshold = static_cast<float>(hsi::rx_threshold_for_false_alarm_rate(B, o.rx_false_alarm_rate));
    }
    const int cap = std::max(o.capacity, 1);
    for (int l = 0; l < 4; ++l)
      if ((rc = alloc(&dets[l], cap)) != HSI_OK) return rc;
    if ((rc = alloc(&counts, 4)) != HSI_OK) return rc;
    auto job = [&](const float* score, const int32_t* target, float thr, int polarity, int l) {
      hsi_detect_job j;
      j.score = score;
      j.target = target;
      j.height = o.height;
      j.width = o.width;
      j.threshold = thr;
      j.nms_radius = o.nms_radius;
      j.polarity = polarity;
      j.capacity = o.capacity;
      j.out = dets[l];
      j.count = counts + l;
      jobs.push_back(j);
    };
    if (sam_cem()) {
      job(sam_best, sam_target, o.sam_threshold, HSI_LOWER_IS_BETTER, 0);
      job(cem_best, cem_target, o.cem_threshold, HSI_HIGHER_IS_BETTER, 1);
    }
    if (rx_ace()) {
      job(ace_best, ace_target, o.ace_threshold, HSI_HIGHER_IS_BETTER, 2);
      job(rx, nullptr, rx_threshold, HSI_HIGHER_IS_BETTER, 3);
    }
    det_bytes = hsi_detect_batch_workspace_bytes(jobs.data(), static_cast<int>(jobs.size()));
    if ((rc = alloc(&w, det_bytes)) != HSI_OK) return rc;
    det_ws = w;
    if (cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) != cudaSuccess) return HSI_E_INVALID;
    for (cudaEvent_t* e : {&cube_ready, &moments_read, &stats_done[0], &stats_done[1], &score_done[0], &score_done[1]})
      if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return HSI_E_INVALID;
    return HSI_OK;
  }
};

extern "C" HSI_API hsi_lagged* hsi_lagged_create(const hsi_lagged_options* o, int* status) {
  auto fail = [&](int st) -> hsi_lagged* {
    if (status) *status = st;
    return nullptr;
  };
  if (!o || !o->targets || o->height <= 0 || o->width <= 0 || o->bands <= 0 || o->bands > HSI_MAX_BANDS ||
      o->num_targets < 1 || o->num_targets > HSI_MAX_FILTERS_PER_PASS || o->capacity < 0 || o->nms_radius < 0 ||
      (o->dtype != HSI_F32 && o->dtype != HSI_F16) ||
      (o->detectors & (HSI_LAGGED_SAM_CEM | HSI_LAGGED_RX_ACE)) == 0 || (o->detectors & ~3) != 0 ||
      !(o->loading >= 0.0))
    return fail(HSI_E_INVALID);
  if ((o->detectors & HSI_LAGGED_RX_ACE) && !(o->rx_false_alarm_rate > 0.0 && o->rx_false_alarm_rate < 1.0))
    return fail(HSI_E_INVALID);
  hsi_lagged* r = new (std::nothrow) hsi_lagged();
  if (!r) return fail(HSI_E_INVALID);
  const int rc = r->create(*o);
  if (rc != HSI_OK) {
    delete r;
    return fail(rc);
  }
  if (status) *status = HSI_OK;
  return r;
}

extern "C" HSI_API int hsi_lagged_push(hsi_lagged* r, const void* d_cube, hsi_stream_t stream) {
  if (!r || !d_cube || (reinterpret_cast<uintptr_t>(d_cube) & 15u) != 0) return HSI_E_INVALID;
  return r->push(d_cube, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" HSI_API int hsi_lagged_outputs_of(const hsi_lagged* r, hsi_lagged_outputs* out) {
  if (!r || !out) return HSI_E_INVALID;
  std::memset(out, 0, sizeof(*out));
  out->frame = r->pushed - 1;
  out->statistics_frame = r->pushed <= 1 ? 0 : r->pushed - 2;
  out->sam_maps = r->sam_maps;
  out->sam_best = r->sam_best;
  out->sam_target = r->sam_target;
  out->cem_maps = r->cem_maps;
  out->cem_best = r->cem_best;
  out->cem_target = r->cem_target;
  out->rx = r->rx;
  out->ace_maps = r->ace_maps;
  out->ace_best = r->ace_best;
  out->ace_target = r->ace_target;
  for (int l = 0; l < 4; ++l) out->detections[l] = r->dets[l];
  out->counts = r->counts;
  // the buffer that scored the last frame: the current one after frame 0,
  // the other one afterwards (cur flips at each later push)
  out->status = r->status[r->pushed <= 1 ? 0 : 1 - r->cur];
  out->map_stride = r->P;
  out->rx_threshold = r->rx_threshold;
  return HSI_OK;
}

extern "C" HSI_API void hsi_lagged_destroy(hsi_lagged* r) { delete r; }
