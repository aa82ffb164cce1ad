/*
 * hsi_b200.h - C ABI of the B200 (sm_100a) hyperspectral detection library.
 *
 * Everything the reference exposes for its per-frame detection path
 * (include/hsi/sam_cuda.hpp, detect_cuda.hpp, stats_cuda.hpp, detector.hpp,
 * detectors.hpp in GokulEdakkePuram/hsi-detectors-cuda) is reachable through
 * these plain-C entry points: plain pointers and sizes, no C++ or CUDA types
 * in the signatures (a stream is the CUDA runtime's opaque stream handle).
 * The C++ drop-in layer in include/hsi/ is implemented on top of them.
 *
 * Conventions
 *  - Cubes are band-sequential (BSQ): element (band b, pixel p) lives at
 *    cube[b * plane_stride + p], p = y * width + x.
 *  - Every device buffer is owned by the caller.  Entry points that need
 *    scratch say so and take it as an explicit workspace argument.
 *  - Every entry point returns an int status: 0 on success, a CUDA runtime
 *    error code (1..9999) when the runtime reported one, or an HSI_E_* code.
 *    Invalid arguments return 1 (cudaErrorInvalidValue), as the reference's
 *    launchers do (src/sam.cu:376,384,392; src/detect.cu:95-97).
 *  - All launches are asynchronous on the given stream unless stated.
 */
#ifndef HSI_B200_H
#define HSI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define HSI_API __declspec(dllexport)
#else
#define HSI_API __attribute__((visibility("default")))
#endif

/* ABI-compatible with cudaStream_t. */
typedef struct CUstream_st* hsi_stream_t;

/* ---- status codes -------------------------------------------------------- */
#define HSI_OK 0
#define HSI_E_INVALID 1             /* == cudaErrorInvalidValue */
#define HSI_E_NOT_POSITIVE_DEFINITE 10001 /* the scene covariance failed to factor */
#define HSI_E_TIMEOUT 10002         /* a bounded device-side wait gave up */
#define HSI_E_WORKSPACE 10003       /* workspace missing or too small */
#define HSI_E_CAPACITY 10004        /* a size exceeds a documented maximum */
#define HSI_E_NO_DEVICE 10005
#define HSI_E_CORRELATION_NOT_PD 10006 /* the CEM autocorrelation failed to factor */
#define HSI_E_EMPTY 10007              /* no pixels accumulated */

/* ---- element types of a cube --------------------------------------------- */
#define HSI_F32 0
#define HSI_F16 1

/* Score polarity (reference: include/hsi/types.hpp:108-117). */
#define HSI_LOWER_IS_BETTER 0
#define HSI_HIGHER_IS_BETTER 1

/* Limits of the scoring kernels. */
#define HSI_MAX_BANDS 256
#define HSI_MAX_FILTERS_PER_PASS 16 /* per kind (SAM, CEM) and pass over the cube */

/* One detection, 16 bytes, same layout as hsi::Detection
 * (reference include/hsi/types.hpp:101-106). */
typedef struct hsi_detection {
  int32_t x;
  int32_t y;
  int32_t target;
  float score;
} hsi_detection;

/* Human-readable text for a status code. */
HSI_API const char* hsi_status_string(int status);

/* Library version as 10000*major + 100*minor + patch. */
HSI_API int hsi_version(void);

/*
 * Plane stride, in elements, of a device BSQ cube: pixels rounded up to a
 * multiple of 32, so every band plane starts on a 128-byte boundary and can
 * be staged by the TMA engine.  Replaces hsi::bsq_plane_stride
 * (reference include/hsi/sam_cuda.hpp:47, src/sam.cu:338-343, which rounds
 * to 8).
 */
HSI_API int64_t hsi_plane_stride(int height, int width);

/* ---- synthetic scenes ------------------------------------------------------
 * The scene model of csrc/synth.h (Dirichlet-mixed endmembers, implanted
 * targets, anomalies, Gaussian noise).  Stands in for the reference's
 * synthetic FrameSource (src/frame_source.cpp:149-293) with the distribution
 * the benchmark configurations specify.
 */
typedef struct hsi_scene {
  int32_t bands;
  int32_t n_end;          /* background endmembers, 1..8 */
  int32_t n_targets;      /* implanted library size, 0..64 */
  float target_frac;      /* per-target implant probability per pixel */
  float anomaly_frac;     /* anomaly probability per pixel */
  float noise_sigma;
  uint64_t library_seed;  /* spectra */
  uint64_t frame_seed;    /* per-pixel draws */
} hsi_scene;

/* Host: the scene's spectra, each `bands` floats: n_end endmembers, then
 * n_targets targets, then one anomaly spectrum ((n_end + n_targets + 1) * bands
 * floats in total). */
HSI_API int hsi_scene_spectra(const hsi_scene* scene, float* out);

/* Device: generate pixels [pixel0, pixel0 + height*width) of a frame into a
 * BSQ cube of element type `dtype` with plane stride `plane_stride`.
 * `d_spectra` is the output of hsi_scene_spectra copied to the device.
 * `d_truth` (nullable) receives one label byte per pixel: 0 background,
 * 1 + t for target t, 255 for an anomaly. */
HSI_API int hsi_generate(const hsi_scene* scene, const float* d_spectra, int height, int width,
                         int64_t pixel0, void* d_cube, int dtype, int64_t plane_stride,
                         uint8_t* d_truth, hsi_stream_t stream);

/* ---- filter-bank scoring (SAM and CEM) --------------------------------------
 * One streaming pass over a BSQ cube scores every pixel against a bank of
 * up to 16 SAM targets and 16 CEM filters at once.  Replaces
 * hsi::launch_sam_best (reference include/hsi/sam_cuda.hpp:91-96,
 * src/sam.cu:371-461) and adds CEM scoring on the device (the reference has
 * CEM only on the CPU: src/detectors_cpu.cpp:158-187).
 *
 * SAM: angle_t = acos(clamp(x.r_t / (|x| |r_t|), -1, 1)); a pixel or target
 *      with zero norm scores pi/2; best = smallest angle, lowest t on ties.
 * CEM: response_t = w_t . x on the uncentred pixel; best = largest response,
 *      lowest t on ties.
 *
 * Frames with more targets than one pass holds are scored in several passes
 * (the best-so-far is carried in the outputs), exactly like the reference's
 * multi-pass launcher.
 */
typedef struct hsi_frame {
  const void* cube;         /* device BSQ cube */
  int64_t plane_stride;     /* elements, multiple of 8, >= height*width */
  int32_t height;
  int32_t width;
  int32_t bands;            /* 1..HSI_MAX_BANDS */
  int32_t dtype;            /* HSI_F32 or HSI_F16 */
  /* SAM library: target-major num_sam x bands, plus each target's L2 norm */
  const float* sam_targets;
  const float* sam_norms;
  int32_t num_sam;
  /* CEM filters: target-major num_cem x bands */
  int32_t num_cem;
  const float* cem_weights;
  /* outputs, each nullable */
  float* sam_maps;          /* num_sam maps, map t at sam_maps + t*map_stride */
  float* sam_best;          /* smallest angle per pixel */
  int32_t* sam_best_target;
  float* cem_maps;
  float* cem_best;
  int32_t* cem_best_target;
  int64_t map_stride;       /* elements between consecutive maps (>= pixels) */
} hsi_frame;

/* Score `num_frames` frames whose descriptors are in HOST memory.  Up to
 * HSI_MAX_INLINE_FRAMES frames travel inside the launch; more need
 * hsi_score_frames_device. */
#define HSI_MAX_INLINE_FRAMES 4
HSI_API int hsi_score_frames(const hsi_frame* frames, int num_frames, hsi_stream_t stream);

/* Any number of frames whose descriptors are on the HOST, element types
 * mixed, up to 64 per launch.  FP16 cubes of at most 128 bands are scored on
 * the tensor cores: the cube is fed by TMA straight into tcgen05.mma.kind::f16
 * (fp16 values are exact operands), each filter is scaled by a power of two
 * and split into an fp16 head and remainder (22 significant bits), FP32
 * accumulation.  Other frames take the FP32-FMA scorer.  Semantics, outputs
 * and `d_status` (nullable) as hsi_score_frames_device; hsi_score_frames
 * takes the same route for its frames. */
HSI_API int hsi_score_frames_batch(const hsi_frame* frames, int num_frames, int* d_status, hsi_stream_t stream);

/* Same for a descriptor table already in DEVICE memory: up to 256 frames of
 * uneven sizes, band counts and libraries in one persistent launch per pass.
 * Every frame must have element type `dtype`, at most `max_bands` bands,
 * `max_sam` SAM targets and `max_cem` CEM filters (they pick the kernel
 * instance); a frame outside those bounds is skipped and HSI_E_INVALID is
 * recorded in `*d_status` (a device int, nullable, left untouched on
 * success). */
#define HSI_MAX_TABLE_FRAMES 256
HSI_API int hsi_score_frames_device(const hsi_frame* d_frames, int num_frames, int dtype, int max_bands,
                                    int max_sam, int max_cem, int* d_status, hsi_stream_t stream);
/* The same with the persistent grid chosen by the caller: `ctas_per_sm`
 * CTAs per SM (0: as many as fit, the default above; larger values are
 * capped at what fits).  The autotuner's knob (hsi::BatchRunner). */
HSI_API int hsi_score_frames_device_grid(const hsi_frame* d_frames, int num_frames, int dtype, int max_bands,
                                         int max_sam, int max_cem, int* d_status, int ctas_per_sm,
                                         hsi_stream_t stream);

/* ---- scene statistics -------------------------------------------------------
 * Raw first and second moments of one frame.  Output `d_moments` (FP64):
 * sum[B], outer[B*B] (full symmetric), count -- the contents of
 * hsi::SpectralMoments.  Replaces the reference's launch_reset_moments /
 * launch_accumulate_mean / launch_accumulate_moments / read_moments
 * (include/hsi/stats_cuda.hpp:26-72, src/stats.cu:169-248) and
 * accumulate_moments_cpu (src/detectors_cpu.cpp:77-93).
 * Sums are taken about a per-band reference r near the mean (`d_reference`,
 * `bands` floats, e.g. the previous frame's mean; null: a subsample mean) and
 * rebuilt as raw moments in FP64.
 * Tensor-core path (bands <= 127, >= 32768 pixels): fixed-point (x - r) split
 * into signed 8-bit limbs, exact INT32 accumulation on tcgen05 (kind::i8),
 * FP64 reduction.  Otherwise the FP32 CUDA-core path below.
 */
HSI_API size_t hsi_stats_workspace_bytes(int height, int width, int bands);
HSI_API int hsi_scene_moments(const void* d_cube, int height, int width, int bands, int dtype,
                              int64_t plane_stride, double* d_moments, const float* d_reference,
                              void* d_workspace, size_t workspace_bytes, hsi_stream_t stream);
/* Same moments with plain FP32 CUDA-core arithmetic (register-blocked, FP32
 * sums over 32-pixel steps folded into FP64): the comparator for the
 * tensor-core path, and the path for small frames and bands >= 128. */
HSI_API int hsi_scene_moments_simt(const void* d_cube, int height, int width, int bands, int dtype,
                                   int64_t plane_stride, double* d_moments, const float* d_reference,
                                   void* d_workspace, size_t workspace_bytes, hsi_stream_t stream);
/* The tensor-core path at any frame size (bands <= 127, else HSI_E_CAPACITY). */
HSI_API int hsi_scene_moments_tc(const void* d_cube, int height, int width, int bands, int dtype,
                                 int64_t plane_stride, double* d_moments, const float* d_reference,
                                 void* d_workspace, size_t workspace_bytes, hsi_stream_t stream);

/* Moments of many frames at once: each job's output is what
 * hsi_scene_moments gives for that frame alone (the tensor path's sums are
 * exact integers until the final FP64 rebuild, so they do not depend on how
 * frames are grouped).  Frames on the tensor path are grouped by element type,
 * up to 64 per group, and each group runs as one launch sequence: a persistent
 * GEMM over all of the group's pixels plus one launch per small step for all
 * frames.  Other frames run one by one on the FP32 path.  Frames of any sizes
 * and band counts may be mixed.  The workspace serves one group at a time
 * (stream order), so its size does not grow past 64 tensor frames. */
typedef struct hsi_moments_job {
  const void* cube;        /* device BSQ cube, 16-byte aligned */
  int64_t plane_stride;    /* elements between band planes (>= height*width, multiple of 8) */
  double* moments;         /* out: B + B*B + 1 doubles */
  const float* reference;  /* nullable: `bands` floats, the shift r */
  int32_t height, width, bands, dtype;
} hsi_moments_job;
HSI_API size_t hsi_scene_moments_batch_workspace_bytes(const hsi_moments_job* jobs, int num_jobs);
HSI_API int hsi_scene_moments_batch(const hsi_moments_job* jobs, int num_jobs, void* d_workspace,
                                    size_t workspace_bytes, hsi_stream_t stream);

/* ---- detector statistics (FP64 factorisation) --------------------------------
 * For each of `num_frames` frames (moments contiguous, B + B*B + 1 doubles
 * each) build the statistics of reference build_statistics
 * (src/detector.cpp:47-152, include/hsi/detector.hpp:62-99) entirely in FP64
 * on the device: Cholesky of the loaded covariance and autocorrelation,
 * triangular inverse, whitened targets, CEM weights.  Packed layout per frame
 * (elements; hsi_statistics_elements gives the total):
 *   mean[B] | whitener[B*B] (row-major, upper zero) | target_white[T*B] |
 *   target_norm2[T] | cem_weight[T*B]
 * `d_stats64` receives it in FP64, `d_stats32` narrowed to float (the
 * reference's DetectorStatistics), `d_cem_weights` just the CEM filters
 * (T*B floats per frame) for the scorer; each nullable.  `d_library`: T*B
 * floats per frame at `library_stride` (0: one library for all frames).
 * `d_status[f]` (nullable) receives HSI_OK, HSI_E_NOT_POSITIVE_DEFINITE,
 * HSI_E_CORRELATION_NOT_PD or HSI_E_EMPTY.  Bands > 128 need a workspace of
 * hsi_factor_workspace_bytes.
 */
HSI_API size_t hsi_statistics_elements(int bands, int num_targets);
HSI_API size_t hsi_factor_workspace_bytes(int num_frames, int bands);
HSI_API int hsi_build_statistics(int num_frames, int bands, int num_targets, double loading,
                                 const double* d_moments, const float* d_library, int64_t library_stride,
                                 double* d_stats64, float* d_stats32, float* d_cem_weights, int* d_status,
                                 void* d_workspace, size_t workspace_bytes, hsi_stream_t stream);

/* ---- RX / ACE scoring ----------------------------------------------------------
 * RX = |W (x - mu)|^2 and ACE_t = (z . u_t)^2 / (|u_t|^2 |z|^2) for every
 * pixel, from the frame's packed FP64 statistics (hsi_build_statistics),
 * with the reference's rules: a target is skipped (ACE 0) when |u_t|^2 <= 0 or
 * |z|^2 <= 0; the best is the largest ACE, lowest t on ties, clamped to [0, 1];
 * score 0 and target -1 when no target is valid (reference rx_cpu /
 * ace_best_cpu, src/detectors_cpu.cpp:95-156; the reference has no GPU RX/ACE).
 * Outputs are each nullable: `d_rx` (P floats), `d_ace_best` (P), `d_ace_target`
 * (P int32), `d_ace_maps` (num_targets maps at `map_stride`).  At most 16
 * targets per call.
 */
/* Tensor-core path: the augmented whitener [W; (W^T u_t)^T] and the centred
 * pixels in exact fixed point (per-row and per-pixel power-of-two scales,
 * signed 8-bit limbs, tcgen05 INT8 MMAs into INT32), combined in FP32; error
 * against FP64 a few 1e-5 (RX relative to max(1, RX), ACE absolute) at 113
 * bands.  bands <= 127 (else HSI_E_CAPACITY); targets beyond 128 - bands per
 * pass take further passes over the cube, the best carried in the outputs.
 * Workspace: hsi_rx_ace_workspace_bytes (256-byte aligned). */
HSI_API size_t hsi_rx_ace_workspace_bytes(int bands, int num_targets);
HSI_API int hsi_rx_ace(const void* d_cube, int height, int width, int bands, int dtype, int64_t plane_stride,
                       const double* d_stats64, int num_targets, float* d_rx, float* d_ace_best,
                       int32_t* d_ace_target, float* d_ace_maps, int64_t map_stride, void* d_workspace,
                       size_t workspace_bytes, hsi_stream_t stream);
HSI_API size_t hsi_rx_ace_simt_workspace_bytes(int bands, int num_targets);
/* Plain FP32 CUDA-core path (register-blocked GEMM over [W; (W^T U)^T]). */
HSI_API int hsi_rx_ace_simt(const void* d_cube, int height, int width, int bands, int dtype,
                            int64_t plane_stride, const double* d_stats64, int num_targets, float* d_rx,
                            float* d_ace_best, int32_t* d_ace_target, float* d_ace_maps, int64_t map_stride,
                            void* d_workspace, size_t workspace_bytes, hsi_stream_t stream);

/* ---- detection compaction ---------------------------------------------------
 * Threshold + non-maximum suppression + compaction of one score map into a
 * detection list, in raster order.  Same semantics as the reference's CPU
 * detect_cpu (src/sam_cpu.cpp:86-138): a pixel is a candidate when
 * score <= threshold (lower is better) or score >= threshold (higher is
 * better); with nms_radius > 0 it is dropped when an in-bounds neighbour in
 * the (2r+1)^2 window is strictly better, or equal with a lower linear index.
 * Replaces hsi::launch_detect (reference include/hsi/detect_cuda.hpp:16-19,
 * src/detect.cu:43-106), whose output order is nondeterministic and which
 * ignores polarity on the GPU.
 *
 * `d_count` is read as the starting offset and receives that plus the number
 * of detections found (callers zero it first, as with the reference).  At
 * most `capacity` entries are written; detections past capacity are counted
 * but not written, and the ones kept are the first in raster order.
 * `d_target` may be null (target 0 is reported).
 */
HSI_API size_t hsi_detect_workspace_bytes(int height, int width);
HSI_API int hsi_detect(const float* d_score, const int32_t* d_target, int height, int width,
                       float threshold, int nms_radius, int polarity, int capacity,
                       hsi_detection* d_out, uint32_t* d_count, void* d_workspace,
                       size_t workspace_bytes, hsi_stream_t stream);

/* The same for up to 64 score maps in three launches (one per stage for the
 * whole batch).  Job descriptors live in host memory; the pointers in them
 * are device pointers. */
typedef struct hsi_detect_job {
  const float* score;
  const int32_t* target;     /* nullable */
  int32_t height;
  int32_t width;
  float threshold;
  int32_t nms_radius;
  int32_t polarity;
  int32_t capacity;
  hsi_detection* out;
  uint32_t* count;
} hsi_detect_job;
#define HSI_MAX_DETECT_JOBS 64
HSI_API size_t hsi_detect_batch_workspace_bytes(const hsi_detect_job* jobs, int num_jobs);
HSI_API int hsi_detect_batch(const hsi_detect_job* jobs, int num_jobs, void* d_workspace,
                             size_t workspace_bytes, hsi_stream_t stream);

/* ---- learned screen (no counterpart in the reference) --------------------------
 * A per-pixel MLP B -> 64 -> 32 -> 1 (ReLU; bfloat16 weights, FP32
 * accumulation) that proposes candidate pixels for the plain ACE detector,
 * which re-scores every proposal and stays the fallback.  Trained on the
 * device on the detector's own decisions by the kernels below.
 * Parameters (FP32 master copy), Bp = bands rounded up to 64:
 *   W1[64][Bp] | b1[64] | W2[32][64] | b2[32] | w3[32] | b3
 * Normaliser: 2*Bp floats, per band the mean and a power-of-two scale near
 * 1/sigma (zero past the bands).  Features: band-major [Bp][n] floats,
 * (x - mean) * scale rounded to bfloat16. */
HSI_API int64_t hsi_screen_param_count(int bands);
/* He-uniform weights from a counter hash (`seed`), zero biases. */
HSI_API int hsi_screen_init(float* d_params, int bands, uint64_t seed, hsi_stream_t stream);
/* Normaliser from a frame's raw FP64 moments (hsi_scene_moments). */
HSI_API int hsi_screen_normaliser(const double* d_moments, int bands, float* d_norm, hsi_stream_t stream);
/* Training batch of n pixel indices and 0/1 labels (score >= threshold): the
 * first `num_positive_draws` drawn from a positive list (e.g. hsi_detect of
 * the score map, radius 0), the rest uniform over the frame. */
HSI_API int hsi_screen_batch(const hsi_detection* d_positives, const uint32_t* d_positive_count,
                             int positive_capacity, int height, int width, const float* d_score, float threshold,
                             uint64_t seed, int num_positive_draws, int n, int32_t* d_index, float* d_labels,
                             hsi_stream_t stream);
/* Features of the indexed pixels, [Bp][n]. */
HSI_API int hsi_screen_gather(const void* d_cube, int dtype, int64_t plane_stride, int bands, const float* d_norm,
                              const int32_t* d_index, int n, float* d_features, hsi_stream_t stream);
/* Mean weighted binary cross-entropy on the logit (positives weighted by
 * pos_weight) and its gradient for every parameter (d_grads, param-count
 * floats); `d_loss` (nullable) receives the loss. */
HSI_API size_t hsi_screen_train_workspace_bytes(int bands, int n);
HSI_API int hsi_screen_gradients(const float* d_params, int bands, const float* d_features, const float* d_labels,
                                 int n, float pos_weight, float* d_grads, float* d_loss, void* d_workspace,
                                 size_t workspace_bytes, hsi_stream_t stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) at iteration `step` >= 1;
 * d_adam_state: 2 * param-count floats, zeroed before the first step. */
HSI_API int hsi_screen_adam(float* d_params, float* d_adam_state, const float* d_grads, int bands, float lr, int step,
                            hsi_stream_t stream);
/* Logit of every pixel of an fp16 cube (tcgen05: layers 1 and 2 on the
 * tensor cores, the cube read once by TMA as the first layer's operand).
 * Workspace: hsi_screen_infer_workspace_bytes, 256-byte aligned. */
HSI_API size_t hsi_screen_infer_workspace_bytes(int bands);
HSI_API int hsi_screen_infer(const void* d_cube, int height, int width, int bands, int dtype, int64_t plane_stride,
                             const float* d_norm, const float* d_params, float* d_logits, void* d_workspace,
                             size_t workspace_bytes, hsi_stream_t stream);
/* hsi_screen_infer on at most max_ctas CTAs (0: one per SM), the same logits.
 * The screen kernel is persistent, one CTA per SM; a caller that runs other
 * work beside it (the FP64 statistics, whose cluster of two CTAs the screen
 * does not need) caps it a few SMs short so both run at once.  No reference
 * counterpart (the screen is this library's). */
HSI_API int hsi_screen_infer_ctas(const void* d_cube, int height, int width, int bands, int dtype,
                                  int64_t plane_stride, const float* d_norm, const float* d_params, float* d_logits,
                                  void* d_workspace, size_t workspace_bytes, int max_ctas, hsi_stream_t stream);
/* Copy the spectra of candidate pixels (a detection list and its count) into
 * a compact BSQ cube of `capacity` pixels at `out_stride`, for re-scoring;
 * slots past the count hold pixel 0. */
HSI_API int hsi_gather_candidates(const void* d_cube, int dtype, int64_t plane_stride, int bands, int width,
                                  const hsi_detection* d_candidates, const uint32_t* d_count, int capacity,
                                  void* d_out, int64_t out_stride, hsi_stream_t stream);

/* ---- data formats ------------------------------------------------------------ */

/* fp32 -> fp16 (round to nearest even) of `count` elements; d_src 16-byte and
 * d_dst 8-byte aligned.  Replaces hsi::launch_narrow_to_half (reference
 * include/hsi/sam_cuda.hpp:108-109, src/sam.cu:311-316,476-482). */
HSI_API int hsi_narrow_to_half(const float* d_src, void* d_dst, int64_t count, hsi_stream_t stream);

/* BIP (pixel-major, `bands` floats per pixel) -> BSQ planes at `plane_stride`.
 * Replaces hsi::launch_transpose_bip_to_bsq (reference
 * include/hsi/sam_cuda.hpp:104-105, src/sam.cu:281-309,463-474), which writes
 * packed planes. */
HSI_API int hsi_transpose_bip_to_bsq(const float* d_src, float* d_dst, int height, int width, int bands,
                                     int64_t plane_stride, hsi_stream_t stream);

/* SAM of a BIP cube (pixel-major: `bands` floats per pixel, packed, 4-byte
 * aligned) in one pass, without a BSQ copy: the transpose is fused into the
 * scoring kernel.  Outputs as hsi_score_frames' SAM outputs (each nullable,
 * at least one given): d_maps (num_targets maps at map_stride), d_best (the
 * smallest angle), d_best_target (its index, lowest on ties); angles are
 * bit-identical to scoring the same cube in BSQ.  All 1..64 targets are
 * scored in one pass.  Replaces the reference's direct BIP scorer behind
 * launch_sam_best(SamVariant::BipDirect) (include/hsi/sam_cuda.hpp:91-96,
 * src/sam.cu:80-125,391-398). */
HSI_API int hsi_sam_bip(const float* d_cube, int height, int width, int bands, const float* d_targets,
                        const float* d_target_norms, int num_targets, float* d_maps, int64_t map_stride,
                        float* d_best, int32_t* d_best_target, hsi_stream_t stream);

/* Snapshot-mosaic demosaic on the device: raw frame (raw_height x raw_width
 * floats, row-major) -> BSQ cube of (raw_height/period) x (raw_width/period)
 * pixels and `bands` <= period^2 bands, element type `dtype`.  Band b takes
 * the mosaic position band_order[b] (HOST array, nullable: position b);
 * positions outside [0, period^2) return HSI_E_INVALID.  Same mapping as the
 * reference's demosaic (src/hot_loader.cpp:144-182). */
HSI_API int hsi_demosaic(const float* d_raw, int raw_height, int raw_width, int period, int bands,
                         const int32_t* band_order, void* d_cube, int dtype, int64_t plane_stride,
                         hsi_stream_t stream);

/* Add the sums about a reference spectrum, S1 = sum(x - r) and the lower
 * triangle (row-major, B*B buffer) of S2 = sum (x - r)(x - r)^T, of raw FP64
 * moments (hsi_scene_moments output) into the caller's accumulators.
 * `d_reference` nullable (r = 0).  Gives hsi_scene_moments the accumulate
 * contract of the reference's launch_accumulate_moments
 * (include/hsi/stats_cuda.hpp:52-55, src/stats.cu:169-248). */
HSI_API int hsi_accumulate_shifted_moments(const double* d_moments, const float* d_reference, int bands,
                                           double* d_sum, double* d_sum_outer, hsi_stream_t stream);

/* Allocation-free detection.  No counterpart in the reference: it is for
 * callers that cannot allocate device memory at all (for example a plug-in
 * that its host application hands only input and output buffers, the
 * application owning all device memory), so they cannot provide the
 * workspace hsi_detect needs.  Same arguments, semantics and results as
 * hsi_detect, without the workspace: the scratch is a 2.06 MiB array inside
 * the library's device image, which every GPU that loads the library holds
 * until the process exits.  Limits and rules:
 *  - height * ceil(width / 2048) must not exceed
 *    HSI_DETECT_NOALLOC_MAX_SEGMENTS (e.g. 8192 rows of up to 2048 pixels,
 *    or 4096 x 4096); larger maps return HSI_E_CAPACITY;
 *  - every call on a device shares that one array, so calls whose work
 *    overlaps on the GPU (on different streams, or from different host
 *    threads without ordering) race and corrupt each other's lists; calls on
 *    one stream are ordered and safe;
 *  - the scratch needs no clearing; as with hsi_detect, *d_count is the
 *    append offset the caller sets (normally zero) before the call;
 *  - the first call on each device does a one-time set-up (it looks up the
 *    array's device address in the current context and reads the detection
 *    kernels' residency), so that first call should come before any stream
 *    capture; the set-up runs again after the device's context is re-created
 *    (for example by cudaDeviceReset), since the array may then move.
 * It calls no allocating routine.  HSI_E_NO_DEVICE for device ordinals >= 64. */
#define HSI_DETECT_NOALLOC_MAX_SEGMENTS 8192
HSI_API int hsi_detect_noalloc(const float* d_score, const int32_t* d_target, int height, int width,
                               float threshold, int nms_radius, int polarity, int capacity,
                               hsi_detection* d_out, uint32_t* d_count, hsi_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* HSI_B200_H */
