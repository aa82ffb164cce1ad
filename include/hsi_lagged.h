/*
 * hsi_lagged.h - C ABI of the lagged-statistics video runner (libhsi_cxx.so).
 *
 * The reference names this mode without building it (include/hsi/linalg.hpp:
 * 79-83, "in the lagged pipeline mode the previous frame's mean is a free and
 * excellent reference"): in a video the scene statistics change slowly, so
 * frame k is scored with the statistics of frame k-1 -- its mean as the
 * moments' shift, its covariance / correlation as the RX, ACE and CEM filters
 * -- and the statistics pass leaves the per-frame critical path.
 *
 * Per pushed frame k >= 1, on two streams:
 *   caller's stream : SAM + CEM maps (one fused pass, CEM weights of frame
 *                     k-1), RX + ACE maps (whitener of frame k-1), the
 *                     detection lists;
 *   internal stream : frame k's moments, shifted by frame k-1's mean, and its
 *                     FP64 statistics (for frame k+1), at the same time.
 * Frame 0 has no predecessor: it is scored with its own statistics, computed
 * first.  hsi_lagged_push returns once the work is queued; the caller's
 * stream then also waits for frame k's moments pass (not its factorisation),
 * so work the caller queues after the push -- for example the next frame's
 * upload into the same cube buffer -- starts only once the cube is read.
 * Every frame of a stream has the options' shape and element type.  Cubes are
 * device BSQ at hsi_plane_stride(height, width).
 */
#ifndef HSI_LAGGED_H
#define HSI_LAGGED_H

#include "hsi_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define HSI_LAGGED_SAM_CEM 1 /* SAM and CEM maps, best, lists */
#define HSI_LAGGED_RX_ACE 2  /* RX and ACE maps, best, lists */

typedef struct hsi_lagged_options {
  int32_t height, width, bands, dtype; /* dtype: HSI_F32 or HSI_F16 */
  const float* targets;                /* HOST: num_targets x bands, the SAM / CEM / ACE library */
  int32_t num_targets;                 /* 1..16 */
  int32_t detectors;                   /* HSI_LAGGED_SAM_CEM | HSI_LAGGED_RX_ACE */
  double loading;                      /* diagonal loading of the statistics */
  float sam_threshold;                 /* radians, lower is better */
  float cem_threshold;                 /* higher is better */
  float ace_threshold;                 /* higher is better */
  double rx_false_alarm_rate;          /* RX threshold: chi-square quantile at this rate */
  int32_t nms_radius;
  int32_t capacity; /* detections kept per list */
} hsi_lagged_options;

/* Device outputs of the last pushed frame (valid once the caller's stream has
 * passed that push).  Lists: 0 SAM, 1 CEM, 2 ACE, 3 RX; counts may exceed
 * capacity.  Maps are target-major at map_stride = height * width. */
typedef struct hsi_lagged_outputs {
  int64_t frame;            /* index of the last pushed frame */
  int64_t statistics_frame; /* frame whose statistics scored it: frame - 1, or 0 for frame 0 */
  const float* sam_maps;    /* num_targets maps, or NULL without HSI_LAGGED_SAM_CEM */
  const float* sam_best;
  const int32_t* sam_target;
  const float* cem_maps;
  const float* cem_best;
  const int32_t* cem_target;
  const float* rx; /* NULL without HSI_LAGGED_RX_ACE */
  const float* ace_maps;
  const float* ace_best;
  const int32_t* ace_target;
  const hsi_detection* detections[4];
  const uint32_t* counts;   /* 4 counts */
  const int32_t* status;    /* factorisation status of statistics_frame (HSI_OK ...) */
  int64_t map_stride;
  float rx_threshold;
} hsi_lagged_outputs;

typedef struct hsi_lagged hsi_lagged;

/* NULL on failure, with *status (nullable) set.  Allocates all device
 * buffers and the internal stream once. */
HSI_API hsi_lagged* hsi_lagged_create(const hsi_lagged_options* options, int* status);
/* Score one frame (see above).  `d_cube` is read by work on `stream` and on
 * the internal stream; it must stay valid until `stream` passes this push. */
HSI_API int hsi_lagged_push(hsi_lagged* runner, const void* d_cube, hsi_stream_t stream);
HSI_API int hsi_lagged_outputs_of(const hsi_lagged* runner, hsi_lagged_outputs* out);
/* Waits for the internal stream, then frees everything. */
HSI_API void hsi_lagged_destroy(hsi_lagged* runner);

#ifdef __cplusplus
}
#endif

#endif /* HSI_LAGGED_H */
