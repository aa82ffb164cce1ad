/*
 * hsi_batch.h - C ABI of the batched frame runner (libhsi_cxx.so).
 *
 * No single counterpart in the reference, whose Pipeline scores one frame
 * shape at a time (src/pipeline.cu:39-469).  A batch is a fixed set of frames
 * of uneven sizes and band counts, each with its own target library; one run
 * does, on one stream:
 *   demosaic (frames given as snapshot mosaics), scene moments and the FP64
 *   statistics per frame, SAM best-angle maps for all frames in one
 *   persistent launch per element type, RX and best-ACE maps per frame, and
 *   raster-ordered detection lists for SAM (lower is better), ACE and RX
 *   (higher is better) in batched launches.
 * hsi_batch_capture records that run as one CUDA graph and hsi_batch_launch
 * replays it.  With autotune set, creation times the persistent scorer's CTAs
 * per SM and, per frame, the tensor-core against the plain RX/ACE path, on
 * the batch itself, and keeps the fastest.
 * Cubes are device BSQ at hsi_plane_stride(height, width).
 */
#ifndef HSI_BATCH_H
#define HSI_BATCH_H

#include "hsi_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hsi_batch_frame {
  const void* cube;        /* device BSQ cube, or NULL when `raw` is given */
  const float* raw;        /* device snapshot mosaic (raw_height x raw_width floats), or NULL */
  int32_t raw_height, raw_width, period;  /* mosaic geometry: bands = period^2 (or fewer) */
  int32_t height, width, bands;           /* of the cube (from the mosaic when raw is given) */
  int32_t dtype;                          /* HSI_F32 or HSI_F16 (a demosaiced cube is HSI_F32) */
  const float* targets;    /* HOST: num_targets x bands */
  int32_t num_targets;     /* 1..16 */
} hsi_batch_frame;

typedef struct hsi_batch_options {
  float sam_threshold;          /* radians, lower is better */
  float ace_threshold;          /* higher is better */
  double rx_false_alarm_rate;   /* RX threshold: chi-square quantile at this rate */
  double loading;               /* diagonal loading of the statistics */
  int32_t nms_radius;
  int32_t capacity;             /* detections kept per list */
  int32_t autotune;             /* 1: time the tunable choices on this batch */
} hsi_batch_options;

typedef struct hsi_batch_outputs {
  const float* sam_best;        /* each P floats / ints, device */
  const int32_t* sam_target;
  const float* rx;
  const float* ace_best;
  const int32_t* ace_target;
  const hsi_detection* detections[3];  /* SAM, ACE, RX lists (capacity each) */
  const uint32_t* counts;              /* 3 counts (may exceed capacity) */
  const int32_t* status;               /* the frame's statistics status (HSI_OK ...) */
  float rx_threshold;
} hsi_batch_outputs;

typedef struct hsi_batch_tuning {
  int32_t score_ctas_per_sm;     /* 0: as many as fit */
  int32_t tensor_core_rx_frames; /* frames whose RX/ACE runs on the tensor cores */
  int32_t plain_rx_frames;
  float tuning_ms;               /* time spent timing candidates */
} hsi_batch_tuning;

typedef struct hsi_batch hsi_batch;

/* NULL on failure, with *status (nullable) set. */
HSI_API hsi_batch* hsi_batch_create(const hsi_batch_frame* frames, int num_frames, const hsi_batch_options* options,
                                    int* status);
/* One run, launched eagerly on `stream`. */
HSI_API int hsi_batch_run(hsi_batch* batch, hsi_stream_t stream);
/* Record one run on `stream` into a CUDA graph (after at least one hsi_batch_run). */
HSI_API int hsi_batch_capture(hsi_batch* batch, hsi_stream_t stream);
/* Replay the recorded graph on `stream`. */
HSI_API int hsi_batch_launch(hsi_batch* batch, hsi_stream_t stream);
HSI_API int hsi_batch_outputs_of(const hsi_batch* batch, int frame, hsi_batch_outputs* out);
HSI_API int hsi_batch_tuning_of(const hsi_batch* batch, hsi_batch_tuning* out);
HSI_API void hsi_batch_destroy(hsi_batch* batch);

#ifdef __cplusplus
}
#endif

#endif /* HSI_BATCH_H */
