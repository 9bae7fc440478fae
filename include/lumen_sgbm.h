/*
 * lumen_sgbm.h -- C ABI of the B200 SGBM stereo engine.
 *
 * Plain C: pointers, sizes and POD structs only, so any FFI (ctypes, cgo, JNI,
 * N-API) can bind it.  Each entry point names the LumenStereo interface it
 * replaces (paths relative to the LumenStereo source tree).  The header-only
 * C++ wrapper in include/stereo/sgbm_gpu.h restores the reference's
 * stereo::StereoSGBM class and exception types on top of these calls.
 *
 * Threading: a handle is not thread-safe (like stereo::StereoSGBM); separate
 * handles may be used from separate threads.  lumen_last_error_string() is
 * per thread.
 */
#ifndef LUMEN_SGBM_H
#define LUMEN_SGBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUMEN_SGBM_ABI_VERSION 1

/* Replaces stereo::kSgbmMaxDisparityRange (include/stereo/sgbm_limits.h:9). */
#define LUMEN_MAX_DISPARITY_RANGE 512

/* Status codes.  INVALID_ARGUMENT and RANGE_EXCEEDS_LIMIT are the cases in
 * which the reference throws StereoException (src/sgbm_gpu.cu:148-166);
 * CUDA_ERROR is the reference's CudaException (include/stereo/common.h:31-84). */
typedef enum lumen_status {
    LUMEN_OK = 0,
    LUMEN_ERR_INVALID_ARGUMENT = 1,   /* empty input, size mismatch, bad disparity range */
    LUMEN_ERR_RANGE_EXCEEDS_LIMIT = 2, /* maxDisparity - minDisparity > 512 */
    LUMEN_ERR_CUDA = 3,               /* a CUDA call failed; see lumen_last_error_string() */
    LUMEN_ERR_OUT_OF_BUDGET = 4,      /* request larger than the device-memory budget */
    LUMEN_ERR_TIMEOUT = 5,            /* a bounded device-side wait gave up */
    LUMEN_ERR_NO_DEVICE = 6           /* no CUDA device / kernels not loadable */
} lumen_status;

/* Field-for-field mirror of stereo::StereoParams (include/stereo/stereo_params.h:57-82,
 * defaults from the same lines; fill with lumen_stereo_params_default()). */
typedef struct lumen_stereo_params {
    int32_t minDisparity;      /* 0 */
    int32_t maxDisparity;      /* 128 */
    int32_t blockSize;         /* 5 */
    int32_t P1;                /* 200 */
    int32_t P2;                /* 800 */
    int32_t preFilterCap;      /* 31 */
    int32_t uniquenessRatio;   /* 10 */
    int32_t disp12MaxDiff;     /* 1, -1 disables the LR check */
    int32_t speckleWindowSize; /* 100, 0 disables the speckle filter */
    int32_t speckleRange;      /* 32 */
    int32_t useGPU;            /* 1 (read and written, never acted on, as in the reference) */
    int32_t useSharedMemory;   /* 1 (accepted; every cost kernel here stages through shared memory) */
    int32_t numDirections;     /* 4, or 8 for the four diagonal paths too */
    int32_t matchingCostMode;  /* 0 = SAD (Sobel-x prefilter), 1 = Census 5x5 */
} lumen_stereo_params;

typedef struct lumen_sgbm lumen_sgbm;

/* StereoParams{} (include/stereo/stereo_params.h:57-82). */
void lumen_stereo_params_default(lumen_stereo_params* out);
/* StereoParams::isValid (stereo_params.h:96-103): 1 valid, 0 not. */
int lumen_stereo_params_is_valid(const lumen_stereo_params* p);
/* StereoParams::autoComputePenalties (stereo_params.h:88-91). */
void lumen_stereo_params_auto_penalties(lumen_stereo_params* p, int numChannels);

/* StereoSGBM::StereoSGBM (include/stereo/sgbm_gpu.h:31, src/sgbm_gpu.cu:100-107):
 * binds the current CUDA device, creates the handle's stream and events.
 * params may be NULL for the defaults. */
lumen_status lumen_sgbm_create(const lumen_stereo_params* params, lumen_sgbm** out);
/* StereoSGBM::~StereoSGBM (src/sgbm_gpu.cu:109-113); frees every device buffer. */
lumen_status lumen_sgbm_destroy(lumen_sgbm* h);
/* StereoSGBM::setParams / getParams (include/stereo/sgbm_gpu.h:46-47). */
lumen_status lumen_sgbm_set_params(lumen_sgbm* h, const lumen_stereo_params* params);
lumen_status lumen_sgbm_get_params(const lumen_sgbm* h, lumen_stereo_params* out);

/* StereoSGBM::compute (include/stereo/sgbm_gpu.h:41, src/sgbm_gpu.cu:147-195) on
 * HOST buffers, synchronous.  left/right: height rows of width*channels bytes,
 * row pitch in_stride bytes (0 = tightly packed); channels 1 (gray) or 3 (BGR,
 * converted with BT.601 15-bit fixed point like cv::cvtColor(COLOR_BGR2GRAY)).
 * out: height rows of width int16 disparities in 1/16 px (-1 = invalid), row
 * pitch out_stride bytes (0 = packed). */
lumen_status lumen_sgbm_compute(lumen_sgbm* h, const uint8_t* left, const uint8_t* right,
                                int width, int height, size_t in_stride, int channels,
                                int16_t* out, size_t out_stride);

/* Same computation on DEVICE buffers, asynchronous on `stream` (a
 * cudaStream_t; NULL = the default stream, as in every CUDA API).  Returns
 * after enqueueing; the caller synchronises.  No host<->device copies. */
lumen_status lumen_sgbm_compute_device(lumen_sgbm* h, const uint8_t* d_left,
                                       const uint8_t* d_right, int width, int height,
                                       size_t in_stride, int channels, int16_t* d_out,
                                       size_t out_stride, void* stream);

/* getLastComputeTimeMs / getCostComputeTimeMs / getAggregationTimeMs /
 * getPostProcessTimeMs (include/stereo/sgbm_gpu.h:52-55), device time in ms of
 * the last synchronous compute: out[0] total, [1] cost, [2] aggregation,
 * [3] disparity selection + post-processing.  After lumen_sgbm_compute_device
 * the first call waits for that compute's last event. */
lumen_status lumen_sgbm_get_timings(lumen_sgbm* h, float out[4]);

/* Human-readable message of the last failing call on this thread ("" if none). */
const char* lumen_last_error_string(void);

/* ---- diagnostics (no counterpart in the reference's public API; they expose the
 * intermediate buffers the parity tests compare stage by stage) ---- */

/* Path-set override for the next computes: bit i selects path i in the order
 * LR, RL, TB, BT, TLBR, BRTL, TRBL, BLTR (src/sgbm_gpu.cu:321-421); 0 restores
 * the numDirections default. */
lumen_status lumen_sgbm_debug_set_paths(lumen_sgbm* h, uint32_t path_mask);
/* Aggregation schedule: 0 = automatic (autotuner / heuristic), 1 = one kernel
 * per direction, 4 = two fused wavefront sweeps with lockstep row bands and
 * helper warps for the band hand-offs (the batched form's usual pick), 6 = four
 * lag-free sweeps, two over rows and two over columns: two paths each with 8
 * paths (the row and the column sweeps as two concurrent launches unless
 * tuned otherwise), one path each with 4 (then no band waits on another) --
 * the default for padded disparities up to 320; wider ranges fall back to
 * schedule 4.
 * Other values are refused (LUMEN_ERR_INVALID_ARGUMENT).  Outputs are
 * identical for every schedule. */
lumen_status lumen_sgbm_set_schedule(lumen_sgbm* h, int schedule);
/* Pin the fused-sweep configuration: lanes per row (8, 16 or 32) and rows per
 * band (`warps_per_block`).  Schedule 4: 32 lanes with 4, 8 or 16 rows; 8
 * lanes (padded disparities up to 128) or 16 lanes (up to 256), rows as lane
 * teams, with 8, 16 or 32 rows.  Schedule 6: its lanes per row (8 up to 128
 * padded disparities, 16 up to 320) with 16, 24 or 32 rows; a configuration
 * without an instance falls back to the default.  0, 0 restores the automatic choice.
 * Values are identical for every setting. */
lumen_status lumen_sgbm_set_tuning(lumen_sgbm* h, int lanes_per_pixel, int warps_per_block);
/* Schedule 6 with 8 paths: rows per band of the column sweeps when they run as
 * a launch of their own beside the row sweeps' (16, 24 or 32), 0 for one
 * launch of all four sweeps, -1 for the automatic choice (the tuned value,
 * else 24; a configuration pinned by lumen_sgbm_set_tuning alone keeps one
 * launch).  No counterpart in the reference. */
lumen_status lumen_sgbm_set_tuning_columns(lumen_sgbm* h, int rows_per_band);
/* The schedule and configuration the last compute used: {schedule, lanes, warps}. */
lumen_status lumen_sgbm_get_tuning(const lumen_sgbm* h, int out[3]);
/* Rows per band of the column sweeps' own launch in the last compute (0: none). */
lumen_status lumen_sgbm_get_tuning_columns(const lumen_sgbm* h, int* rows_per_band);
/* Autotuner (no counterpart in the reference): runs every aggregation schedule
 * and sweep configuration `repeats` times on the given DEVICE pair, keeps the
 * fastest for this (size, disparity range, cost mode, path set) key, and
 * writes one line per candidate into `report`.  Synchronous. */
lumen_status lumen_sgbm_autotune(lumen_sgbm* h, const uint8_t* d_left, const uint8_t* d_right,
                                 int width, int height, size_t in_stride, int channels,
                                 int repeats, char* report, size_t report_bytes);
/* Persist / restore the autotuner's decisions (text, one key per line). */
lumen_status lumen_sgbm_tuning_save(const lumen_sgbm* h, const char* path);
lumen_status lumen_sgbm_tuning_load(lumen_sgbm* h, const char* path);
/* Copies one internal buffer of the last compute to host memory `dst`
 * (capacity dst_bytes).  which: 0 prefiltered left, 1 prefiltered right,
 * 2 census left (uint32), 3 census right, 4 cost volume (uint8 HxWxD),
 * 5 aggregated volume (uint16 HxWxD), 6 left WTA disparity, 7 right
 * disparity, 8 disparity after the LR check (and speckle filter), 9 gray left,
 * 10 gray right.  Volumes are returned densely packed with D entries per
 * pixel.  The debug-retain flag must have been set before the compute. */
lumen_status lumen_sgbm_debug_retain(lumen_sgbm* h, int enable);
lumen_status lumen_sgbm_debug_copy(lumen_sgbm* h, int which, void* dst, size_t dst_bytes);
/* Band timeline of the row-band sweeps for the next computes (enable = 1) or
 * off (0).  lumen_sgbm_debug_trace_copy returns the last such launch's
 * records, 4 words per band ticket t.  Schedule 4 (t = 2*band + sweep):
 * globaltimer ns when the band's first row and its last row finished the
 * middle pixel (u = width / 2), when the band ended, and SM id << 48 |
 * import polls << 32 | export polls << 16 | row waits on the helpers.
 * Schedule 6 with the diagonal paths (t in the sweeps' ticket order): when
 * the band's rows started their first pixel, finished the middle pixel and
 * finished the row, and SM id << 32 | sweep << 16 | 1.
 * *words receives the record size; dst may be NULL to query it. */
lumen_status lumen_sgbm_debug_trace(lumen_sgbm* h, int enable);
lumen_status lumen_sgbm_debug_trace_copy(lumen_sgbm* h, unsigned long long* dst,
                                         size_t dst_words, size_t* words);
/* Number of kernels this handle has enqueued so far (all computes). */
unsigned long long lumen_sgbm_debug_launch_count(const lumen_sgbm* h);
/* Iteration limit of every device-side wait (0 restores the default, 2^22). */
lumen_status lumen_sgbm_debug_set_wait_limit(lumen_sgbm* h, long long spins);
/* Issue-rate probe (no counterpart in the reference): device ns per
 * warp-instruction per SM of __vminu2, __vimin3_u16x2, __viaddmin_u16x2 and a
 * 32-bit add, each timed with CUDA events over independent chains on every
 * SM (out[0..3]).  Informs how the recurrence's minima are written. */
lumen_status lumen_debug_op_rates(float out[4]);
/* Failure-path self test of schedules 4 and 6: while enabled, one wait of a band
 * that imports from the band above can never be satisfied, so it runs out
 * after the wait limit and the compute returns LUMEN_ERR_TIMEOUT (no fault, no
 * hang; the handle stays usable). */
lumen_status lumen_sgbm_debug_stall_test(lumen_sgbm* h, int enable);

/* ---- rectification remap (replaces stereo::StereoRectifier,
 * include/stereo/rectification.h:41-84, and rectifyImageGPU :92-97) ---- */
typedef struct lumen_rectifier lumen_rectifier;

/* StereoRectifier(const CameraParams&) (src/rectification.cu:259-284): uploads
 * the four CV_32FC1 maps (width*height floats each) once; NULL maps mean the
 * pair is pre-rectified and rectify() copies. */
lumen_status lumen_rectifier_create(int width, int height, const float* map0x,
                                    const float* map0y, const float* map1x,
                                    const float* map1y, lumen_rectifier** out);
lumen_status lumen_rectifier_destroy(lumen_rectifier* r);
int lumen_rectifier_is_pre_rectified(const lumen_rectifier* r);
/* StereoRectifier::rectify (src/rectification.cu:286-345) on host buffers. */
lumen_status lumen_rectifier_rectify(lumen_rectifier* r, const uint8_t* left_raw,
                                     const uint8_t* right_raw, int channels,
                                     uint8_t* left_rect, uint8_t* right_rect);
/* Device-buffer form, asynchronous on `stream` (NULL = the default stream). */
lumen_status lumen_rectifier_rectify_device(lumen_rectifier* r, const uint8_t* d_left_raw,
                                            const uint8_t* d_right_raw, int channels,
                                            uint8_t* d_left_rect, uint8_t* d_right_rect,
                                            void* stream);
/* rectifyImageGPU (src/rectification.cu:354-411): one image, host buffers. */
lumen_status lumen_remap(const uint8_t* src, const float* map_x, const float* map_y,
                         uint8_t* dst, int width, int height, int channels);

/* BGR -> gray on the device (the reference calls cv::cvtColor on the host,
 * src/sgbm_gpu.cu:169-172); host buffers, one image. */
lumen_status lumen_bgr_to_gray(const uint8_t* bgr, size_t stride, uint8_t* gray, int width,
                               int height);

/* ---- either side of the disparity map ---- */
/* disparityToDepthGPU (src/depth_map.cu:74-102, 169-187): depth = f * B /
 * (d / 16 + doffs) in the caller's units of B for positive 1/16-px
 * disparities, 0 elsewhere.  Device buffers (strides in bytes, 0 = packed),
 * asynchronous on `stream`. */
lumen_status lumen_disparity_to_depth_device(const int16_t* d_disp, int width, int height,
                                             size_t disp_stride, float focal_px, float baseline,
                                             float disparity_offset_px, float* d_depth,
                                             size_t depth_stride, void* stream);
/* The same conversion with a colour output in one pass (the reference runs
 * disparityToDepthKernel, then colorizeDepthKernel on the stored depth,
 * src/depth_map.cu:74-142): d_depth may be NULL when only the colours are
 * wanted; d_rgb (3 bytes a pixel, NULL: none) gets the colours of
 * lumen_depth_colorize_device.  `lut` is a HOST table of 256 channel triplets
 * in output order (768 bytes). */
lumen_status lumen_disparity_to_depth_color_device(const int16_t* d_disp, int width, int height,
                                                   size_t disp_stride, float focal_px, float baseline,
                                                   float disparity_offset_px, float* d_depth,
                                                   size_t depth_stride, float min_depth,
                                                   float max_depth, const uint8_t* lut, uint8_t* d_rgb,
                                                   size_t rgb_stride, void* stream);
/* colorizeDepthKernel (src/depth_map.cu:104-142): colour index 0 where
 * z <= 0 or z > 2 max_depth, else (int)((1 - clamp((z - min) / (max - min),
 * 0, 1)) * 255); each pixel gets lut[3 i .. 3 i + 2] (HOST table of 256
 * triplets; the reference's is a Turbo-like ramp in RGB order). */
lumen_status lumen_depth_colorize_device(const float* d_depth, int width, int height,
                                         size_t depth_stride, float min_depth, float max_depth,
                                         const uint8_t* lut, uint8_t* d_rgb, size_t rgb_stride,
                                         void* stream);
/* Point3D (include/stereo/point_cloud.h:17-25): 16 bytes, pad = 0. */
typedef struct lumen_point3d {
    float x, y, z;
    uint8_t r, g, b, pad;
} lumen_point3d;
/* depthToPointCloud (src/point_cloud.cpp:11-55) on the device: every pixel
 * with 0 < Z <= 100 (NaN kept, as in the reference) becomes the point
 * ((float)((u - cx) Z / fx), (float)((v - cy) Z / fy), Z), computed in double,
 * with the colour of d_bgr (BGR, 3 bytes a pixel, NULL: white), in raster
 * order.  d_points: device room for width*height points, 16-byte aligned;
 * d_row_offsets: device room for height + 1 ints, which receive row y's first
 * point index at [y] and the number of points at [height].  Asynchronous. */
lumen_status lumen_depth_to_points_device(const float* d_depth, int width, int height,
                                          size_t depth_stride, const uint8_t* d_bgr, size_t bgr_stride,
                                          double fx, double fy, double cx, double cy,
                                          lumen_point3d* d_points, int* d_row_offsets, void* stream);
/* depthToPointCloud (src/point_cloud.cpp:11-55) with HOST buffers: the same
 * points as lumen_depth_to_points_device, `count` of them written to
 * `points` (room for width*height).  Synchronous. */
lumen_status lumen_depth_to_points(const float* depth, int width, int height, size_t depth_stride,
                                   const uint8_t* bgr, size_t bgr_stride, double fx, double fy, double cx,
                                   double cy, lumen_point3d* points, int* count);
/* The CV_32FC1 maps cv::initUndistortRectifyMap produces for one camera
 * (src/calibration.cpp:253-266), generated on the device: K row-major 3x3,
 * dist = (k1, k2, p1, p2, k3) or NULL, R the rectifying rotation (3x3), P the
 * new projection (3x4, row-major).  Device maps of width*height floats. */
lumen_status lumen_rectify_maps_device(const double K[9], const double dist[5], const double R[9],
                                       const double P[12], int width, int height, float* d_map_x,
                                       float* d_map_y, void* stream);

/* ---- batched form (no counterpart in the reference's API; LumenStereo's
 * callers loop over StereoSGBM::compute, e.g. tools/evaluate.cpp:158-160) ----
 *
 * A batch holds stereo pairs of any sizes and parameters (gray DEVICE images
 * of width*height bytes with row pitch width; int16 DEVICE outputs with row
 * pitch width, 1/16 px, -1 invalid).  lumen_sgbm_batch_run enqueues every pair
 * on `stream`: cost volumes per pair, one persistent aggregation launch per
 * group of pairs of one kernel class (the sweeps of all its pairs share the
 * GPU; schedule 6, the default: the four lag-free sweeps of the plain call's
 * 8- and 4-path default, over every pair's bands; schedule 4: the two
 * wavefront sweeps), then selection per pair; consecutive groups overlap on the device
 * (one group's sweep beside the next one's cost volumes and the previous one's
 * selections, on internal streams joined back into `stream`).  The first run
 * after an add, a clear or an option change plans and allocates one pooled
 * buffer of at most device_budget_bytes (default 80 GiB; groups are cut to
 * fit it, two at a time when possible) and, with graphs enabled,
 * captures the run into a CUDA graph that later runs replay.  Outputs equal
 * lumen_sgbm_compute_device's bit for bit.  lumen_sgbm_batch_sync waits for
 * `stream` and reports a device-side timeout. */
typedef struct lumen_sgbm_batch lumen_sgbm_batch;
lumen_status lumen_sgbm_batch_create(lumen_sgbm_batch** out);
lumen_status lumen_sgbm_batch_destroy(lumen_sgbm_batch* b);
lumen_status lumen_sgbm_batch_add(lumen_sgbm_batch* b, const lumen_stereo_params* params,
                                  const uint8_t* d_left, const uint8_t* d_right, int width,
                                  int height, int16_t* d_out);
lumen_status lumen_sgbm_batch_clear(lumen_sgbm_batch* b);
/* rows_per_band: 4, 8 or 16 with schedule 4, 16, 24 or 32 with schedule 6 (0 = the
 * schedule's default, 8 / 16); use_graph: capture and replay; budget 0 = keep. */
lumen_status lumen_sgbm_batch_set_options(lumen_sgbm_batch* b, int rows_per_band, int use_graph,
                                          size_t device_budget_bytes);
lumen_status lumen_sgbm_batch_run(lumen_sgbm_batch* b, void* stream);
/* Autotuner of the batched launch (no counterpart in the reference): runs the
 * batch with schedule 6 at 16, 24 and 32 rows per band and schedule 4 at 4, 8
 * and 16 (only the pinned schedule's, when one is set) -- `repeats` timed runs
 * each, on `stream`, writing the outputs -- and keeps the fastest schedule and
 * band height for later runs. */
lumen_status lumen_sgbm_batch_autotune(lumen_sgbm_batch* b, void* stream, int repeats, int* best_rows,
                                       float* best_ms);
/* Aggregation schedule of the batch: 0 (automatic: 6 until the autotuner
 * picks), 4 or 6 (no counterpart in the reference). */
lumen_status lumen_sgbm_batch_set_schedule(lumen_sgbm_batch* b, int schedule);
/* The schedule and rows per band the next run plans with. */
lumen_status lumen_sgbm_batch_config(const lumen_sgbm_batch* b, int* schedule, int* rows_per_band);
lumen_status lumen_sgbm_batch_sync(lumen_sgbm_batch* b, void* stream);
/* Pooled device bytes, number of launch groups, kernels per run. */
lumen_status lumen_sgbm_batch_info(const lumen_sgbm_batch* b, size_t* device_bytes, int* groups,
                                   unsigned long long* launches);

/* ---- served form (no counterpart in the reference's API) ----
 *
 * A server owns a device arena of device_budget_bytes (allocated once), the
 * resident rectification maps of registered calibration ids, and a thread
 * that batches queued requests continuously: whenever one of max_inflight
 * batch slots is free it admits waiting requests in arrival order while their
 * buffers fit in the arena (at most max_batch_pairs per batch) and launches
 * them through the batched kernels; a batch admitted while another runs
 * overlaps with it on the device.  Each result is bit-exact with
 * lumen_sgbm_compute on the same (rectified) pair. */
typedef struct lumen_server lumen_server;
typedef struct lumen_server_options {
    size_t device_budget_bytes; /* arena size; default 40 GiB */
    int max_batch_pairs;        /* default 32 */
    int rows_per_band;          /* schedule 4: 4, 8 or 16; schedule 6: 16 (default), 24 or 32 */
    int max_inflight;           /* batch slots on the device at once, 1..8; default 2 */
    int watchdog_ms;            /* host deadline of a batch, 0 = none; default 60000 */
    long long spin_limit;       /* device-side wait limit, 0 = default (2^24) */
    int plain_fallback;         /* 1 (default): the requests of a batch whose launch fails or
                                   whose device-side waits run out are computed again one by one
                                   through the plain call (lumen_sgbm_compute_device with the
                                   default wait limit); 0: they complete with the batch's error */
    int schedule;               /* aggregation of the batches: 6 (default, four lag-free sweeps)
                                   or 4 (two wavefront sweeps) */
} lumen_server_options;
typedef struct lumen_request_info {
    lumen_status status;
    double latency_ms;  /* submit -> result in the caller's buffer */
    double queue_ms;    /* submit -> admission */
    double device_ms;   /* the batch's device time */
    int batch_pairs;    /* requests in the batch */
    unsigned long long batch_id;
} lumen_request_info;
typedef struct lumen_server_stats {
    unsigned long long submitted, completed, rejected, failed, batches, watchdog_expired;
    size_t budget_bytes, admitted_bytes, peak_admitted_bytes;
    int queue_depth, peak_queue_depth, inflight_batches, peak_batch_pairs;
    unsigned long long fallbacks; /* requests served by the plain-call fallback */
} lumen_server_stats;
void lumen_server_options_default(lumen_server_options* o);
lumen_status lumen_server_create(const lumen_server_options* o, lumen_server** out);
/* Finishes every queued request, then frees the server. */
lumen_status lumen_server_destroy(lumen_server* s);
/* Uploads the four CV_32FC1 maps of a calibration once (NULL maps: the pairs
 * are pre-rectified); an id is bound once. */
lumen_status lumen_server_set_calibration(lumen_server* s, int calib_id, int width, int height,
                                          const float* map0x, const float* map0y,
                                          const float* map1x, const float* map1y);
/* Same, from the calibration itself: the maps of both cameras are generated
 * on the device (lumen_rectify_maps_device) from K, distortion (k1, k2, p1, p2,
 * k3 or NULL), rectifying rotation and new projection, as
 * src/calibration.cpp:230-266 gets them from OpenCV; no host maps. */
lumen_status lumen_server_set_calibration_params(lumen_server* s, int calib_id, int width, int height,
                                                 const double K0[9], const double D0[5],
                                                 const double R0[9], const double P0[12],
                                                 const double K1[9], const double D1[5],
                                                 const double R1[9], const double P1[12]);
/* Queues one gray pair (host buffers, width*height bytes each, copied before
 * the call returns); calib_id -1 = already rectified.  `out` (width*height
 * int16) is written before lumen_server_wait reports the request done and
 * must stay valid until then.  Invalid parameters and requests larger than
 * the budget are rejected here, the server keeps serving. */
lumen_status lumen_server_submit(lumen_server* s, const lumen_stereo_params* params, int calib_id,
                                 const uint8_t* left, const uint8_t* right, int width, int height,
                                 int16_t* out, unsigned long long* request_id);
/* Waits for a request (timeout_ms < 0: no limit) and releases its id; returns
 * the request's status (LUMEN_ERR_TIMEOUT also when the wait itself ran out,
 * with the id kept). */
lumen_status lumen_server_wait(lumen_server* s, unsigned long long request_id, int timeout_ms,
                               lumen_request_info* info);
lumen_status lumen_server_get_stats(lumen_server* s, lumen_server_stats* out);
/* Failure injection on the host (tests): the next `n` batch launches fail
 * before any device work, as a launch that cannot be enqueued would. */
lumen_status lumen_server_debug_fail_batches(lumen_server* s, int n);

/* ---- Census cost volume without device allocation.  No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc (a real-time loop
 * that must not take cudaMalloc's implicit device synchronisation, a plugin host
 * whose pool owns all device memory). ----
 *
 * Census 5x5 descriptors of both DEVICE images (gray, width*height bytes, pitch
 * width) and the uint8 cost volume d_cost[(y*width + x)*cost_stride + d], the
 * values of the Census stage of lumen_sgbm_compute (entries d >= maxDisparity -
 * minDisparity are 0).  cost_stride: a multiple of 16, >= the disparity range;
 * d_cost: 16-byte aligned (LUMEN_ERR_INVALID_ARGUMENT otherwise).
 * Asynchronous on `stream` (NULL = the default stream).  The descriptors live
 * in a fixed 16 MiB array inside the library (held by every GPU that loads it
 * until exit): images above lumen_census_cost_noalloc_max_pixels() pixels
 * (2^21, so 1920x1080 fits) return LUMEN_ERR_OUT_OF_BUDGET.  The first call on
 * a device looks up that array's device address (make it before any stream
 * capture).  All calls share the array: calls whose work overlaps on the GPU
 * race and must be serialised. */
lumen_status lumen_census_cost_noalloc(const uint8_t* d_left, const uint8_t* d_right, int width,
                                       int height, int min_disparity, int max_disparity,
                                       uint8_t* d_cost, int cost_stride, void* stream);
size_t lumen_census_cost_noalloc_max_pixels(void);

#ifdef __cplusplus
}
#endif
#endif /* LUMEN_SGBM_H */
