/*
 * nx_stereo_b200: NxStereo's full-search Stage.Disparity path (census, Hamming
 * costs, 8- or 3-path SGM, winner-take-all with uniqueness, subpixel, the
 * left-right check and the median) with Stage.Rectification,
 * Stage.SpeckleFilter and the stages after them, as CUDA kernels for B200
 * (sm_100a) behind a C ABI.
 *
 * Two layers:
 *
 *  1. The segment protocol: configure / run / release, the three requests the
 *     reference's native Port serves (native/stereo_match/src/protocol.rs:1-23),
 *     as in-process calls an Erlang NIF (or ctypes, cgo, JNI) binds. A segment is
 *     a run of stages configured once, fed one pair per request, FIFO, with the
 *     values its stages carry from pair to pair kept on the device.
 *
 *  2. Direct entry points: the matcher on one pair (NxStereo.sgm/3) and each
 *     stage kernel on device buffers, for callers that manage their own memory
 *     and streams, and for checking intermediates bit for bit.
 *
 * Conventions: images are row-major, width fastest. Every call returns an
 * nxs_status; on failure a UTF-8 message is written to `error` (at most
 * error_len bytes including the terminating zero) when `error` is not NULL.
 * No exception crosses the ABI. Pointers named `d_*` are device pointers;
 * `stream` is a cudaStream_t (NULL for the legacy default stream).
 */
#ifndef NX_STEREO_B200_H
#define NX_STEREO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NXS_OK = 0,
    NXS_PENDING = 1,       /* a request is still on the device */
    NXS_REFUSED = 2,       /* a configuration the segment refuses: {:stop, reason} */
    NXS_BAD_RUN = 3,       /* a request the segment cannot run: {:error, reason} */
    NXS_CUDA_ERROR = 4,    /* the device failed */
    NXS_TIMEOUT = 5,       /* a wait ran out */
    NXS_BAD_ARGUMENT = 6,  /* a direct entry point's arguments are out of range */
    NXS_NO_SEGMENT = 7     /* no segment of that id is configured */
} nxs_status;

/* Element types: the Port's tensor type codes (native/stereo_match/src/tensor.rs:25-30). */
enum { NXS_U8 = 0, NXS_U16 = 1, NXS_F32 = 2, NXS_S32 = 3 };

typedef struct nxs_context nxs_context;
typedef struct nxs_request nxs_request;

/* ------------------------------------------------------------------------ */
/* Context                                                                   */

/* Opens a context on CUDA device `device`. Replaces starting the Port
 * (lib/nx_stereo/matcher.ex:248-260, native/stereo_match/src/main.rs:21-38). */
nxs_status nxs_create(int device, nxs_context **context, char *error, size_t error_len);

/* Releases every segment and the context's device memory. */
void nxs_destroy(nxs_context *context);

/* The library's version string. */
const char *nxs_version(void);

/* ------------------------------------------------------------------------ */
/* Layer 1: the segment protocol                                             */

/* A stage's build setting or native constant, as the configure request
 * carries them: a name and an f64 (lib/nx_stereo/native_segment.ex:256-290). */
typedef struct {
    const char *name;
    double value;
} nxs_setting;

/* A member: its native kind ("rectification", "disparity", "speckle_filter",
 * "temporal_filter", "depth", "point_cloud", "quality") and its settings. */
typedef struct {
    const char *kind;
    uint32_t n_settings;
    const nxs_setting *settings;
} nxs_member;

/* The sizes every stage works with (native/stereo_match/src/segment.rs:19-27). */
typedef struct {
    uint32_t width, height;             /* the rectified working size */
    uint32_t frame_width, frame_height; /* the camera frames' size */
} nxs_geometry;

/* A live input of a member for one pair: a name and its f32 values, as the
 * run request flattens a stage's params/2 (native_segment.ex:292-322;
 * e.g. "p1", "uniqueness", "left.k", "right.inverse_pr"). */
typedef struct {
    const char *name;
    uint32_t count;
    const float *values;
} nxs_param;

typedef struct {
    uint32_t n_params;
    const nxs_param *params;
} nxs_member_params;

/* A tensor entering a request (host memory, borrowed for the call only) or
 * returned by one (owned by the request until nxs_request_free). */
typedef struct {
    const char *name;
    uint32_t type; /* NXS_U8, NXS_U16, NXS_F32 or NXS_S32 */
    uint32_t rank; /* 0 to 4 */
    uint32_t dims[4];
    const void *data;
    uint64_t bytes;
} nxs_tensor;

/* Configures segment `segment` with `members` for `geometry`, replacing any
 * segment of that id (which starts the values its stages carry over).
 * NXS_REFUSED with the reason for a kind without an implementation, a
 * setting a kind does not take, or frames smaller than the working size to
 * rectify (native/stereo_match/src/segment.rs:181-333). Replaces the configure
 * request (protocol.rs:5-9). */
nxs_status nxs_configure(nxs_context *context, uint32_t segment, const nxs_geometry *geometry,
                         uint32_t n_members, const nxs_member *members, char *error,
                         size_t error_len);

/* Called on a CUDA host-callback thread once a request's outputs are in host
 * memory; it must not call CUDA. A NIF passes enif_send here. */
typedef void (*nxs_done_fn)(void *user, uint64_t tag);

/* Sends one pair through segment `segment` without waiting: copies the
 * entries' host bytes into the request before returning, enqueues every
 * stage on the segment's stream, and returns the request. Requests on one
 * segment run in the order sent. NXS_BAD_RUN for missing, misshapen or
 * mistyped entries or params; NXS_NO_SEGMENT for an unknown id. Replaces the
 * run request (protocol.rs:10-15) and NativeSegment.send_request/2
 * (lib/nx_stereo/native_segment.ex:164-189). */
nxs_status nxs_run_async(nxs_context *context, uint32_t segment, uint32_t n_members,
                         const nxs_member_params *params, uint32_t n_entries,
                         const nxs_tensor *entries, nxs_done_fn done, void *user, uint64_t tag,
                         nxs_request **request, char *error, size_t error_len);

/* NXS_OK once the request is done, NXS_PENDING while it is on the device, or
 * the device's error. */
nxs_status nxs_request_poll(nxs_request *request, char *error, size_t error_len);

/* Waits up to timeout_ms (negative: without limit) for the request: NXS_OK,
 * NXS_TIMEOUT, or the device's error. Replaces NativeSegment.await/3
 * (native_segment.ex:207-218). */
nxs_status nxs_request_wait(nxs_request *request, int64_t timeout_ms, char *error,
                            size_t error_len);

/* The tensors the members filled, each once, in the order first filled
 * (segment.rs:203-239); valid until nxs_request_free. */
nxs_status nxs_request_outputs(nxs_request *request, uint32_t *n_outputs,
                               const nxs_tensor **outputs);

/* Each member's device time in microseconds (the reply's times, protocol.rs:11-15). */
nxs_status nxs_request_times(nxs_request *request, uint32_t *n_members,
                             const uint32_t **times_us);

/* When the device finished the request, in nanoseconds of CLOCK_MONOTONIC
 * (the clock of a serving loop's arrival times), from the device's timestamp
 * of the request's completion mapped onto that clock; 0 while it is pending. */
uint64_t nxs_request_done_ns(nxs_request *request);

/* Frees a request; waits for it first if it is still on the device. */
void nxs_request_free(nxs_request *request);

/* The device's free and total memory in bytes, for admission control. */
nxs_status nxs_device_memory(nxs_context *context, uint64_t *free_bytes,
                             uint64_t *total_bytes);

/* Releases segment `segment` after its requests finish. Replaces the release
 * request (protocol.rs:16). */
nxs_status nxs_release(nxs_context *context, uint32_t segment);

/* ------------------------------------------------------------------------ */
/* Layer 2: direct entry points                                              */

/* NxStereo.sgm/3's settings (lib/nx_stereo.ex:44-62). disparities: 64 or 128
 * as the reference takes them, and 96, 192 and 256 beyond it; paths 3 or 8;
 * integers 0 <= p1 < p2 <= 79; uniqueness >= 1. */
typedef struct {
    uint32_t disparities;
    uint32_t paths;
    uint32_t p1, p2;
    float uniqueness;
    uint32_t stage_mask; /* non-zero: Stage.Disparity's step, disparity <= 0 becomes -1 */
} nxs_sgm_params;

/* Why NxStereo.sgm/3 would refuse these settings for a width x height pair
 * (lib/nx_stereo.ex:89-134, native/stereo_match/src/lib.rs:41-72), extended to
 * the disparity counts above: NXS_OK or NXS_BAD_ARGUMENT with the reason. */
nxs_status nxs_sgm_check(const nxs_sgm_params *params, uint32_t width, uint32_t height,
                         char *error, size_t error_len);

/* The shape of the path-aggregation kernels at `disparities` disparities:
 * each lane of a scan line holds `words` u16x2 words (4, 8 or 16, so 8, 16
 * or 32 disparities). A tuning knob for the whole library (nx_stereo_b200.batch's
 * autotuner sets it); results do not depend on it. */
nxs_status nxs_set_path_words(uint32_t disparities, uint32_t words);
uint32_t nxs_path_words(uint32_t disparities);

/* How the matcher aggregates the 8 (or 3) directions before selection
 * (lib/nx_stereo.ex:545-573, one sum per pixel and disparity): mode 0 (the
 * default) keeps each direction's u8 path volume and selection sums them;
 * mode 1 has every direction add its path costs into one u16 aggregate
 * volume in L2 as it scans (nxs_path_sums_device), which measured slower. A
 * tuning knob for the whole library; results do not depend on it.
 * nxs_path_sums: 1 where the matcher sums at that size. */
nxs_status nxs_set_path_sums(uint32_t mode);
uint32_t nxs_path_sums(uint32_t width, uint32_t height, uint32_t disparities);

/* How the path scans stream the cost volume: with tiles, the blocks of 8
 * steps that every line of a warp covers come as bulk tensor copies, one
 * [8][D] tile a line, into shared memory; without, every lane copies its own
 * 16 bytes a step. Mode 0 never tiles, 2 always, 1 (the default) from 96 Mi
 * pixel-disparities a pair on (1280x720 at 128 and up), where tiles measured
 * faster. A tuning knob for the whole library; results do not depend on it.
 * nxs_path_wait_failures: the path scans' waits on those copies that gave up
 * on the current device (each wait is bounded, about 1 s; 0 unless a copy
 * never landed, after which that launch's path volumes are incomplete). */
nxs_status nxs_set_path_tiles(uint32_t mode);

/* Segments configured after the call (on 1, the default) run a full-search
 * Disparity member split over two streams when no stage before it carries
 * state: each pair's stages up to its census, costs and path volumes on one,
 * its selection and the stages after (TemporalFilter and Quality among them,
 * in request order) on the other, so that one pair's front half runs beside
 * the pair before's back half; pairs alternate between two matcher scratches.
 * Off (0): a segment without state runs each pair wholly on one of two
 * streams, pairs alternating, and one with state on one stream. Results do
 * not depend on it. */
nxs_status nxs_set_split_lanes(uint32_t on);
/* In split segments, the selection on the back stream runs with this many
 * resident blocks a SM stepping through the pixel blocks (8 by default; 0:
 * one block for each, all launched), so that it holds fewer warps beside the
 * next pair's path scan; at most 16. A tuning knob; results do not depend on it.
 * nxs_lean_select: the current setting. */
nxs_status nxs_set_lean_select(uint32_t blocks_per_sm);
uint32_t nxs_lean_select(void);
uint32_t nxs_path_tiles(void);
uint32_t nxs_path_wait_failures(void);

/* The disparity of each left pixel, -1.0 where unmatched: NxStereo.sgm/3 on a
 * rectified u8 pair in host memory (lib/nx_stereo.ex:64-74; natively
 * Matcher::disparity, native/stereo_match/src/lib.rs:105-124). Synchronous. */
nxs_status nxs_sgm(nxs_context *context, const uint8_t *left, const uint8_t *right,
                   uint32_t width, uint32_t height, const nxs_sgm_params *params,
                   float *disparity, char *error, size_t error_len);

/* The same on device buffers, enqueued on `stream` (the context's scratch is
 * used: one call at a time per context and stream). */
nxs_status nxs_sgm_device(nxs_context *context, const uint8_t *d_left, const uint8_t *d_right,
                          uint32_t width, uint32_t height, const nxs_sgm_params *params,
                          float *d_disparity, void *stream, char *error, size_t error_len);

/* nxs_sgm_device for callers that must not allocate device memory: no
 * counterpart in the reference (whose Rust matcher keeps its buffers in host
 * memory). Callers whose device memory belongs to another allocator, or that
 * cannot afford cudaMalloc's device synchronisation on their thread, pass only
 * their inputs and outputs; the matcher's scratch is one fixed 64 MiB array in
 * the library, held on every device that loads it until the process exits.
 * Pairs needing more scratch than that (nxs_sgm_scratch_bytes; about 7 million
 * pixel-disparities, e.g. 364x272 at 64) are refused with NXS_BAD_ARGUMENT.
 * The call works on the calling thread's current device (cudaGetDevice), and
 * `stream` must belong to that device. The first call on a device finds the
 * array's device address (and loads it there); make that first call before
 * any stream capture. The address is kept for the process: after a
 * cudaDeviceReset of that device, this entry point must not be used again.
 * All calls on a device share the array: calls that overlap on the device
 * race, so the caller serialises them. No context is needed and none is
 * used. */
nxs_status nxs_sgm_device_static(const uint8_t *d_left, const uint8_t *d_right, uint32_t width,
                                 uint32_t height, const nxs_sgm_params *params,
                                 float *d_disparity, void *stream, char *error,
                                 size_t error_len);

/* The matcher's device scratch, in bytes, for one pair of this size. */
uint64_t nxs_sgm_scratch_bytes(uint32_t width, uint32_t height, uint32_t disparities);

/* --- the coarse-to-fine search: NxStereo.sgm_coarse_to_fine/3 and
 * NxStereo.sgm_band/4 (lib/nx_stereo.ex:138-471), Stage.Disparity's
 * search "coarse_to_fine" (lib/nx_stereo/stage/disparity.ex:140-158) --- */
typedef struct {
    nxs_sgm_params sgm;    /* 128 disparities for coarse to fine (as sgm/3 checks the rest) */
    uint32_t band;         /* candidates a pixel searches: 8, 16, 32 or 64 */
    uint32_t margin;       /* how far below twice the coarse estimate a band starts, 0..127 */
    uint32_t coarse_paths; /* the half-size match's paths, 3 or 8 */
    uint32_t census;       /* the fine census window: 0 sparse 9x7, 1 dense 9x5,
                              2 dense 9x5 with the blended centre (lib/nx_stereo.ex:491-526) */
} nxs_band_params;

/* Why sgm_band/4 (coarse_to_fine 0) or sgm_coarse_to_fine/3 (non-zero) would
 * refuse these settings: sgm/3's checks (nxs_sgm_check) of the pair and, for
 * coarse to fine, of the half-size pair; the band width and census window;
 * and for coarse to fine an even width and height and 128 disparities
 * (lib/nx_stereo.ex:160-183, 300-312). NXS_OK or NXS_BAD_ARGUMENT. */
nxs_status nxs_band_check(const nxs_band_params *params, uint32_t width, uint32_t height,
                          int32_t coarse_to_fine, char *error, size_t error_len);

/* NxStereo.sgm_band/4 on device buffers: each pixel searches the disparities
 * base .. base + band - 1 of d_base (s32 [height][width]; a negative base
 * marks a pixel with no estimate, searched from 0 and never matched; the
 * caller keeps base + band within the disparities), enqueued on `stream`
 * with the context's scratch. */
nxs_status nxs_sgm_band_device(nxs_context *context, const uint8_t *d_left,
                               const uint8_t *d_right, const int32_t *d_base, uint32_t width,
                               uint32_t height, const nxs_band_params *params,
                               float *d_disparity, void *stream, char *error, size_t error_len);

/* NxStereo.sgm_coarse_to_fine/3 on device buffers: sgm/3 on the pair shrunk
 * 2x (rounded 2x2 means) at 64 disparities with coarse_paths, each pixel's
 * band base from it, then sgm_band/4 over 128 disparities; d_base (may be
 * NULL) receives the bases. With sgm.stage_mask, Stage.Disparity's mask. */
nxs_status nxs_sgm_coarse_to_fine_device(nxs_context *context, const uint8_t *d_left,
                                         const uint8_t *d_right, uint32_t width, uint32_t height,
                                         const nxs_band_params *params, float *d_disparity,
                                         int32_t *d_base, void *stream, char *error,
                                         size_t error_len);

/* The same on a pair in host memory. Synchronous. */
nxs_status nxs_sgm_coarse_to_fine(nxs_context *context, const uint8_t *left,
                                  const uint8_t *right, uint32_t width, uint32_t height,
                                  const nxs_band_params *params, float *disparity, char *error,
                                  size_t error_len);

/* The device scratch, in bytes, of sgm_band/4 (coarse_to_fine 0) or of
 * sgm_coarse_to_fine/3 for one pair. */
uint64_t nxs_band_scratch_bytes(uint32_t width, uint32_t height, uint32_t band,
                                int32_t coarse_to_fine);

/* --- the matcher's steps, for checking intermediates (device buffers) --- */

/* 48-bit 9x7 census codes, u64 per pixel (lib/nx_stereo.ex:491-505). */
nxs_status nxs_census_device(const uint8_t *d_image, uint32_t width, uint32_t height,
                             uint64_t *d_codes, void *stream);

/* Both images' census codes in one launch. */
nxs_status nxs_census_pair_device(const uint8_t *d_left, const uint8_t *d_right, uint32_t width,
                                  uint32_t height, uint64_t *d_left_codes,
                                  uint64_t *d_right_codes, void *stream);

/* u8 Hamming costs, [height][width][disparities] (lib/nx_stereo.ex:528-542). */
nxs_status nxs_costs_device(const uint64_t *d_left_codes, const uint64_t *d_right_codes,
                            uint32_t width, uint32_t height, uint32_t disparities,
                            uint8_t *d_costs, void *stream);

/* The sum of the path costs over every direction, u16
 * [height][width][disparities] (lib/nx_stereo.ex:544-606); disparities a
 * multiple of 32 from 64 to 256. Uses the context's scratch. */
nxs_status nxs_aggregate_device(nxs_context *context, const uint8_t *d_costs, uint32_t width,
                                uint32_t height, uint32_t disparities, uint32_t paths,
                                uint32_t p1, uint32_t p2, uint16_t *d_sums, void *stream);

/* Each direction's path costs, u8 [paths][height][width][disparities], the
 * directions in the reference's order (lib/nx_stereo.ex:544-606): one warp per
 * scan line. d_paths holds `paths` volumes; disparities a multiple of 32
 * from 64 to 256. */
nxs_status nxs_paths_device(const uint8_t *d_costs, uint32_t width, uint32_t height,
                            uint32_t disparities, uint32_t paths, uint32_t p1, uint32_t p2,
                            uint8_t *d_paths, void *stream);

/* Selection straight from the path volumes: their sum, winner, uniqueness and
 * subpixel (lib/nx_stereo.ex:608-641). */
nxs_status nxs_select_paths_device(const uint8_t *d_paths, uint32_t width, uint32_t height,
                                   uint32_t disparities, uint32_t paths, float uniqueness,
                                   float *d_disparity, uint32_t *d_keys, void *stream);

/* The order the matcher keeps its cost and path volumes in: within each run
 * of `span` disparities (8 or 16), bytes 2k and 2k + 1 hold disparities k and
 * k + span / 2, so that a packed pair of path costs has its d - 1 and d + 1
 * neighbours in whole neighbouring words; span 0 is the natural order above.
 * nxs_matcher_span gives the span nxs_sgm uses at this disparity count; the
 * _ordered entry points are nxs_costs_device, nxs_paths_device and
 * nxs_select_paths_device writing and reading their volumes in that order. */
uint32_t nxs_matcher_span(uint32_t disparities);
nxs_status nxs_costs_device_ordered(const uint64_t *d_left_codes, const uint64_t *d_right_codes,
                                    uint32_t width, uint32_t height, uint32_t disparities,
                                    uint32_t span, uint8_t *d_costs, void *stream);
/* The census of both u8 images and the cost volume in one launch, the codes
 * kept in shared memory: the costs nxs_census_pair_device followed by
 * nxs_costs_device_ordered give (lib/nx_stereo.ex:491-542), in the order of
 * `span`; this is the first step nxs_sgm runs. */
nxs_status nxs_census_costs_device_ordered(const uint8_t *d_left, const uint8_t *d_right,
                                           uint32_t width, uint32_t height, uint32_t disparities,
                                           uint32_t span, uint8_t *d_costs, void *stream);
nxs_status nxs_paths_device_ordered(const uint8_t *d_costs, uint32_t width, uint32_t height,
                                    uint32_t disparities, uint32_t paths, uint32_t p1, uint32_t p2,
                                    uint32_t span, uint8_t *d_paths, void *stream);
nxs_status nxs_select_paths_device_ordered(const uint8_t *d_paths, uint32_t width,
                                           uint32_t height, uint32_t disparities, uint32_t paths,
                                           float uniqueness, uint32_t span, float *d_disparity,
                                           uint32_t *d_keys, void *stream);

/* The aggregation as one sum (lib/nx_stereo.ex:545-573, the sum of the
 * direction volumes that selection reads): every direction's path costs from
 * costs in the span-16 order added, as the scan goes, into d_sums, a u16
 * volume of width x height x disparities values (disparities a multiple of
 * 16, 64..256) that the call zeroes first and keeps in its own layout; then
 * selection over it, as nxs_select_paths_device_ordered over the path
 * volumes. The two give the same disparities and keys. */
nxs_status nxs_path_sums_device(const uint8_t *d_costs, uint32_t width, uint32_t height,
                                uint32_t disparities, uint32_t paths, uint32_t p1, uint32_t p2,
                                uint16_t *d_sums, void *stream);
nxs_status nxs_select_path_sums_device(const uint16_t *d_sums, uint32_t width, uint32_t height,
                                       uint32_t disparities, float uniqueness,
                                       float *d_disparity, uint32_t *d_keys, void *stream);

/* Winner, uniqueness and subpixel from u16 sums: f32 disparity and u32 keys
 * (lib/nx_stereo.ex:608-641). */
nxs_status nxs_select_device(const uint16_t *d_sums, uint32_t width, uint32_t height,
                             uint32_t disparities, float uniqueness, float *d_disparity,
                             uint32_t *d_keys, void *stream);

/* The left-right check (lib/nx_stereo.ex:643-683). */
nxs_status nxs_consistency_device(const float *d_disparity, const uint32_t *d_keys,
                                  uint32_t width, uint32_t height, float *d_checked,
                                  void *stream);

/* The 3x3 median (lib/nx_stereo/image.ex:483-505), then, when stage_mask is
 * non-zero, Stage.Disparity's mask (stage/disparity.ex:162). */
nxs_status nxs_median3_device(const float *d_image, uint32_t width, uint32_t height,
                              uint32_t stage_mask, float *d_filtered, void *stream);

/* nxs_consistency_device followed by nxs_median3_device in one pass, as the
 * matcher runs them (width at most 4096). */
nxs_status nxs_check_median_device(const float *d_disparity, const uint32_t *d_keys,
                                   uint32_t width, uint32_t height, uint32_t stage_mask,
                                   float *d_filtered, void *stream);

/* --- the stages around the matcher (device buffers) --- */

/* A camera as NxStereo.Rectify.camera/4 builds it, rows moved by the stage
 * (lib/nx_stereo/rectify.ex:20-50, stage/rectification.ex:84-89): the camera
 * matrix, the plumb_bob coefficients k1 k2 p1 p2 k3 and the inverse of
 * (rectified camera matrix x rectifying rotation), row-major f32. */
typedef struct {
    float k[9];
    float d[5];
    float inverse_pr[9];
} nxs_camera;

/* NxStereo.Rectify.rectify/3 of a frame to width x height
 * (lib/nx_stereo/rectify.ex:133-207). Frames must be at least the working
 * size (stage/rectification.ex:75-82). */
nxs_status nxs_rectify_device(const uint8_t *d_frame, uint32_t frame_width,
                              uint32_t frame_height, const nxs_camera *camera, uint32_t width,
                              uint32_t height, uint8_t *d_rectified, void *stream);

/* Both frames of a pair, each through its own camera, in one launch
 * (Stage.Rectification's step, lib/nx_stereo/stage/rectification.ex:48-58). */
nxs_status nxs_rectify_pair_device(const uint8_t *d_left_frame, const uint8_t *d_right_frame,
                                   uint32_t frame_width, uint32_t frame_height,
                                   const nxs_camera *left, const nxs_camera *right, uint32_t width,
                                   uint32_t height, uint8_t *d_left, uint8_t *d_right,
                                   void *stream);

/* The rectification split in two: the frame position every rectified pixel of
 * both sides samples, d_maps[side][y][x] = (x, y) as f32 (2 x height x width
 * pairs, 8-byte aligned; a function of the cameras and sizes alone), then the
 * pair sampled from its frames through them. The two give nxs_rectify_pair_device's
 * bytes; a segment keeps the maps on the device and remakes them only when a
 * request's cameras change. */
nxs_status nxs_rectify_maps_device(const nxs_camera *left, const nxs_camera *right,
                                   uint32_t frame_width, uint32_t frame_height, uint32_t width,
                                   uint32_t height, float *d_maps, void *stream);
nxs_status nxs_rectify_pair_mapped_device(const uint8_t *d_left_frame,
                                          const uint8_t *d_right_frame, uint32_t frame_width,
                                          uint32_t frame_height, const float *d_maps,
                                          uint32_t width, uint32_t height, uint8_t *d_left,
                                          uint8_t *d_right, void *stream);

/* NxStereo.Filter.despeckle/2 (lib/nx_stereo/filter.ex:14-80); radius 1..8. */
nxs_status nxs_despeckle_device(const float *d_disparity, uint32_t width, uint32_t height,
                                float min_support, float max_diff, uint32_t radius,
                                float *d_despeckled, void *stream);

/* NxStereo.Filter.temporal/4 in place (lib/nx_stereo/filter.ex:82-130). */
nxs_status nxs_temporal_device(float *d_disparity, float *d_previous, float *d_missed,
                               uint64_t pixels, float alpha, float delta, float hold,
                               float max_missed, void *stream);

/* NxStereo.Depth.depth/3 (lib/nx_stereo/depth.ex:8-32). */
nxs_status nxs_depth_device(const float *d_disparity, uint64_t pixels, float focal_length_px,
                            float baseline_m, uint16_t *d_depth_mm, float *d_depth_m,
                            void *stream);

/* NxStereo.Depth.point_cloud/5 (lib/nx_stereo/depth.ex:34-89): the
 * {height/decimation, width/decimation, 3} grid and the kept count (s32). */
nxs_status nxs_cloud_device(const float *d_depth_m, uint32_t width, uint32_t height,
                            uint32_t decimation, float focal_length_px, float cx, float cy,
                            float nearest_m, float farthest_m, float *d_grid, int32_t *d_kept,
                            void *stream);

/* SpeckleFilter -> Depth -> PointCloud in one launch: the outputs of
 * nxs_despeckle_device, then nxs_depth_device on its result, then
 * nxs_cloud_device on that depth, bit for bit (radius 1..5). */
nxs_status nxs_despeckle_depth_cloud_device(const float *d_disparity, uint32_t width,
                                            uint32_t height, float min_support, float max_diff,
                                            uint32_t radius, float focal_length_px,
                                            float baseline_m, uint32_t decimation, float cx,
                                            float cy, float nearest_m, float farthest_m,
                                            float *d_despeckled, uint16_t *d_depth_mm,
                                            float *d_depth_m, float *d_grid, int32_t *d_kept,
                                            void *stream);

/* Stage.Quality's sums (lib/nx_stereo/diagnostics.ex:258-271), f32[5]; then
 * previous := disparity. */
nxs_status nxs_quality_device(const float *d_disparity, float *d_previous, uint32_t width,
                              uint32_t height, float *d_sums, void *stream);


/* ------------------------------------------------------------------------ */
/* Layer 3: batched matching                                                 */
/*
 * Many rectified pairs of uneven size and disparity range matched in one
 * persistent, graph-captured launch: NxStereo.sgm/3 (lib/nx_stereo.ex:64-74)
 * on each pair, with Stage.Disparity's mask where a pair asks for it, bit for
 * bit as nxs_sgm gives it. The reference matches pairs one call at a time
 * (Matcher::disparity, native/stereo_match/src/lib.rs:105-124); a batch is
 * planned once (buffers, work queue, graphs) and run many times.
 */
typedef struct nxs_batch nxs_batch;

typedef struct {
    uint32_t width, height;
    nxs_sgm_params params;
} nxs_batch_pair;

/* Shapes of the batched launch, which nx_stereo_b200.batch's autotuner picks. */
typedef struct {
    int32_t blocks_per_sm;  /* resident blocks of 128 threads per SM, 1..16 */
    int32_t cost_rows;      /* rows of 64 pixels per costs item, 1..64 */
    int32_t select_passes;  /* 128 / lanes pixels per pass, passes per selection item */
    int32_t group_pairs;    /* pairs a group of the queue's pipeline holds, 1..1024 */
    float quantum_us;       /* whole-GPU microseconds of one run of a phase in the queue */
    int32_t order;          /* 0: the group pipeline; 1: each phase over all pairs in turn */
    int32_t path_words;     /* u16x2 words a path lane holds, 4, 8 or 16; 0: nxs_path_words */
    int32_t engine;         /* 0: one persistent launch over the work queue; 1: each pair's
                               single-pair kernels as a chain on one of `streams` streams,
                               the chains overlapping (both in one CUDA graph) */
    int32_t streams;        /* streams of engine 1, 1..64 */
    uint32_t wait_limit_us; /* engine 0: the longest an item waits for the phase before it,
                               1..60,000,000 us, after which the launch records a timeout
                               and ends (NXS_TIMEOUT); 0: 2 s */
} nxs_batch_tuning;

typedef struct {
    uint32_t pairs, items, runs, blocks;
    uint64_t shared_bytes, device_bytes, input_bytes, output_bytes;
} nxs_batch_stats;

void nxs_batch_default_tuning(nxs_batch_tuning *tuning);

/* Plans a batch: every pair is checked as nxs_sgm_check does; the device
 * memory of all pairs is allocated at once (NXS_BAD_ARGUMENT when it does not
 * fit); `tuning` may be NULL for the defaults. */
nxs_status nxs_batch_create(nxs_context *context, uint32_t n_pairs, const nxs_batch_pair *pairs,
                            const nxs_batch_tuning *tuning, nxs_batch **batch, char *error,
                            size_t error_len);

/* Pair `pair`'s images and disparity: in pinned host memory (device_side 0),
 * which nxs_batch_run copies in and out, or on the device (device_side 1). */
nxs_status nxs_batch_buffers(nxs_batch *batch, uint32_t pair, int32_t device_side,
                             uint8_t **left, uint8_t **right, float **disparity);

/* Re-plans the batch for other shapes (the buffers and their contents stay). */
nxs_status nxs_batch_retune(nxs_batch *batch, const nxs_batch_tuning *tuning, char *error,
                            size_t error_len);

/* Matches every pair: the host images in, one launch, the disparities out.
 * Synchronous; NXS_TIMEOUT if a wait inside the launch ran out. */
nxs_status nxs_batch_run(nxs_batch *batch, char *error, size_t error_len);

/* Enqueues one run on `stream` (NULL: the batch's own stream) without
 * waiting: with host_buffers, the copies in and out are part of it;
 * otherwise the device buffers are used as they are. */
nxs_status nxs_batch_launch(nxs_batch *batch, int32_t host_buffers, void *stream, char *error,
                            size_t error_len);

/* After a launch has finished: NXS_TIMEOUT if a wait inside it ran out. */
nxs_status nxs_batch_check(nxs_batch *batch, char *error, size_t error_len);

/* For testing the bounded waits of engine 0: plans phase `phase` (1..5, costs
 * to median) of pair `pair` to wait for one item more of the phase before it
 * than that phase has, a dependency no launch meets, so every such wait runs
 * out after wait_limit_us and nxs_batch_run returns NXS_TIMEOUT. The change
 * is to the device copy of the plan only; nxs_batch_retune plans afresh. */
nxs_status nxs_batch_hold_phase(nxs_batch *batch, uint32_t pair, uint32_t phase, char *error,
                                size_t error_len);

nxs_status nxs_batch_info(const nxs_batch *batch, nxs_batch_stats *stats);

/* Where the last launch spent its blocks' time (call it once the launch has
 * finished; the batch's own stream is waited for), in SM cycles summed over
 * blocks, 16 values: cycles[k] for the items of phase k (census, costs,
 * paths, selection, check, median), cycles[6 + k] for phase k's items
 * waiting for phase k - 1, cycles[12] taking items from the queue. */
nxs_status nxs_batch_clocks(nxs_batch *batch, uint64_t *cycles);

/* The work queue nxs_batch_create would lay out, computed on the host only:
 * items[6 * i + k] is the number of items of phase k (census, costs, paths,
 * selection, check, median) of pair i, and each run r of the queue is
 * runs[4r..4r+3] = (first queue position, pair, phase, first item of the
 * phase); a run ends where the next begins, the last at the total. Runs are
 * written when `capacity` holds them all; *n_runs is always set. */
nxs_status nxs_batch_queue(uint32_t n_pairs, const nxs_batch_pair *pairs,
                           const nxs_batch_tuning *tuning, uint32_t *items, uint32_t *runs,
                           uint32_t capacity, uint32_t *n_runs, char *error, size_t error_len);

void nxs_batch_destroy(nxs_batch *batch);

#ifdef __cplusplus
}
#endif
#endif
