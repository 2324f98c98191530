// Launchers of the device kernels (one stream each, asynchronous). Sizes are
// checked by the callers; each launcher returns cudaGetLastError().
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

struct nxs_context;

namespace nxs {

// Directions in the reference's order (lib/nx_stereo.ex:566-570,
// native/stereo_match/src/reference.rs:123-129).
constexpr int kDirections[8][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0},
                                   {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

struct Camera {
    float k[9];
    float d[5];
    float inverse_pr[9];
};

// ---- the matcher ----
// codes[image][y][x]: image 0 from `left`, 1 from `right` (right may be null
// to run one image).
cudaError_t launch_census(const uint8_t *left, const uint8_t *right, int width, int height,
                          uint64_t *left_codes, uint64_t *right_codes, cudaStream_t stream);
// span 8 or 16: each run of `span` disparities in the permuted order of
// span_disparity (the matcher's internal order); 0: d0, d1, d2, ...
cudaError_t launch_costs(const uint64_t *left_codes, const uint64_t *right_codes, int width,
                         int height, int disparities, uint8_t *costs, cudaStream_t stream,
                         int span = 0);
// The census of both images and the costs in one launch (the codes stay in
// shared memory): the same costs as launch_census then launch_costs.
cudaError_t launch_census_costs(const uint8_t *left, const uint8_t *right, int width, int height,
                                int disparities, uint8_t *costs, cudaStream_t stream,
                                int span = 0);
// paths_out[p][y][x][d] (u8) for p < paths; span 8 or 16: costs and path
// costs in that permuted order (span 0: natural).
cudaError_t launch_paths(const uint8_t *costs, int width, int height, int disparities, int paths,
                         int p1, int p2, uint8_t *paths_out, cudaStream_t stream, int span = 0);
// The order the matcher keeps its costs and path volumes in at this many
// disparities: 8 with 4 words a path lane, 16 otherwise.
int matcher_span(int disparities);
// The summing path scan: the aggregate volume (u16, the lane-split layout of
// sum_position in span-16 order, D a multiple of 16) zeroed, then every
// direction's path costs added into it; selection over it with
// launch_select_path_sums.
cudaError_t launch_paths_sums(const uint8_t *costs, int width, int height, int disparities,
                              int paths, int p1, int p2, uint16_t *sums, cudaStream_t stream);
cudaError_t launch_select_path_sums(const uint16_t *sums, int width, int height,
                                    int disparities, float uniqueness, float *disparity,
                                    uint32_t *keys, cudaStream_t stream);
// Whether the matcher aggregates with the summing scan at this size, by the
// mode of set_path_sums (0 never, the default; 1 where the layout allows).
bool path_sums_wanted(int width, int height, int disparities);
void set_path_sums(int mode);
int path_sums_mode();
// Whether the path scans take the costs of the blocks of steps every line of
// a warp covers by bulk tensor copies: 0 never, 1 (the default) for large
// pairs, 2 always.
void set_path_tiles(int mode);
int path_tiles();
// The path scans' waits on their tensor copies that ran out of tries since
// the library was loaded on this device (0 unless a copy never landed).
unsigned path_wait_failures();
// sums[y][x][d] = sum over paths of paths_in (u16).
cudaError_t launch_sum_paths(const uint8_t *paths_in, int width, int height, int disparities,
                             int paths, uint16_t *sums, cudaStream_t stream);
// lean > 0: that many resident blocks a SM step through the pixel blocks.
cudaError_t launch_select_paths(const uint8_t *paths_in, int width, int height, int disparities,
                                int paths, float uniqueness, float *disparity, uint32_t *keys,
                                cudaStream_t stream, int span = 0, int lean = 0);
void set_lean_select(int blocks_per_sm);
int lean_select();
cudaError_t launch_select_sums(const uint16_t *sums, int width, int height, int disparities,
                               float uniqueness, float *disparity, uint32_t *keys,
                               cudaStream_t stream);
cudaError_t launch_consistency(const float *disparity, const uint32_t *keys, int width,
                               int height, float *checked, cudaStream_t stream);
// The left-right check and the median (with the stage mask) in one pass.
cudaError_t launch_check_median(const float *disparity, const uint32_t *keys, int width,
                                int height, int stage_mask, float *filtered, cudaStream_t stream);
cudaError_t launch_median3(const float *image, int width, int height, int stage_mask,
                           float *filtered, cudaStream_t stream);

// ---- the stages around it ----
// The frame positions both sides' rectified pixels sample, maps[side][v][u]
// (2 x height x width), and the pair rectified from them: launch_rectify_maps
// then launch_rectify_mapped gives launch_rectify_pair's bytes.
cudaError_t launch_rectify_maps(const Camera &left_camera, const Camera &right_camera,
                                int frame_width, int frame_height, int width, int height,
                                float2 *maps, cudaStream_t stream);
cudaError_t launch_rectify_mapped(const uint8_t *left_frame, const uint8_t *right_frame,
                                  int frame_width, int frame_height, const float2 *maps,
                                  int width, int height, uint8_t *left, uint8_t *right,
                                  cudaStream_t stream);
// Both sides of a pair in one launch (scale as launch_rectify).
cudaError_t launch_rectify_pair(const uint8_t *left_frame, const uint8_t *right_frame,
                                int frame_width, int frame_height, const Camera &left_camera,
                                const Camera &right_camera, int width, int height,
                                uint8_t *left, uint8_t *right, cudaStream_t stream);
cudaError_t launch_rectify(const uint8_t *frame, int frame_width, int frame_height,
                           const Camera &camera, int width, int height, uint8_t *rectified,
                           cudaStream_t stream);
cudaError_t launch_despeckle(const float *disparity, int width, int height, float min_support,
                             float max_diff, int radius, float *despeckled, cudaStream_t stream);
cudaError_t launch_temporal(float *disparity, float *previous, float *missed, size_t pixels,
                            float alpha, float delta, float hold, float max_missed,
                            cudaStream_t stream);
cudaError_t launch_depth(const float *disparity, size_t pixels, float focal_length_px,
                         float baseline_m, uint16_t *depth_mm, float *depth_m,
                         cudaStream_t stream);
cudaError_t launch_cloud(const float *depth_m, int width, int height, int decimation,
                         float focal_length_px, float cx, float cy, float nearest_m,
                         float farthest_m, float *grid, int32_t *kept, cudaStream_t stream);
// launch_despeckle, launch_depth and launch_cloud in one launch (radius 1..5).
cudaError_t launch_despeckle_depth_cloud(const float *disparity, int width, int height,
                                         float min_support, float max_diff, int radius,
                                         float focal_length_px, float baseline_m,
                                         int decimation, float cx, float cy, float nearest_m,
                                         float farthest_m, float *despeckled, uint16_t *depth_mm,
                                         float *depth_m, float *grid, int32_t *kept,
                                         cudaStream_t stream);
// column_sums: scratch of 5 * width floats.
cudaError_t launch_quality(const float *disparity, float *previous, int width, int height,
                           float *column_sums, float *sums, cudaStream_t stream);

// The matcher's device scratch for one pair, and its layout: the cost volume,
// the path volumes, and selection's disparities and keys (the census codes stay
// in shared memory; the check and median write the output).
struct MatcherScratch {
    uint8_t *costs;
    uint8_t *paths;
    float *selected;
    uint32_t *keys;
};
size_t matcher_scratch_bytes(int width, int height, int disparities);
MatcherScratch carve_matcher_scratch(void *base, int width, int height, int disparities);

// The whole matcher on device buffers: census, costs, paths, selection, the
// check and the median (with Stage.Disparity's mask when stage_mask). beside:
// the selection runs beside other pairs' path scans (the lean grid of
// set_lean_select).
cudaError_t run_matcher(const uint8_t *left, const uint8_t *right, int width, int height,
                        int disparities, int paths, int p1, int p2, float uniqueness,
                        int stage_mask, const MatcherScratch &scratch, float *disparity,
                        cudaStream_t stream, bool beside = false);
// Its two halves: the census, costs and path volumes (front); selection, the
// check and the median from the path volumes (back). run_matcher runs both on
// one stream; a segment may run them on two, pairs apart.
cudaError_t run_matcher_front(const uint8_t *left, const uint8_t *right, int width, int height,
                              int disparities, int paths, int p1, int p2,
                              const MatcherScratch &scratch, cudaStream_t stream);
cudaError_t run_matcher_back(int width, int height, int disparities, int paths,
                             float uniqueness, int stage_mask, const MatcherScratch &scratch,
                             float *disparity, cudaStream_t stream, bool beside = false);

// ---- the coarse-to-fine search (band.cu) ----
// Both images' rounded 2x2 means.
cudaError_t launch_shrink_pair(const uint8_t *left, const uint8_t *right, int width, int height,
                               uint8_t *left_half, uint8_t *right_half, cudaStream_t stream);
// Each full-size pixel's band base from the coarse disparity {ch, cw}.
cudaError_t launch_band_base(const float *coarse, int coarse_width, int coarse_height, int band,
                             int margin, int32_t *base, cudaStream_t stream);
// window 0: the sparse 9x7 census (launch_census); 1: dense 9x5; 2: dense 9x5 blended.
cudaError_t launch_census_window(const uint8_t *left, const uint8_t *right, int width,
                                 int height, int window, uint64_t *left_codes,
                                 uint64_t *right_codes, cudaStream_t stream);
cudaError_t launch_band_costs(const uint64_t *left_codes, const uint64_t *right_codes,
                              const int32_t *base, int width, int height, int band,
                              uint8_t *costs, cudaStream_t stream);
cudaError_t launch_band_paths(const uint8_t *costs, const int32_t *base, int width, int height,
                              int band, int paths, int p1, int p2, uint8_t *out,
                              cudaStream_t stream);
cudaError_t launch_band_select(const uint8_t *paths_in, const int32_t *base, int width,
                               int height, int band, int paths, int disparities, float uniqueness,
                               float *disparity, uint32_t *keys, cudaStream_t stream);
int band_lane_values(int band);

// The band matcher's scratch: both images' codes, the bases (when the
// search makes them), the band costs and path volumes, selection's outputs.
struct BandScratch {
    uint64_t *left_codes, *right_codes;
    int32_t *base;
    uint8_t *costs, *paths;
    float *selected;
    uint32_t *keys;
};
size_t band_scratch_bytes(int width, int height, int band);
BandScratch carve_band_scratch(void *base, int width, int height, int band);
// band_scratch_bytes plus the half images, the coarse disparity and the
// coarse matcher's scratch.
size_t coarse_to_fine_scratch_bytes(int width, int height, int band);

// sgm_band/4 on device buffers: `base` s32 [height][width].
cudaError_t run_band_matcher(const uint8_t *left, const uint8_t *right, const int32_t *base,
                             int width, int height, int disparities, int paths, int band,
                             int window, int p1, int p2, float uniqueness, int stage_mask,
                             const BandScratch &scratch, float *disparity, cudaStream_t stream);
// sgm_coarse_to_fine/3 on device buffers (even width and height); the bases
// go to base_out when it is not null. `scratch` holds
// coarse_to_fine_scratch_bytes.
cudaError_t run_coarse_to_fine(const uint8_t *left, const uint8_t *right, int width, int height,
                               int paths, int coarse_paths, int band, int margin, int window,
                               int p1, int p2, float uniqueness, int stage_mask, void *scratch,
                               float *disparity, int32_t *base_out, cudaStream_t stream);

// The device a context was opened on.
int context_device(nxs_context *context);

// The warp layout of one pair's path launch with `lanes` lanes a scan line;
// returns the number of warps.
int path_setup(int width, int height, int disparities, int paths, int p1, int p2, int lanes,
               struct PathSetup *setup);

// Words (4, 8 or 16, so 8, 16 or 32 disparities) a path lane holds at this
// many disparities, and setting it.
int path_words(int disparities);
void set_path_words(int disparities, int words);

}  // namespace nxs
