/*
 * CPU oracle for the NxStereo full-search Stage.Disparity path and the stages
 * around it. TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the
 * CPU-baseline leg of bench.py call it as the checker; the product path never
 * links, loads or calls it.
 *
 * Two formulations live here:
 *   - nxs_oracle.c: a literal restatement of NxStereo's Nx definition
 *     (lib/nx_stereo.ex:475-683) as the reference's own test transcription
 *     does it (native/stereo_match/src/reference.rs), on full int32 volumes;
 *   - nxs_oracle_fast.c: the optimised CPU formulation of the reference's
 *     Rust matcher (byte path states with sentinels, a horizontal pass per
 *     row, a down sweep into u16 totals and an up sweep with selection),
 *     used as a differential check of the first and as the timed CPU
 *     baseline.
 *
 * Parity is pinned by the reference's known-answer tests, restated in
 * tests/test_oracle_known_answers.py (the reference ships no stored golden
 * vectors).
 */
#ifndef NXS_ORACLE_H
#define NXS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_INVALID_KEY 0xFFFFFFFFu

/* ---- the matcher, step by step (reference.rs, nx_stereo.ex) ---- */
void oracle_census(const uint8_t *image, int width, int height, uint64_t *codes);
void oracle_costs(const uint64_t *left, const uint64_t *right, int width, int height,
                  int disparities, int32_t *costs);
void oracle_path(const int32_t *costs, int width, int height, int disparities, int dy, int dx,
                 int p1, int p2, int32_t *path);
void oracle_aggregate(const int32_t *costs, int width, int height, int disparities, int paths,
                      int p1, int p2, int32_t *sums);
void oracle_select(const int32_t *sums, int width, int height, int disparities, float uniqueness,
                   float *disparity, uint32_t *keys);
void oracle_consistency(const float *disparity, const uint32_t *keys, int width, int height,
                        int disparities, float *consistent);
void oracle_median3(const float *image, int width, int height, float *filtered);
/* NxStereo.sgm/3: returns 0, or -1 when the sizes are refused. */
int oracle_sgm(const uint8_t *left, const uint8_t *right, int width, int height,
               int disparities, int paths, int p1, int p2, float uniqueness, float *disparity);
/* Stage.Disparity's step: sgm/3, then disparity 0 (or less) becomes -1. */
int oracle_disparity_stage(const uint8_t *left, const uint8_t *right, int width, int height,
                           int disparities, int paths, int p1, int p2, float uniqueness,
                           float *disparity);

/* ---- the coarse-to-fine search (nxs_oracle_band.c) ---- */
#define ORACLE_SPARSE_9X7 0
#define ORACLE_DENSE_9X5 1
#define ORACLE_DENSE_9X5_BLEND 2
void oracle_census_window(const uint8_t *image, int width, int height, int window,
                          uint64_t *codes);
void oracle_shrink(const uint8_t *image, int width, int height, uint8_t *half);
void oracle_band_base(const float *coarse, int coarse_width, int coarse_height, int band,
                      int margin, int32_t *base);
void oracle_band_costs(const uint64_t *left, const uint64_t *right, const int32_t *searched,
                       int width, int height, int band, int32_t *costs);
void oracle_band_path(const int32_t *costs, const int32_t *searched, int width, int height,
                      int band, int dy, int dx, int p1, int p2, int32_t *path);
void oracle_band_aggregate(const int32_t *costs, const int32_t *searched, int width, int height,
                           int band, int paths, int p1, int p2, int32_t *sums);
void oracle_band_select(const int32_t *sums, const int32_t *base, int width, int height, int band,
                        int disparities, float uniqueness, float *disparity, uint32_t *keys);
int oracle_sgm_band(const uint8_t *left, const uint8_t *right, const int32_t *base, int width,
                    int height, int disparities, int paths, int band, int window, int p1, int p2,
                    float uniqueness, float *disparity);
/* base_out (may be NULL) receives the band bases of the fine pass. */
int oracle_sgm_coarse_to_fine(const uint8_t *left, const uint8_t *right, int width, int height,
                              int paths, int coarse_paths, int band, int margin, int fine_window,
                              int p1, int p2, float uniqueness, float *disparity,
                              int32_t *base_out);

/* ---- the stages around the matcher ---- */
typedef struct {
    float k[9];          /* camera matrix, row-major */
    float d[5];          /* plumb_bob k1, k2, p1, p2, k3 */
    float inverse_pr[9]; /* inverse of (rectified camera matrix x rectifying rotation) */
} oracle_camera;

void oracle_rectify(const uint8_t *frame, int frame_width, int frame_height,
                    const oracle_camera *camera, int width, int height, uint8_t *rectified);
void oracle_despeckle(const float *disparity, int width, int height, float min_support,
                      float max_diff, int radius, float *despeckled);
void oracle_temporal(float *disparity, float *previous, float *missed, size_t pixels,
                     float alpha, float delta, float hold, float max_missed);
void oracle_depth(const float *disparity, size_t pixels, float focal_length_px,
                  float baseline_m, uint16_t *depth_mm, float *depth_m);
int32_t oracle_cloud(const float *depth_m, int width, int height, int decimation,
                     float focal_length_px, float cx, float cy, float nearest_m,
                     float farthest_m, float *grid);
void oracle_quality(const float *disparity, float *previous, int width, int height,
                    float sums[5]);

/* ---- the reference tests' generators (lib.rs test module) ---- */
uint64_t oracle_random_seed(uint64_t seed);
uint64_t oracle_random_next(uint64_t *state);
void oracle_noise(int width, int height, uint64_t seed, uint8_t *image);
void oracle_scene(int width, int height, uint64_t seed, uint8_t *left, uint8_t *right);

/* ---- the optimised CPU formulation (nxs_oracle_fast.c) ---- */
/* One pair; scratch is allocated per call. Returns 0, or -1 on refusal. */
int oracle_fast_sgm(const uint8_t *left, const uint8_t *right, int width, int height,
                    int disparities, int paths, int p1, int p2, float uniqueness,
                    float *disparity);
/* `pairs` pairs of the same size on `threads` threads, a whole pair per
 * thread at a time; lefts/rights/outputs are pair-major. Returns 0 or -1. */
int oracle_fast_sgm_batch(const uint8_t *lefts, const uint8_t *rights, int pairs, int width,
                          int height, int disparities, int paths, int p1, int p2,
                          float uniqueness, float *disparities_out, int threads);

/* The full frame-to-depth chain per pair (rectification of both frames, the
 * matcher with Stage.Disparity's mask, despeckle, depth, point cloud) on
 * `threads` threads, a whole pair per thread at a time. Frames are pair-major
 * [pairs][frame_height][frame_width]; disparities_out [pairs][height][width]
 * (may be NULL). Returns the total of kept cloud points, or -1. */
long oracle_fast_pipeline_batch(const uint8_t *left_frames, const uint8_t *right_frames,
                                int pairs, int frame_width, int frame_height,
                                const oracle_camera *left_camera,
                                const oracle_camera *right_camera, int width, int height,
                                int disparities, int paths, int p1, int p2, float uniqueness,
                                float min_support, float max_diff, float focal_length_px,
                                float baseline_m, int decimation, float cx, float cy,
                                float nearest_m, float farthest_m, float *disparities_out,
                                int threads);

#ifdef __cplusplus
}
#endif
#endif
