/*
 * The CPU oracle: NxStereo's full-search matcher and the stages around it,
 * restated step by step. TEST INFRASTRUCTURE ONLY (see nxs_oracle.h).
 *
 * Compiled with -ffp-contract=off: every f32 expression is evaluated one
 * rounded operation at a time, in the order the reference writes it, as
 * Nx's evaluator and the reference's Rust port compute it.
 *
 * Citations are paths within the NxStereo repository.
 */
#include "nxs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* 9x7 sparse census: bit i for the i-th neighbour in row-major order over
 * dy in -3..3, dx in -4..4, both non-zero; set where the neighbour plus one is
 * below the centre, borders replicated.
 * lib/nx_stereo.ex:492-505 (neighbours 503-505), lib/nx_stereo/image.ex:508-537
 * (shift replicates the border), native/stereo_match/src/reference.rs:8-38. */
void oracle_census(const uint8_t *image, int width, int height, uint64_t *codes) {
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            int centre = image[y * width + x];
            uint64_t code = 0;
            int bit = 0;
            for (int dy = -3; dy <= 3; ++dy) {
                if (dy == 0) continue;
                for (int dx = -4; dx <= 4; ++dx) {
                    if (dx == 0) continue;
                    int sy = clampi(y + dy, 0, height - 1);
                    int sx = clampi(x + dx, 0, width - 1);
                    if ((int)image[sy * width + sx] + 1 < centre) code |= (uint64_t)1 << bit;
                    ++bit;
                }
            }
            codes[y * width + x] = code;
        }
    }
}

/* costs[(y * width + x) * D + d] = popcount(left[y, x] ^ right[y, x - d]),
 * right codes left of the image being zero.
 * lib/nx_stereo.ex:528-542, reference.rs:40-63. */
void oracle_costs(const uint64_t *left, const uint64_t *right, int width, int height,
                  int disparities, int32_t *costs) {
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x)
            for (int d = 0; d < disparities; ++d) {
                uint64_t feature = x >= d ? right[y * width + x - d] : 0;
                costs[((size_t)y * width + x) * disparities + d] =
                    __builtin_popcountll(left[y * width + x] ^ feature);
            }
}

/* One path of libSGM's normalised recurrence: pixel (y, x) continues the path
 * from (y - dy, x - dx), from zero outside the image:
 *   a = prev - min(prev);
 *   L[d] = min(min(a[d], p2), min(a[d-1], a[d+1]) + p1) + C[d],
 * out-of-range neighbours reading p2 - p1.
 * lib/nx_stereo.ex:575-606 (scan, follow), reference.rs:65-121. */
void oracle_path(const int32_t *costs, int width, int height, int disparities, int dy, int dx,
                 int p1, int p2, int32_t *path) {
    int32_t *normalized = (int32_t *)malloc(sizeof(int32_t) * disparities);
    for (int r = 0; r < height; ++r) {
        int y = dy < 0 ? height - 1 - r : r;
        for (int c = 0; c < width; ++c) {
            int x = dx < 0 ? width - 1 - c : c;
            int py = y - dy, px = x - dx;
            int inside = py >= 0 && py < height && px >= 0 && px < width;
            const int32_t *previous =
                inside ? path + ((size_t)py * width + px) * disparities : NULL;
            int32_t minimum = 0;
            if (inside) {
                minimum = previous[0];
                for (int d = 1; d < disparities; ++d)
                    if (previous[d] < minimum) minimum = previous[d];
            }
            for (int d = 0; d < disparities; ++d)
                normalized[d] = inside ? previous[d] - minimum : 0;
            size_t at = ((size_t)y * width + x) * disparities;
            for (int d = 0; d < disparities; ++d) {
                int32_t lower = d == 0 ? p2 - p1 : normalized[d - 1];
                int32_t upper = d == disparities - 1 ? p2 - p1 : normalized[d + 1];
                int32_t jump = normalized[d] < p2 ? normalized[d] : p2;
                int32_t step = (lower < upper ? lower : upper) + p1;
                path[at + d] = (jump < step ? jump : step) + costs[at + d];
            }
        }
    }
    free(normalized);
}

/* The aggregation directions in the reference's order: left to right, right
 * to left, top to bottom, then bottom to top and the four diagonals.
 * lib/nx_stereo.ex:545-573, reference.rs:123-146. */
static const int DIRECTIONS[8][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0},
                                     {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

void oracle_aggregate(const int32_t *costs, int width, int height, int disparities, int paths,
                      int p1, int p2, int32_t *sums) {
    size_t volume = (size_t)width * height * disparities;
    int32_t *path = (int32_t *)malloc(sizeof(int32_t) * volume);
    memset(sums, 0, sizeof(int32_t) * volume);
    int count = paths == 8 ? 8 : 3;
    for (int p = 0; p < count; ++p) {
        oracle_path(costs, width, height, disparities, DIRECTIONS[p][0], DIRECTIONS[p][1], p1,
                    p2, path);
        for (size_t i = 0; i < volume; ++i) sums[i] += path[i];
    }
    free(path);
}

/* Winner with ties to the lowest disparity, disparities past x raised by
 * 0x8000; the uniqueness test on the best cost outside the winner's
 * neighbours; the parabolic subpixel step in f32; the key
 * (best cost << 16) | winner, or 0xFFFFFFFF where not accepted.
 * lib/nx_stereo.ex:608-641, reference.rs:148-186. */
void oracle_select(const int32_t *sums, int width, int height, int disparities, float uniqueness,
                   float *disparity, uint32_t *keys) {
    int32_t *values = (int32_t *)malloc(sizeof(int32_t) * disparities);
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            size_t at = ((size_t)y * width + x) * disparities;
            for (int d = 0; d < disparities; ++d) values[d] = sums[at + d] + (d > x ? 0x8000 : 0);
            int32_t minimum = values[0];
            int winner = 0;
            for (int d = 1; d < disparities; ++d)
                if (values[d] < minimum) { minimum = values[d]; winner = d; }
            int32_t second = 0x7FFFFFFF;
            for (int d = 0; d < disparities; ++d)
                if (abs(d - winner) > 1 && values[d] < second) second = values[d];
            int below = winner - 1 < 0 ? 0 : winner - 1;
            int above = winner + 1 > disparities - 1 ? disparities - 1 : winner + 1;
            float lower = (float)values[below];
            float upper = (float)values[above];
            float minimum_f = (float)minimum;
            int accepted = (float)second > minimum_f * uniqueness;
            float denominator = lower + upper - 2.0f * minimum_f;
            float bounded = denominator > 1.0f ? denominator : 1.0f;
            float correction = (lower - upper) / (2.0f * bounded);
            if (correction < -0.5f) correction = -0.5f;
            if (correction > 0.5f) correction = 0.5f;
            int limit = disparities - 1 < x ? disparities - 1 : x;
            int refine = denominator > 0.0f && winner > 0 && winner < limit;
            float value = (float)winner + (refine ? correction : 0.0f);
            uint32_t key = ((uint32_t)minimum << 16) | (uint32_t)winner;
            disparity[y * width + x] = accepted ? value : -1.0f;
            keys[y * width + x] = accepted ? key : ORACLE_INVALID_KEY;
        }
    }
    free(values);
}

/* OpenCV's left-right check: each right pixel keeps the cheapest left match
 * projected onto it, ties to the larger disparity (key low half 65535 - d); a
 * left pixel is rejected when both floor and ceil of its disparity disagree:
 * inside, found, and more than one apart.
 * lib/nx_stereo.ex:643-683, reference.rs:188-235. */
void oracle_consistency(const float *disparity, const uint32_t *keys, int width, int height,
                        int disparities, float *consistent) {
    uint32_t *right = (uint32_t *)malloc(sizeof(uint32_t) * width);
    for (int y = 0; y < height; ++y) {
        const uint32_t *row = keys + (size_t)y * width;
        for (int rx = 0; rx < width; ++rx) {
            uint32_t best = ORACLE_INVALID_KEY;
            for (int d = 0; d < disparities; ++d) {
                uint32_t key = rx + d < width ? row[rx + d] : ORACLE_INVALID_KEY;
                uint32_t candidate = ORACLE_INVALID_KEY;
                if (key != ORACLE_INVALID_KEY && (int)(key & 0xFFFF) == d)
                    candidate = (key & 0xFFFF0000u) | (uint32_t)(65535 - d);
                if (candidate < best) best = candidate;
            }
            right[rx] = best;
        }
        for (int x = 0; x < width; ++x) {
            float value = disparity[(size_t)y * width + x];
            int low = (int)floorf(value), high = (int)ceilf(value);
            int rejected = 1;
            for (int k = 0; k < 2; ++k) {
                int d = k == 0 ? low : high;
                int rx = x - d;
                int inside = rx >= 0 && rx < width;
                uint32_t found = right[clampi(rx, 0, width - 1)];
                int right_d = 65535 - (int)(found & 0xFFFF);
                int disagrees = inside && found != ORACLE_INVALID_KEY && abs(right_d - d) > 1;
                rejected = rejected && disagrees;
            }
            consistent[(size_t)y * width + x] = (value >= 0.0f && !rejected) ? value : -1.0f;
        }
    }
    free(right);
}

static int compare_floats(const void *a, const void *b) {
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

/* 3x3 median, borders replicated: the middle of the sorted window.
 * lib/nx_stereo/image.ex:483-505, reference.rs:237-254. */
void oracle_median3(const float *image, int width, int height, float *filtered) {
    float window[9];
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            int n = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                    window[n++] = image[clampi(y + dy, 0, height - 1) * width +
                                        clampi(x + dx, 0, width - 1)];
            qsort(window, 9, sizeof(float), compare_floats);
            filtered[(size_t)y * width + x] = window[4];
        }
}

/* sgm_n: census, costs, aggregation, selection, the consistency check and
 * the median. lib/nx_stereo.ex:475-480, reference.rs:256-277. The size check
 * is config!'s (lib/nx_stereo.ex:98-106). */
int oracle_sgm(const uint8_t *left, const uint8_t *right, int width, int height,
               int disparities, int paths, int p1, int p2, float uniqueness, float *disparity) {
    if (!(width > 8 && height > 6 && width <= 4096) || disparities < 2) return -1;
    size_t pixels = (size_t)width * height, volume = pixels * disparities;
    uint64_t *lc = (uint64_t *)malloc(8 * pixels), *rc = (uint64_t *)malloc(8 * pixels);
    int32_t *costs = (int32_t *)malloc(4 * volume), *sums = (int32_t *)malloc(4 * volume);
    float *selected = (float *)malloc(4 * pixels), *checked = (float *)malloc(4 * pixels);
    uint32_t *keys = (uint32_t *)malloc(4 * pixels);
    oracle_census(left, width, height, lc);
    oracle_census(right, width, height, rc);
    oracle_costs(lc, rc, width, height, disparities, costs);
    oracle_aggregate(costs, width, height, disparities, paths, p1, p2, sums);
    oracle_select(sums, width, height, disparities, uniqueness, selected, keys);
    oracle_consistency(selected, keys, width, height, disparities, checked);
    oracle_median3(checked, width, height, disparity);
    free(lc); free(rc); free(costs); free(sums); free(selected); free(checked); free(keys);
    return 0;
}

/* Stage.Disparity.step: a disparity of 0 has no depth and is unmatched.
 * lib/nx_stereo/stage/disparity.ex:162, native/stereo_match/src/segment.rs:407-418. */
int oracle_disparity_stage(const uint8_t *left, const uint8_t *right, int width, int height,
                           int disparities, int paths, int p1, int p2, float uniqueness,
                           float *disparity) {
    int status = oracle_sgm(left, right, width, height, disparities, paths, p1, p2, uniqueness,
                            disparity);
    if (status) return status;
    for (size_t i = 0; i < (size_t)width * height; ++i)
        if (!(disparity[i] > 0.0f)) disparity[i] = -1.0f;
    return 0;
}

/* ---------------------------------------------------------------------- */

/* The projection of rectified pixel (u, v) into the camera frame: inverse
 * rectification, plumb_bob distortion with the radial polynomial summed as
 * 1 + (k3 r2^3 + (k2 r2^2 + k1 r2)), then the camera matrix.
 * lib/nx_stereo/rectify.ex:156-174; native/stereo_match/src/rectify.rs:107-128
 * gives the evaluator's summation order of the radial term. */
static void project(const oracle_camera *camera, float u, float v, float *map_x, float *map_y) {
    const float *ir = camera->inverse_pr;
    float x = ir[0] * u + ir[1] * v + ir[2];
    float y = ir[3] * u + ir[4] * v + ir[5];
    float w = ir[6] * u + ir[7] * v + ir[8];
    x = x / w;
    y = y / w;
    float k1 = camera->d[0], k2 = camera->d[1], t1 = camera->d[2], t2 = camera->d[3],
          k3 = camera->d[4];
    float r2 = x * x + y * y;
    float radial = 1.0f + (k3 * r2 * r2 * r2 + (k2 * r2 * r2 + k1 * r2));
    float xd = x * radial + 2.0f * t1 * x * y + t2 * (r2 + 2.0f * x * x);
    float yd = y * radial + t1 * (r2 + 2.0f * y * y) + 2.0f * t2 * x * y;
    const float *k = camera->k;
    *map_x = k[0] * xd + k[1] * yd + k[2];
    *map_y = k[4] * yd + k[5];
}

static float frame_sample(const uint8_t *frame, int fw, int fh, int x, int y) {
    if (x >= 0 && x < fw && y >= 0 && y < fh) return (float)frame[(size_t)y * fw + x];
    return 0.0f;
}

/* Undistortion, rectification and shrinking in one bilinear sample per
 * pixel, zero outside the frame, rounded half away from zero and clipped.
 * lib/nx_stereo/rectify.ex:133-207, native/stereo_match/src/rectify.rs:34-104. */
void oracle_rectify(const uint8_t *frame, int frame_width, int frame_height,
                    const oracle_camera *camera, int width, int height, uint8_t *rectified) {
    float scale_x = (float)((double)frame_width / (double)width);
    float scale_y = (float)((double)frame_height / (double)height);
    for (int v = 0; v < height; ++v)
        for (int u = 0; u < width; ++u) {
            float map_x, map_y;
            project(camera, (float)u, (float)v, &map_x, &map_y);
            float source_x = (map_x + 0.5f) * scale_x - 0.5f;
            float source_y = (map_y + 0.5f) * scale_y - 0.5f;
            float fx0 = floorf(source_x), fy0 = floorf(source_y);
            float wx = source_x - fx0, wy = source_y - fy0;
            /* f32 -> i32 as Rust's `as` casts: NaN to 0, saturating. */
            int x0 = isnan(fx0) ? 0 : (fx0 >= 2147483647.0f ? 2147483647
                                       : (fx0 <= -2147483648.0f ? (-2147483647 - 1) : (int)fx0));
            int y0 = isnan(fy0) ? 0 : (fy0 >= 2147483647.0f ? 2147483647
                                       : (fy0 <= -2147483648.0f ? (-2147483647 - 1) : (int)fy0));
            float tl = frame_sample(frame, frame_width, frame_height, x0, y0);
            float tr = frame_sample(frame, frame_width, frame_height, x0 + 1, y0);
            float bl = frame_sample(frame, frame_width, frame_height, x0, y0 + 1);
            float br = frame_sample(frame, frame_width, frame_height, x0 + 1, y0 + 1);
            float top = (1.0f - wx) * tl + wx * tr;
            float bottom = (1.0f - wx) * bl + wx * br;
            float value = (1.0f - wy) * top + wy * bottom;
            float r = roundf(value);
            r = r < 0.0f ? 0.0f : (r > 255.0f ? 255.0f : r);
            rectified[(size_t)v * width + u] = (uint8_t)r;
        }
}

/* Keeps a matched pixel where at least min_support of the others in its
 * (2r+1)^2 window matched within max_diff of it; unmatched outside the image.
 * lib/nx_stereo/filter.ex:47-80, native/stereo_match/src/filters.rs:222-268. */
void oracle_despeckle(const float *disparity, int width, int height, float min_support,
                      float max_diff, int radius, float *despeckled) {
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            float centre = disparity[(size_t)y * width + x];
            unsigned support = 0;
            for (int dy = -radius; dy <= radius; ++dy)
                for (int dx = -radius; dx <= radius; ++dx) {
                    if (dy == 0 && dx == 0) continue;
                    int sy = y + dy, sx = x + dx;
                    float n = (sy >= 0 && sy < height && sx >= 0 && sx < width)
                                  ? disparity[(size_t)sy * width + sx]
                                  : -1.0f;
                    support += (n > 0.0f) & (fabsf(n - centre) <= max_diff);
                }
            int kept = centre > 0.0f && (float)support >= min_support;
            despeckled[(size_t)y * width + x] = kept ? centre : -1.0f;
        }
}

/* One step of the temporal filter, in place over disparity, previous and
 * missed. lib/nx_stereo/filter.ex:122-130, native/stereo_match/src/filters.rs:507-530. */
void oracle_temporal(float *disparity, float *previous, float *missed, size_t pixels,
                     float alpha, float delta, float hold, float max_missed) {
    for (size_t i = 0; i < pixels; ++i) {
        float current = disparity[i], before = previous[i];
        int matched = current > 0.0f;
        int agree = matched && before > 0.0f && fabsf(current - before) <= delta;
        float smoothed = agree ? alpha * current + (1.0f - alpha) * before : current;
        float pairs_missed = matched ? 0.0f : missed[i] + 1.0f;
        int held = !matched && before > 0.0f && pairs_missed <= hold;
        float filtered = held ? before : smoothed;
        disparity[i] = filtered;
        previous[i] = filtered;
        missed[i] = pairs_missed < max_missed ? pairs_missed : max_missed;
    }
}

/* depth_m = (f * B) / d where matched, else 0; depth_mm the rounded
 * millimetres, 0 beyond 65535. lib/nx_stereo/depth.ex:26-32,
 * native/stereo_match/src/depth.rs:12-44. */
void oracle_depth(const float *disparity, size_t pixels, float focal_length_px,
                  float baseline_m, uint16_t *depth_mm, float *depth_m) {
    float focal_baseline = focal_length_px * baseline_m;
    for (size_t i = 0; i < pixels; ++i) {
        float d = disparity[i];
        float metres = d > 0.0f ? focal_baseline / d : 0.0f;
        float rounded = roundf(metres * 1000.0f);
        depth_m[i] = metres;
        depth_mm[i] = rounded > 65535.0f ? 0 : (uint16_t)(rounded > 0.0f ? rounded : 0.0f);
    }
}

/* The decimated organised cloud: point (i, j) from pixel (i*dec, j*dec), NaN
 * outside (nearest, farthest), both excluded; returns the kept count.
 * lib/nx_stereo/depth.ex:73-89, native/stereo_match/src/depth.rs:58-89. */
int32_t oracle_cloud(const float *depth_m, int width, int height, int decimation,
                     float focal_length_px, float cx, float cy, float nearest_m,
                     float farthest_m, float *grid) {
    int gw = width / decimation, gh = height / decimation;
    int32_t kept = 0;
    for (int row = 0; row < gh; ++row)
        for (int col = 0; col < gw; ++col) {
            int y = row * decimation, x = col * decimation;
            float z = depth_m[(size_t)y * width + x];
            float *point = grid + 3 * ((size_t)row * gw + col);
            if (z > nearest_m && z < farthest_m) {
                float z_over_f = z / focal_length_px;
                point[0] = ((float)x - cx) * z_over_f;
                point[1] = ((float)y - cy) * z_over_f;
                point[2] = z;
                ++kept;
            } else {
                point[0] = point[1] = point[2] = NAN;
            }
        }
    return kept;
}

/* [matched, sum, sum of squares, matched in both, change]: per-column sums
 * accumulated in f64 and rounded to f32, then summed across columns in f64
 * and rounded; previous := disparity.
 * lib/nx_stereo/diagnostics.ex:264-271, native/stereo_match/src/measures.rs:265-309. */
void oracle_quality(const float *disparity, float *previous, int width, int height,
                    float sums[5]) {
    double *columns = (double *)calloc((size_t)width * 5, sizeof(double));
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            float current = disparity[(size_t)y * width + x];
            float before = previous[(size_t)y * width + x];
            float matched = current > 0.0f ? 1.0f : 0.0f;
            float both = (before > 0.0f ? 1.0f : 0.0f) * matched;
            float value = current * matched;
            float planes[5] = {matched, value, value * value, both,
                               fabsf(current - before) * both};
            for (int p = 0; p < 5; ++p) columns[x * 5 + p] += (double)planes[p];
        }
    for (int p = 0; p < 5; ++p) {
        double total = 0.0;
        for (int x = 0; x < width; ++x) total += (double)(float)columns[x * 5 + p];
        sums[p] = (float)total;
    }
    memcpy(previous, disparity, sizeof(float) * (size_t)width * height);
    free(columns);
}

/* ---------------------------------------------------------------------- */

/* The xorshift generator of the reference's tests, and its images.
 * native/stereo_match/src/lib.rs:447-508. */
uint64_t oracle_random_seed(uint64_t seed) { return (seed * 0x9E3779B97F4A7C15ull) | 1ull; }

uint64_t oracle_random_next(uint64_t *state) {
    uint64_t x = *state;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    *state = x;
    return x;
}

void oracle_noise(int width, int height, uint64_t seed, uint8_t *image) {
    uint64_t state = oracle_random_seed(seed);
    for (size_t i = 0; i < (size_t)width * height; ++i)
        image[i] = (uint8_t)(oracle_random_next(&state) >> 24);
}

/* A smooth texture behind a slanted plane, disparity 4 + 30 x / W + 6 y / H,
 * with a flat patch of ties. lib.rs:472-508. */
void oracle_scene(int width, int height, uint64_t seed, uint8_t *left, uint8_t *right) {
    uint64_t state = oracle_random_seed(seed);
    int tw = width + 160;
    float *coarse = (float *)malloc(sizeof(float) * (size_t)tw * height);
    for (size_t i = 0; i < (size_t)tw * height; ++i)
        coarse[i] = (float)(uint8_t)(oracle_random_next(&state) >> 24);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            float disparity = 4.0f + 30.0f * (float)x / (float)width +
                              6.0f * (float)y / (float)height;
            int flat = x > width / 3 && x < width / 3 + 10 && y > height / 2 &&
                       y < height / 2 + 8;
            uint8_t values[2];
            for (int side = 0; side < 2; ++side) {
                float at = (float)x + 100.0f;
                if (side) at = at + disparity;
                float f0 = floorf(at);
                if (f0 < 0.0f) f0 = 0.0f;
                if (f0 > (float)tw - 2.0f) f0 = (float)tw - 2.0f;
                int x0 = (int)f0;
                float weight = at - (float)x0;
                float t = coarse[(size_t)y * tw + x0] * (1.0f - weight) +
                          coarse[(size_t)y * tw + x0 + 1] * weight;
                values[side] = (uint8_t)t;
            }
            left[(size_t)y * width + x] = flat ? 90 : values[0];
            right[(size_t)y * width + x] = flat ? 90 : values[1];
        }
    free(coarse);
}
