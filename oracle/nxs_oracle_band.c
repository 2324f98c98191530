/*
 * The CPU oracle for NxStereo's coarse-to-fine search: the 2x shrink, the
 * coarse matching's band bases, the band-limited matcher (sgm_band/4) and
 * the census windows its fine pass may use, restated step by step from
 * lib/nx_stereo.ex:138-471. TEST INFRASTRUCTURE ONLY (see nxs_oracle.h).
 *
 * Compiled with -ffp-contract=off, as nxs_oracle.c: every f32 operation is
 * rounded on its own, in the reference's order.
 */
#include "nxs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* The census of `window` (ORACLE_SPARSE_9X7, ORACLE_DENSE_9X5,
 * ORACLE_DENSE_9X5_BLEND): bit i for the i-th neighbour in row-major order,
 * set where the neighbour plus one is below the anchor, borders replicated.
 * The sparse window is dy -3..3, dx -4..4 with neither zero; the dense one
 * dy -2..2, dx -4..4 but the centre. The blended anchor is the centre's
 * rounded average with its 3x3 Gaussian mean: (sum of the 1-2-1 x 1-2-1
 * weighted neighbourhood + 16 x centre + 24) / 32.
 * lib/nx_stereo.ex:491-526 (census, neighbours, census_anchor). */
void oracle_census_window(const uint8_t *image, int width, int height, int window,
                          uint64_t *codes) {
    const int reach_y = window == ORACLE_SPARSE_9X7 ? 3 : 2;
    static const int weights[3] = {1, 2, 1};
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            int anchor = image[y * width + x];
            if (window == ORACLE_DENSE_9X5_BLEND) {
                int weighted = 0;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx)
                        weighted += image[clampi(y + dy, 0, height - 1) * width +
                                          clampi(x + dx, 0, width - 1)] *
                                    weights[dy + 1] * weights[dx + 1];
                anchor = (weighted + 16 * anchor + 24) / 32;
            }
            uint64_t code = 0;
            int bit = 0;
            for (int dy = -reach_y; dy <= reach_y; ++dy)
                for (int dx = -4; dx <= 4; ++dx) {
                    if (window == ORACLE_SPARSE_9X7 ? (dy == 0 || dx == 0) : (dy == 0 && dx == 0))
                        continue;
                    int n = image[clampi(y + dy, 0, height - 1) * width + clampi(x + dx, 0, width - 1)];
                    if (n + 1 < anchor) code |= (uint64_t)1 << bit;
                    ++bit;
                }
            codes[(size_t)y * width + x] = code;
        }
}

/* The rounded 2x2 average: (sum + 2) / 4. lib/nx_stereo.ex:227-238. */
void oracle_shrink(const uint8_t *image, int width, int height, uint8_t *half) {
    const int hw = width / 2, hh = height / 2;
    for (int y = 0; y < hh; ++y)
        for (int x = 0; x < hw; ++x) {
            int sum = image[(2 * y) * width + 2 * x] + image[(2 * y) * width + 2 * x + 1] +
                      image[(2 * y + 1) * width + 2 * x] + image[(2 * y + 1) * width + 2 * x + 1];
            half[y * hw + x] = (uint8_t)((sum + 2) / 4);
        }
}

/* Each full-resolution pixel's band base from the coarse disparity {ch, cw}:
 * margin below twice the lowest match (a value >= 0) in its coarse 3x3
 * neighbourhood, clipped to 0..128 - band, or -1 with no match there; each
 * coarse pixel's base covers its 2x2 block. lib/nx_stereo.ex:240-254. */
void oracle_band_base(const float *coarse, int coarse_width, int coarse_height, int band,
                      int margin, int32_t *base) {
    const float none = 1.0e9f;
    const int width = 2 * coarse_width;
    for (int y = 0; y < coarse_height; ++y)
        for (int x = 0; x < coarse_width; ++x) {
            float lowest = none;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int sy = y + dy, sx = x + dx;
                    float v = none;  /* the padding */
                    if (sy >= 0 && sy < coarse_height && sx >= 0 && sx < coarse_width) {
                        float c = coarse[sy * coarse_width + sx];
                        v = c >= 0.0f ? c : none;
                    }
                    if (v < lowest) lowest = v;
                }
            float start_f = floorf(lowest * 2.0f) - (float)margin;
            int start = clampi((int)start_f, 0, 128 - band);
            int value = lowest < none ? start : -1;
            for (int by = 0; by < 2; ++by)
                for (int bx = 0; bx < 2; ++bx) base[(2 * y + by) * width + 2 * x + bx] = value;
        }
}

/* costs[(y * width + x) * band + k] = popcount(left[y, x] ^ right[y, x -
 * searched[y, x] - k]), right codes left of the image being zero.
 * lib/nx_stereo.ex:362-383 (band_costs). */
void oracle_band_costs(const uint64_t *left, const uint64_t *right, const int32_t *searched,
                       int width, int height, int band, int32_t *costs) {
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            const int b = searched[y * width + x];
            for (int k = 0; k < band; ++k) {
                int column = x - b - k;
                uint64_t feature = column >= 0 ? right[y * width + column] : 0;
                costs[((size_t)y * width + x) * band + k] =
                    __builtin_popcountll(left[y * width + x] ^ feature);
            }
        }
}

/* One path of the band-limited recurrence: pixel (y, x) continues the path
 * from (y - dy, x - dx) (from zero, in its own band, where that is outside
 * the image). The previous pixel's normalised costs are moved to this
 * pixel's band by disparity: candidate k of this band is candidate
 * k + base - previous base of the previous one, p2 where that band lacks
 * it; then L[k] = min(min(own, p2), min(lower, upper) + p1) + C[k].
 * lib/nx_stereo.ex:385-454 (band_aggregate, scan_band, follow_base). */
void oracle_band_path(const int32_t *costs, const int32_t *searched, int width, int height,
                      int band, int dy, int dx, int p1, int p2, int32_t *path) {
    int32_t *a = (int32_t *)malloc(sizeof(int32_t) * band);
    int32_t *window = (int32_t *)malloc(sizeof(int32_t) * (band + 2));
    for (int r = 0; r < height; ++r) {
        int y = dy < 0 ? height - 1 - r : r;
        for (int c = 0; c < width; ++c) {
            int x = dx < 0 ? width - 1 - c : c;
            int py = y - dy, px = x - dx;
            int inside = py >= 0 && py < height && px >= 0 && px < width;
            const int current_base = searched[y * width + x];
            int previous_base = current_base;
            if (inside) {
                const int32_t *previous = path + ((size_t)py * width + px) * band;
                int32_t minimum = previous[0];
                for (int k = 1; k < band; ++k)
                    if (previous[k] < minimum) minimum = previous[k];
                for (int k = 0; k < band; ++k) a[k] = previous[k] - minimum;
                previous_base = searched[py * width + px];
            } else {
                for (int k = 0; k < band; ++k) a[k] = 0;
            }
            /* window[j] for j = 0..band + 1 is candidate j - 1 of this band */
            for (int j = 0; j < band + 2; ++j) {
                int index = j - 1 + current_base - previous_base;
                window[j] = index >= 0 && index < band ? a[index] : p2;
            }
            size_t at = ((size_t)y * width + x) * band;
            for (int k = 0; k < band; ++k) {
                int32_t own = window[k + 1], lower = window[k], upper = window[k + 2];
                int32_t jump = own < p2 ? own : p2;
                int32_t step = (lower < upper ? lower : upper) + p1;
                path[at + k] = (jump < step ? jump : step) + costs[at + k];
            }
        }
    }
    free(a);
    free(window);
}

/* The aggregation directions, as oracle_aggregate's: lib/nx_stereo.ex:385-416. */
static const int DIRECTIONS[8][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0},
                                     {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

void oracle_band_aggregate(const int32_t *costs, const int32_t *searched, int width, int height,
                           int band, int paths, int p1, int p2, int32_t *sums) {
    size_t volume = (size_t)width * height * band;
    int32_t *path = (int32_t *)malloc(sizeof(int32_t) * volume);
    memset(sums, 0, sizeof(int32_t) * volume);
    int count = paths == 8 ? 8 : 3;
    for (int p = 0; p < count; ++p) {
        oracle_band_path(costs, searched, width, height, band, DIRECTIONS[p][0],
                         DIRECTIONS[p][1], p1, p2, path);
        for (size_t i = 0; i < volume; ++i) sums[i] += path[i];
    }
    free(path);
}

/* select/3 within each pixel's band: values raised by 0x8000 where the
 * disparity base + k is past x; the winner k with ties low; the second best
 * outside k - 1..k + 1; the subpixel step from the band's neighbours of the
 * winner (clamped to the band). Accepted where the pixel has a base (>= 0),
 * its disparity base + k is at most x and the uniqueness test passes;
 * refined where the denominator is positive and the winner is inside the
 * band and below min(disparities - 1, x). The key is
 * (cost << 16) | (base + k). lib/nx_stereo.ex:429-469 (band_select). */
void oracle_band_select(const int32_t *sums, const int32_t *base, int width, int height, int band,
                        int disparities, float uniqueness, float *disparity, uint32_t *keys) {
    int32_t *values = (int32_t *)malloc(sizeof(int32_t) * band);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            const size_t pixel = (size_t)y * width + x;
            const int estimated = base[pixel] >= 0;
            const int b = base[pixel] > 0 ? base[pixel] : 0;
            for (int k = 0; k < band; ++k)
                values[k] = sums[pixel * band + k] + (b + k > x ? 0x8000 : 0);
            int winner = 0;
            int32_t minimum = values[0];
            for (int k = 1; k < band; ++k)
                if (values[k] < minimum) { minimum = values[k]; winner = k; }
            int32_t second = 0x7FFFFFFF;
            for (int k = 0; k < band; ++k)
                if (abs(k - winner) > 1 && values[k] < second) second = values[k];
            float lower = (float)values[winner - 1 < 0 ? 0 : winner - 1];
            float upper = (float)values[winner + 1 > band - 1 ? band - 1 : winner + 1];
            float minimum_f = (float)minimum;
            const int winner_d = b + winner;
            int accepted = estimated && winner_d <= x && (float)second > minimum_f * uniqueness;
            float denominator = lower + upper - 2.0f * minimum_f;
            float bounded = denominator > 1.0f ? denominator : 1.0f;
            float correction = (lower - upper) / (2.0f * bounded);
            if (correction < -0.5f) correction = -0.5f;
            if (correction > 0.5f) correction = 0.5f;
            int limit = disparities - 1 < x ? disparities - 1 : x;
            int refine = denominator > 0.0f && winner > 0 && winner < band - 1 && winner_d < limit;
            float value = (float)winner_d + (refine ? correction : 0.0f);
            disparity[pixel] = accepted ? value : -1.0f;
            keys[pixel] = accepted ? (((uint32_t)minimum << 16) | (uint32_t)winner_d)
                                   : ORACLE_INVALID_KEY;
        }
    free(values);
}

/* sgm_band/4's band_n: the census, the band's costs, its aggregation and
 * selection, the consistency check and the median.
 * lib/nx_stereo.ex:290-360. Returns 0, or -1 when the reference refuses the
 * sizes or settings (config!, lib/nx_stereo.ex:94-133, and sgm_band/4's
 * band check). */
int oracle_sgm_band(const uint8_t *left, const uint8_t *right, const int32_t *base, int width,
                    int height, int disparities, int paths, int band, int window, int p1, int p2,
                    float uniqueness, float *disparity) {
    if (!(width > 8 && height > 6 && width <= 4096) || disparities < 2 ||
        !(band == 8 || band == 16 || band == 32 || band == 64) || window < 0 || window > 2)
        return -1;
    const size_t pixels = (size_t)width * height, volume = pixels * band;
    uint64_t *lc = (uint64_t *)malloc(8 * pixels), *rc = (uint64_t *)malloc(8 * pixels);
    int32_t *searched = (int32_t *)malloc(4 * pixels);
    int32_t *costs = (int32_t *)malloc(4 * volume), *sums = (int32_t *)malloc(4 * volume);
    float *selected = (float *)malloc(4 * pixels), *checked = (float *)malloc(4 * pixels);
    uint32_t *keys = (uint32_t *)malloc(4 * pixels);
    for (size_t i = 0; i < pixels; ++i) searched[i] = base[i] > 0 ? base[i] : 0;
    oracle_census_window(left, width, height, window, lc);
    oracle_census_window(right, width, height, window, rc);
    oracle_band_costs(lc, rc, searched, width, height, band, costs);
    oracle_band_aggregate(costs, searched, width, height, band, paths, p1, p2, sums);
    oracle_band_select(sums, base, width, height, band, disparities, uniqueness, selected, keys);
    oracle_consistency(selected, keys, width, height, disparities, checked);
    oracle_median3(checked, width, height, disparity);
    free(lc); free(rc); free(searched); free(costs); free(sums); free(selected); free(checked);
    free(keys);
    return 0;
}

/* sgm_coarse_to_fine/3: sgm/3 on the pair shrunk 2x with 64 disparities and
 * `coarse_paths`, its band bases, then sgm_band/4 at full resolution over
 * 128 disparities with `fine_window`'s census. lib/nx_stereo.ex:138-225.
 * Returns 0, or -1 for an odd size or a size either pass refuses. */
int oracle_sgm_coarse_to_fine(const uint8_t *left, const uint8_t *right, int width, int height,
                              int paths, int coarse_paths, int band, int margin, int fine_window,
                              int p1, int p2, float uniqueness, float *disparity,
                              int32_t *base_out) {
    if (width % 2 != 0 || height % 2 != 0) return -1;
    const int hw = width / 2, hh = height / 2;
    uint8_t *lh = (uint8_t *)malloc((size_t)hw * hh), *rh = (uint8_t *)malloc((size_t)hw * hh);
    float *coarse = (float *)malloc(sizeof(float) * hw * hh);
    int32_t *base = (int32_t *)malloc(sizeof(int32_t) * width * height);
    oracle_shrink(left, width, height, lh);
    oracle_shrink(right, width, height, rh);
    int status = oracle_sgm(lh, rh, hw, hh, 64, coarse_paths, p1, p2, uniqueness, coarse);
    if (status == 0) {
        oracle_band_base(coarse, hw, hh, band, margin, base);
        if (base_out) memcpy(base_out, base, sizeof(int32_t) * width * height);
        status = oracle_sgm_band(left, right, base, width, height, 128, paths, band, fine_window,
                                 p1, p2, uniqueness, disparity);
    }
    free(lh); free(rh); free(coarse); free(base);
    return status;
}
