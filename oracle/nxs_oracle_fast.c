/*
 * The optimised CPU formulation of NxStereo's full-search matcher, after the
 * reference's Rust matcher (native/stereo_match/src/{lib,census,paths,
 * select,check}.rs). TEST INFRASTRUCTURE ONLY (see nxs_oracle.h): a
 * differential check of nxs_oracle.c and the CPU baseline bench.py times.
 *
 * Same arithmetic as the reference's: path costs are bytes (at most
 * p2 + 48 <= 127) held between two 255 sentinels that stand for libSGM's
 * p2 - p1 padding (paths.rs:1-8), so one step is
 *   next[d] = min(prev[d], prev_min + p2, sat(min(prev[d-1], prev[d+1]) + p1))
 *             - prev_min + cost[d]                               (paths.rs:190-217)
 * The work is arranged in one pass down the image and one up it:
 *   down: per row, census and costs (census.rs:18-84), the two horizontal
 *         paths (paths.rs:257-301), and a step of the three downward paths;
 *         totals[y, x, d] = horizontal + down paths (lib.rs:289-322);
 *   up:   the three upward paths added to the totals, then selection
 *         (lib.rs:323-349, select.rs:18-46);
 * then the left-right check and median per row (check.rs:12-85). The 3-path
 * mode is the horizontal pair plus the downward vertical path with selection
 * in the down pass (lib.rs:170-286).
 *
 * A pair runs on one thread; oracle_fast_sgm_batch spreads pairs over threads
 * (the reference spreads one pair's rows and column chunks instead,
 * parallel.rs; the arithmetic is the same).
 */
#include "nxs_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#define SENTINEL 255u

static inline uint8_t minu8(uint8_t a, uint8_t b) { return a < b ? a : b; }

/* One census row as a 48-bit code per pixel, borders replicated
 * (census.rs:14-48 keeps byte planes; the bits are the same). */
static void census_row(const uint8_t *image, int width, int height, int y, uint64_t *codes) {
    for (int x = 0; x < width; ++x) {
        int centre = image[(size_t)y * width + x];
        uint64_t code = 0;
        int bit = 0;
        for (int dy = -3; dy <= 3; ++dy) {
            if (!dy) continue;
            int sy = y + dy < 0 ? 0 : (y + dy >= height ? height - 1 : y + dy);
            const uint8_t *row = image + (size_t)sy * width;
            for (int dx = -4; dx <= 4; ++dx) {
                if (!dx) continue;
                int sx = x + dx < 0 ? 0 : (x + dx >= width ? width - 1 : x + dx);
                code |= (uint64_t)(centre - (int)row[sx] > 1) << bit;
                ++bit;
            }
        }
        codes[x] = code;
    }
}

static void reset_state(uint8_t *state, int D) {
    state[0] = SENTINEL;
    memset(state + 1, 0, (size_t)D);
    state[D + 1] = SENTINEL;
}

/* paths.rs:190-217: writes next[1..D], returns the new minimum. */
static uint8_t step(const uint8_t *prev, uint8_t prev_min, const uint8_t *costs, uint8_t *next,
                    int D, uint8_t p1, uint8_t p2) {
    uint8_t jump = (uint8_t)(prev_min + p2);
    uint8_t minimum = 255;
    for (int d = 0; d < D; ++d) {
        unsigned n = (unsigned)minu8(prev[d], prev[d + 2]) + p1;
        uint8_t neighbour = n > 255 ? 255 : (uint8_t)n;
        uint8_t value = (uint8_t)(minu8(minu8(prev[d + 1], jump), neighbour) - prev_min + costs[d]);
        next[d + 1] = value;
        if (value < minimum) minimum = value;
    }
    return minimum;
}

/* select.rs:18-46, the arithmetic of lib/nx_stereo.ex:610-641 on u16 sums. */
static void select_pixel(const uint16_t *sums, int D, int x, float uniqueness, float *disparity,
                         uint32_t *key_out) {
    uint16_t values[256];
    for (int d = 0; d < D; ++d) values[d] = (uint16_t)(sums[d] + (d > x ? 0x8000 : 0));
    uint16_t minimum = values[0];
    int winner = 0;
    for (int d = 1; d < D; ++d)
        if (values[d] < minimum) { minimum = values[d]; winner = d; }
    int below = winner > 0 ? winner - 1 : 0, above = winner + 1 < D ? winner + 1 : D - 1;
    uint16_t second = 0xFFFF;
    int any_other = 0;
    for (int d = 0; d < D; ++d)
        if (d < below || d > above) {
            any_other = 1;
            if (values[d] < second) second = values[d];
        }
    /* With no disparity outside the winner's neighbours the reference's
     * minimum is i32::MAX (reference.rs:166-170). */
    float second_f = any_other ? (float)second : 2147483647.0f;
    float lower = (float)values[below], upper = (float)values[above];
    float minimum_f = (float)minimum;
    int accepted = second_f > minimum_f * uniqueness;
    float denominator = lower + upper - 2.0f * minimum_f;
    float bounded = denominator > 1.0f ? denominator : 1.0f;
    float correction = (lower - upper) / (2.0f * bounded);
    if (correction < -0.5f) correction = -0.5f;
    if (correction > 0.5f) correction = 0.5f;
    int limit = D - 1 < x ? D - 1 : x;
    int refine = denominator > 0.0f && winner > 0 && winner < limit;
    float value = (float)winner + (refine ? correction : 0.0f);
    *disparity = accepted ? value : -1.0f;
    *key_out = accepted ? (((uint32_t)minimum << 16) | (uint32_t)winner) : ORACLE_INVALID_KEY;
}

typedef struct {
    int width, height, D;
    uint8_t *costs;     /* [H][W][D] */
    uint16_t *totals;   /* [H][W][D] */
    uint8_t *states;    /* 3 paths x 2 parities x (W + 2) slots x (D + 2) */
    uint8_t *minimums;  /* 3 x 2 x (W + 2) */
    uint8_t *hstate;    /* 4 x (D + 2) */
    uint8_t *backward;  /* [W][D] */
    uint64_t *lcodes, *rcodes;
    float *selected, *checked;
    uint32_t *keys, *right;
    uint16_t *sums;
} scratch_t;

static int scratch_init(scratch_t *s, int width, int height, int D) {
    memset(s, 0, sizeof(*s));
    s->width = width; s->height = height; s->D = D;
    size_t pixels = (size_t)width * height, volume = pixels * D, slots = (size_t)width + 2;
    s->costs = malloc(volume);
    s->totals = malloc(volume * 2);
    s->states = malloc(3 * 2 * slots * (D + 2));
    s->minimums = malloc(3 * 2 * slots);
    s->hstate = malloc(4 * (size_t)(D + 2));
    s->backward = malloc((size_t)width * D);
    s->lcodes = malloc(8 * (size_t)width);
    s->rcodes = malloc(8 * (size_t)width);
    s->selected = malloc(4 * pixels);
    s->checked = malloc(4 * pixels);
    s->keys = malloc(4 * pixels);
    s->right = malloc(4 * (size_t)width);
    s->sums = malloc(2 * (size_t)D);
    return s->costs && s->totals && s->states && s->minimums && s->hstate && s->backward &&
           s->lcodes && s->rcodes && s->selected && s->checked && s->keys && s->right && s->sums
               ? 0 : -1;
}

static void scratch_free(scratch_t *s) {
    free(s->costs); free(s->totals); free(s->states); free(s->minimums); free(s->hstate);
    free(s->backward); free(s->lcodes); free(s->rcodes); free(s->selected); free(s->checked);
    free(s->keys); free(s->right); free(s->sums);
}

/* Row y's costs and its horizontal pair's sum into `horizontal` (u16, added). */
static void costs_and_horizontal(scratch_t *s, const uint8_t *left, const uint8_t *right, int y,
                                 uint8_t p1, uint8_t p2, uint16_t *horizontal) {
    int W = s->width, D = s->D;
    census_row(left, W, s->height, y, s->lcodes);
    census_row(right, W, s->height, y, s->rcodes);
    uint8_t *costs = s->costs + (size_t)y * W * D;
    for (int x = 0; x < W; ++x)
        for (int d = 0; d < D; ++d) {
            uint64_t feature = x >= d ? s->rcodes[x - d] : 0;
            costs[(size_t)x * D + d] = (uint8_t)__builtin_popcountll(s->lcodes[x] ^ feature);
        }
    int stride = D + 2;
    uint8_t *fp = s->hstate, *fn = fp + stride, *bp = fn + stride, *bn = bp + stride;
    reset_state(fp, D); reset_state(fn, D); reset_state(bp, D); reset_state(bn, D);
    uint8_t fmin = 0, bmin = 0;
    for (int x = 0; x < W; ++x) {
        int bx = W - 1 - x;
        fmin = step(fp, fmin, costs + (size_t)x * D, fn, D, p1, p2);
        bmin = step(bp, bmin, costs + (size_t)bx * D, bn, D, p1, p2);
        for (int d = 0; d < D; ++d) horizontal[(size_t)x * D + d] = fn[d + 1];
        memcpy(s->backward + (size_t)bx * D, bn + 1, (size_t)D);
        uint8_t *t = fp; fp = fn; fn = t;
        t = bp; bp = bn; bn = t;
    }
    for (size_t i = 0; i < (size_t)W * D; ++i) horizontal[i] += s->backward[i];
}

/* One sweep row of the three paths with column offsets {0, +1, -1}: a path at
 * x continues the one at x - offset on the row before (paths.rs:310-395). */
static void sweep_row(scratch_t *s, int row, int y, uint8_t p1, uint8_t p2, int add_to_totals,
                      float uniqueness, int do_select) {
    static const int offsets[3] = {0, 1, -1};
    int W = s->width, D = s->D, stride = D + 2;
    size_t slots = (size_t)W + 2;
    int current = row % 2, previous = 1 - current;
    for (int x = 0; x < W; ++x) {
        const uint8_t *costs = s->costs + ((size_t)y * W + x) * D;
        uint16_t *totals = s->totals + ((size_t)y * W + x) * D;
        for (int p = 0; p < 3; ++p) {
            size_t source = (size_t)(p * 2 + previous) * slots + (size_t)(x + 1 - offsets[p]);
            size_t target = (size_t)(p * 2 + current) * slots + (size_t)(x + 1);
            uint8_t *next = s->states + target * stride;
            s->minimums[target] = step(s->states + source * stride, s->minimums[source], costs,
                                       next, D, p1, p2);
            if (add_to_totals)
                for (int d = 0; d < D; ++d) totals[d] = (uint16_t)(totals[d] + next[d + 1]);
        }
        if (do_select)
            select_pixel(totals, D, x, uniqueness, s->selected + (size_t)y * W + x,
                         s->keys + (size_t)y * W + x);
    }
}

static void reset_sweep(scratch_t *s) {
    int D = s->D;
    size_t slots = (size_t)s->width + 2;
    for (size_t i = 0; i < 6 * slots; ++i) reset_state(s->states + i * (D + 2), D);
    memset(s->minimums, 0, 6 * slots);
}

/* check.rs:12-47 */
static void consistency_row(const float *disparity, const uint32_t *keys, int W, uint32_t *right,
                            float *consistent) {
    for (int x = 0; x < W; ++x) right[x] = ORACLE_INVALID_KEY;
    for (int x = 0; x < W; ++x) {
        uint32_t key = keys[x];
        if (key == ORACLE_INVALID_KEY) continue;
        uint32_t winner = key & 0xFFFF;
        uint32_t candidate = (key & 0xFFFF0000u) | (65535u - winner);
        uint32_t *target = &right[x - (int)winner];
        if (candidate < *target) *target = candidate;
    }
    for (int x = 0; x < W; ++x) {
        float value = disparity[x];
        consistent[x] = -1.0f;
        if (value >= 0.0f) {
            long low = (long)value;
            long high = low + ((float)low != value);
            int rejected = 1;
            for (int k = 0; k < 2; ++k) {
                long d = k ? high : low, rx = x - d;
                int disagrees = 0;
                if (rx >= 0 && rx < W) {
                    uint32_t found = right[rx];
                    long rd = 65535 - (long)(found & 0xFFFF);
                    disagrees = found != ORACLE_INVALID_KEY && labs(rd - d) > 1;
                }
                rejected = rejected && disagrees;
            }
            if (!rejected) consistent[x] = value;
        }
    }
}

/* Devillard's 9-element median network (filters.rs:219-242): the median ends
 * in the middle slot. Values are -1 or non-negative, so f32 order is used. */
static const int MEDIAN_9[19][2] = {{1, 2}, {4, 5}, {7, 8}, {0, 1}, {3, 4}, {6, 7}, {1, 2},
                                    {4, 5}, {7, 8}, {0, 3}, {5, 8}, {4, 7}, {3, 6}, {1, 4},
                                    {2, 5}, {4, 7}, {4, 2}, {6, 4}, {4, 2}};

static void median_image(const float *image, int W, int H, float *filtered) {
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float v[9];
            int n = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int sy = y + dy < 0 ? 0 : (y + dy >= H ? H - 1 : y + dy);
                    int sx = x + dx < 0 ? 0 : (x + dx >= W ? W - 1 : x + dx);
                    v[n++] = image[(size_t)sy * W + sx];
                }
            for (int i = 0; i < 19; ++i) {
                int a = MEDIAN_9[i][0], b = MEDIAN_9[i][1];
                float lo = v[a] < v[b] ? v[a] : v[b], hi = v[a] < v[b] ? v[b] : v[a];
                v[a] = lo;
                v[b] = hi;
            }
            filtered[(size_t)y * W + x] = v[4];
        }
}

static int run_pair(scratch_t *s, const uint8_t *left, const uint8_t *right, int paths, int p1,
                    int p2, float uniqueness, float *disparity) {
    int W = s->width, H = s->height, D = s->D;
    reset_sweep(s);
    /* Down: costs, horizontal pair, downward paths (all three, or only the
     * vertical one with selection for 3 paths). */
    for (int y = 0; y < H; ++y) {
        uint16_t *totals = s->totals + (size_t)y * W * D;
        memset(totals, 0, (size_t)W * D * 2);
        costs_and_horizontal(s, left, right, y, (uint8_t)p1, (uint8_t)p2, totals);
        if (paths == 8) {
            sweep_row(s, y, y, (uint8_t)p1, (uint8_t)p2, 1, uniqueness, 0);
        } else {
            /* Only the vertical path: slot 0 of sweep_row's three. */
            int stride = D + 2, current = y % 2, previous = 1 - current;
            size_t slots = (size_t)W + 2;
            for (int x = 0; x < W; ++x) {
                size_t source = (size_t)previous * slots + x + 1, target = (size_t)current * slots + x + 1;
                uint8_t *next = s->states + target * stride;
                s->minimums[target] = step(s->states + source * stride, s->minimums[source],
                                           s->costs + ((size_t)y * W + x) * D, next, D,
                                           (uint8_t)p1, (uint8_t)p2);
                uint16_t *t = totals + (size_t)x * D;
                for (int d = 0; d < D; ++d) t[d] = (uint16_t)(t[d] + next[d + 1]);
                select_pixel(t, D, x, uniqueness, s->selected + (size_t)y * W + x,
                             s->keys + (size_t)y * W + x);
            }
        }
    }
    if (paths == 8) {
        reset_sweep(s);
        for (int row = 0; row < H; ++row)
            sweep_row(s, row, H - 1 - row, (uint8_t)p1, (uint8_t)p2, 1, uniqueness, 1);
    }
    for (int y = 0; y < H; ++y)
        consistency_row(s->selected + (size_t)y * W, s->keys + (size_t)y * W, W, s->right,
                        s->checked + (size_t)y * W);
    median_image(s->checked, W, H, disparity);
    return 0;
}

static int refused(int width, int height, int disparities, int paths, int p1, int p2) {
    return !(width > 8 && height > 6 && width <= 4096) || disparities < 4 || disparities > 256 ||
           (paths != 3 && paths != 8) || !(p1 >= 0 && p1 < p2 && p2 + 48 <= 127);
}

int oracle_fast_sgm(const uint8_t *left, const uint8_t *right, int width, int height,
                    int disparities, int paths, int p1, int p2, float uniqueness,
                    float *disparity) {
    if (refused(width, height, disparities, paths, p1, p2)) return -1;
    scratch_t s;
    int status = scratch_init(&s, width, height, disparities);
    if (!status)
        status = run_pair(&s, left, right, paths, p1, p2, uniqueness, disparity);
    scratch_free(&s);
    return status;
}

typedef struct {
    const uint8_t *lefts, *rights;
    float *outputs;
    int pairs, width, height, D, paths, p1, p2;
    float uniqueness;
    atomic_int next;
    atomic_int failed;
} batch_t;

static void *batch_worker(void *arg) {
    batch_t *b = (batch_t *)arg;
    scratch_t s;
    if (scratch_init(&s, b->width, b->height, b->D)) {
        atomic_store(&b->failed, 1);
        scratch_free(&s);
        return NULL;
    }
    size_t pixels = (size_t)b->width * b->height;
    for (;;) {
        int i = atomic_fetch_add(&b->next, 1);
        if (i >= b->pairs) break;
        run_pair(&s, b->lefts + i * pixels, b->rights + i * pixels, b->paths, b->p1, b->p2,
                 b->uniqueness, b->outputs + i * pixels);
    }
    scratch_free(&s);
    return NULL;
}

int oracle_fast_sgm_batch(const uint8_t *lefts, const uint8_t *rights, int pairs, int width,
                          int height, int disparities, int paths, int p1, int p2,
                          float uniqueness, float *disparities_out, int threads) {
    if (refused(width, height, disparities, paths, p1, p2) || pairs < 0) return -1;
    if (threads < 1) threads = 1;
    if (threads > pairs) threads = pairs > 0 ? pairs : 1;
    batch_t b = {lefts, rights, disparities_out, pairs, width, height, disparities, paths, p1, p2,
                 uniqueness};
    atomic_init(&b.next, 0);
    atomic_init(&b.failed, 0);
    pthread_t *ids = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    for (int t = 0; t < threads; ++t) pthread_create(&ids[t], NULL, batch_worker, &b);
    for (int t = 0; t < threads; ++t) pthread_join(ids[t], NULL);
    free(ids);
    return atomic_load(&b.failed) ? -1 : 0;
}

typedef struct {
    const uint8_t *lefts, *rights;
    int pairs, fw, fh, width, height, D, paths, p1, p2, decimation;
    const oracle_camera *cameras[2];
    float uniqueness, min_support, max_diff, focal, baseline, cx, cy, nearest, farthest;
    float *outputs;
    atomic_int next;
    atomic_long kept;
    atomic_int failed;
} pipeline_t;

static void *pipeline_worker(void *arg) {
    pipeline_t *b = (pipeline_t *)arg;
    scratch_t s;
    size_t pixels = (size_t)b->width * b->height, frame = (size_t)b->fw * b->fh;
    uint8_t *images = malloc(2 * pixels);
    float *disparity = malloc(4 * pixels), *speckled = malloc(4 * pixels);
    float *depth_m = malloc(4 * pixels);
    uint16_t *depth_mm = malloc(2 * pixels);
    int gw = b->width / b->decimation, gh = b->height / b->decimation;
    float *grid = malloc(sizeof(float) * 3 * ((size_t)gw * gh + 1));
    if (scratch_init(&s, b->width, b->height, b->D) || !images || !disparity || !speckled ||
        !depth_m || !depth_mm || !grid) {
        atomic_store(&b->failed, 1);
    } else {
        for (;;) {
            int i = atomic_fetch_add(&b->next, 1);
            if (i >= b->pairs) break;
            oracle_rectify(b->lefts + i * frame, b->fw, b->fh, b->cameras[0], b->width,
                           b->height, images);
            oracle_rectify(b->rights + i * frame, b->fw, b->fh, b->cameras[1], b->width,
                           b->height, images + pixels);
            run_pair(&s, images, images + pixels, b->paths, b->p1, b->p2, b->uniqueness,
                     disparity);
            for (size_t k = 0; k < pixels; ++k)
                if (!(disparity[k] > 0.0f)) disparity[k] = -1.0f;
            oracle_despeckle(disparity, b->width, b->height, b->min_support, b->max_diff, 3,
                             speckled);
            oracle_depth(speckled, pixels, b->focal, b->baseline, depth_mm, depth_m);
            long kept = oracle_cloud(depth_m, b->width, b->height, b->decimation, b->focal,
                                     b->cx, b->cy, b->nearest, b->farthest, grid);
            atomic_fetch_add(&b->kept, kept);
            if (b->outputs) memcpy(b->outputs + i * pixels, speckled, 4 * pixels);
        }
    }
    scratch_free(&s);
    free(images); free(disparity); free(speckled); free(depth_m); free(depth_mm); free(grid);
    return NULL;
}

long oracle_fast_pipeline_batch(const uint8_t *left_frames, const uint8_t *right_frames,
                                int pairs, int frame_width, int frame_height,
                                const oracle_camera *left_camera,
                                const oracle_camera *right_camera, int width, int height,
                                int disparities, int paths, int p1, int p2, float uniqueness,
                                float min_support, float max_diff, float focal_length_px,
                                float baseline_m, int decimation, float cx, float cy,
                                float nearest_m, float farthest_m, float *disparities_out,
                                int threads) {
    if (refused(width, height, disparities, paths, p1, p2) || pairs < 0 || decimation < 1)
        return -1;
    if (threads < 1) threads = 1;
    if (threads > pairs) threads = pairs > 0 ? pairs : 1;
    pipeline_t b;
    memset(&b, 0, sizeof b);
    b.lefts = left_frames; b.rights = right_frames; b.pairs = pairs;
    b.fw = frame_width; b.fh = frame_height; b.width = width; b.height = height;
    b.D = disparities; b.paths = paths; b.p1 = p1; b.p2 = p2; b.decimation = decimation;
    b.cameras[0] = left_camera; b.cameras[1] = right_camera;
    b.uniqueness = uniqueness; b.min_support = min_support; b.max_diff = max_diff;
    b.focal = focal_length_px; b.baseline = baseline_m; b.cx = cx; b.cy = cy;
    b.nearest = nearest_m; b.farthest = farthest_m; b.outputs = disparities_out;
    atomic_init(&b.next, 0);
    atomic_init(&b.kept, 0);
    atomic_init(&b.failed, 0);
    pthread_t *ids = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    for (int t = 0; t < threads; ++t) pthread_create(&ids[t], NULL, pipeline_worker, &b);
    for (int t = 0; t < threads; ++t) pthread_join(ids[t], NULL);
    free(ids);
    return atomic_load(&b.failed) ? -1 : atomic_load(&b.kept);
}
