// Batched SGM: many rectified pairs of uneven size and disparity range in one
// persistent launch, captured in a CUDA graph.
//
// The matcher of NxStereo.sgm/3 (lib/nx_stereo.ex:64-74, 475-683) runs as six
// phases per pair: census, costs, path aggregation, selection (which also
// builds the right image's map for the left-right check), the check, and the
// median with Stage.Disparity's mask (lib/nx_stereo/stage/disparity.ex:162).
// The costs and path volumes are in the permuted order of the path lanes'
// span (span_disparity in nxs_matcher.cuh), as the single-pair matcher keeps
// them.
// Each phase is cut into items a block of 128 threads does: a census tile, a
// few rows of costs, four warps of scan lines, a run of pixels to select, a
// run of pixels to check or filter. Blocks stay resident for the whole launch
// and take the next item of one queue from an atomic counter.
//
// The host lays the queue out as a pipeline over groups of pairs (see
// build_runs): a group's path aggregation (integer-pipe bound) is interleaved
// with the previous group's selection (HBM bound), and the next group's
// census and costs (popcount bound) with the check and median of the group
// before, so different kinds of work share the SMs instead of one phase
// following another; each group's path items are ordered longest first over
// all its pairs so that its last items are short.
//
// An item of phase k of a pair waits, before it starts, until every item of
// phase k - 1 of that pair is done. Items are taken in queue order and an
// item only waits on items earlier in the queue, all taken by running blocks,
// so the earliest unfinished item always runs and the queue cannot deadlock.
// The wait still has a time limit (the plan's, 2 s by default), after which the block
// records a timeout in the status word and goes on, so a launch always ends.
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/nx_stereo_b200.h"
#include "nxs_kernels.h"
#include "nxs_matcher.cuh"

namespace nxs {
namespace {

enum Phase { kCensus = 0, kCosts, kPaths, kSelect, kCheck, kMedian, kPhases };

constexpr int kThreads = 128;
constexpr int kCensusRows = 4;         // census tile: 128 x 4 pixels (census4_tile)
constexpr int kPixelsPerItem = 1024;   // check and median items
// Control words: queue head, status, 2 unused, then 16 u64 cycle sums (each
// phase's
// items, each phase's waits for the phase before, taking items, 3 unused),
// then done[pair][phase].
constexpr int kClocks = 16;
constexpr int kControlWords = 4 + 2 * kClocks;
constexpr int kClockWait = kPhases, kClockTake = 2 * kPhases;
// The default limit of one wait (nxs_batch_tuning.wait_limit_us 0).
constexpr uint64_t kWaitLimitNs = 2000000000ull;

struct BatchPair {
    const uint8_t *left, *right;
    uint64_t *left_codes, *right_codes;
    uint8_t *costs, *paths;
    float *raw;           // selection's disparity
    uint32_t *right_map;  // per right pixel: min of (cost << 16 | 65535 - d)
    float *checked;
    float *disparity;     // the pair's output
    float uniqueness;
    int stage_mask;
    int select_lanes;     // lanes per pixel in selection
    int path_lanes;       // lanes per scan line
    int path_words;       // u16x2 words a path lane holds (4 or 8); the order's span is twice
    int census_columns;   // census tiles per row band
    int census_tiles;     // census tiles per image
    int cost_columns;     // 64-pixel blocks per row
    int cost_rows;        // rows per costs item
    int select_passes;    // 128 / select_lanes pixels per pass
    int items[kPhases];
    PathSetup setup;
};

__device__ __forceinline__ unsigned load_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The permuted order's span: 8 with 4 words a lane, 16 otherwise.
template <int WORDS>
constexpr int kSpan = WORDS == 4 ? 8 : 16;

template <int G, int WORDS>
__device__ __forceinline__ void paths_item(const BatchPair &P, const PathSetup &s, int warp,
                                           int lane, uint8_t *ring) {
    if (P.setup.disparities == G * 2 * WORDS)
        path_warp<G, WORDS, true, kSpan<WORDS>>(P.costs, P.paths, s, warp, lane, ring);
    else
        path_warp<G, WORDS, false, kSpan<WORDS>>(P.costs, P.paths, s, warp, lane, ring);
}

template <int G, int PATHS, int SPAN>
__device__ __forceinline__ void select_item(const BatchPair &P, int item, uint8_t *smem) {
    constexpr int PIXELS = 128 / G;
    const int W = P.setup.width, H = P.setup.height;
    const size_t pixels = (size_t)W * H;
    for (int pass = 0; pass < P.select_passes; ++pass) {
        const size_t block = (size_t)item * P.select_passes + pass;
        if (block * PIXELS >= pixels) break;  // the same for the whole block
        select_pixels<G, PATHS, SPAN>(P.paths, W, H, P.setup.disparities, P.setup.volume,
                                P.uniqueness, P.raw, nullptr, P.right_map, block,
                                reinterpret_cast<uint16_t(*)[256]>(smem), P.setup.one);
        __syncwarp();
    }
}

template <int PATHS, int SPAN>
__device__ __forceinline__ void select_lanes(const BatchPair &P, int item, uint8_t *smem) {
    if (P.select_lanes == 4) select_item<4, PATHS, SPAN>(P, item, smem);
    else if (P.select_lanes == 8) select_item<8, PATHS, SPAN>(P, item, smem);
    else select_item<16, PATHS, SPAN>(P, item, smem);
}

template <int PATHS>
__device__ __forceinline__ void select_dispatch(const BatchPair &P, int item, uint8_t *smem) {
    if (P.path_words == 4) select_lanes<PATHS, 8>(P, item, smem);
    else select_lanes<PATHS, 16>(P, item, smem);
}

// Waits (thread 0, or lane 0 of a warp) until `*counter` reaches `need`; gives
// up after `limit_ns` and records it in the status word. After one wait has
// run out none waits again, so the launch ends instead of waiting out every
// item.
__device__ __forceinline__ void wait_for(const unsigned *counter, unsigned need,
                                         unsigned *control, uint64_t limit_ns) {
    if (load_acquire(counter) >= need || load_acquire(control + 1)) return;
    const uint64_t start = global_ns();
    while (load_acquire(counter) < need) {
        __nanosleep(256);
        if (global_ns() - start > limit_ns) {
            atomicOr(control + 1, 1u);
            return;
        }
    }
}

// A block takes items from the queue in order; an item of phase k waits for
// every item of phase k - 1 of its pair.
// queue[q] = (pair << 4 | phase, item) of queue position q. WIDE: with the
// path kernels of 16 words a lane (more registers a thread).
template <bool WIDE>
__device__ __forceinline__ void work(const BatchPair *__restrict__ pairs,
                                     const uint2 *__restrict__ queue, unsigned total,
                                     unsigned *control, uint8_t *smem, PathSetup &setup,
                                     unsigned long long *clocks, uint64_t limit_ns) {
    __shared__ unsigned taken_pair, taken_phase, taken_item, taken_more;
    const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
    unsigned *const done = control + kControlWords;
    unsigned next = 0;
    uint64_t started = 0;
    if (tid == 0) next = atomicAdd(control, 1u);
    for (;;) {
        if (tid == 0) {
            const uint64_t taking = clock64();
            const unsigned q = next;
            taken_more = q < total;
            if (q < total) {
                next = atomicAdd(control, 1u);  // the next item's claim overlaps this one
                const uint2 entry = __ldg(queue + q);
                const unsigned pair = entry.x >> 4, phase = entry.x & 15u;
                taken_pair = pair;
                taken_phase = phase;
                taken_item = entry.y;
                const uint64_t waiting = clock64();
                clocks[kClockTake] += waiting - taking;
                if (phase > 0)
                    wait_for(done + pair * kPhases + phase - 1,
                             (unsigned)pairs[pair].items[phase - 1], control, limit_ns);
                started = clock64();
                clocks[kClockWait + phase] += started - waiting;
            }
        }
        __syncthreads();
        if (!taken_more) break;
        const int pair = (int)taken_pair, phase = (int)taken_phase, item = (int)taken_item;
        const BatchPair &P = pairs[pair];
        const int W = P.setup.width, H = P.setup.height;
        switch (phase) {
        case kCensus: {
            const int image = item / P.census_tiles, tile = item % P.census_tiles;
            const int x0 = (tile % P.census_columns) * kCensus4X;
            const int y0 = (tile / P.census_columns) * kCensusRows;
            census4_tile<kCensusRows, kThreads>(image ? P.right : P.left, W, H,
                                                image ? P.right_codes : P.left_codes, x0, y0,
                                                tid, smem);
            if (image == 0) {  // the right map of these pixels starts empty
                for (int i = tid; i < kCensus4X * kCensusRows; i += kThreads) {
                    const int x = x0 + i % kCensus4X, y = y0 + i / kCensus4X;
                    if (x < W && y < H) P.right_map[(size_t)y * W + x] = kInvalidKey;
                }
            }
            break;
        }
        case kCosts: {
            const int x0 = (item % P.cost_columns) * kCostPixels;
            const int y0 = (item / P.cost_columns) * P.cost_rows;
            for (int r = 0; r < P.cost_rows; ++r) {
                if (y0 + r >= H) break;  // the same for the whole block
                if (r) __syncthreads();  // the last row's tile is read out
                if (P.path_words == 4)
                    costs_tile<8>(P.left_codes, P.right_codes, W, P.setup.disparities, P.costs,
                                  x0, y0 + r, smem);
                else
                    costs_tile<16>(P.left_codes, P.right_codes, W, P.setup.disparities, P.costs,
                                   x0, y0 + r, smem);
            }
            break;
        }
        case kPaths: {  // four warps of scan lines
            if (tid < (int)(sizeof(PathSetup) / 4))
                reinterpret_cast<int *>(&setup)[tid] = reinterpret_cast<const int *>(&P.setup)[tid];
            __syncthreads();
            const int index = item * (kThreads / 32) + warp;
            // A warp's ring: kPrefetch x 32 lanes x 2 x words bytes, in pieces of
            // at most 16 bytes strided by 32 lanes; a lane starts at its piece.
            const int bytes = 2 * P.path_words, piece = bytes < 16 ? bytes : 16;
            uint8_t *ring = smem + warp * kPrefetch * 32 * bytes + lane * piece;
            if (index < setup.first_warp[8]) {
                if (WIDE && P.path_words == 16) {
                    if (P.path_lanes == 2) paths_item<2, 16>(P, setup, index, lane, ring);
                    else if (P.path_lanes == 4) paths_item<4, 16>(P, setup, index, lane, ring);
                    else paths_item<8, 16>(P, setup, index, lane, ring);
                } else if (P.path_words == 8) {
                    if (P.path_lanes == 4) paths_item<4, 8>(P, setup, index, lane, ring);
                    else if (P.path_lanes == 8) paths_item<8, 8>(P, setup, index, lane, ring);
                    else paths_item<16, 8>(P, setup, index, lane, ring);
                } else {
                    if (P.path_lanes == 8) paths_item<8, 4>(P, setup, index, lane, ring);
                    else if (P.path_lanes == 16) paths_item<16, 4>(P, setup, index, lane, ring);
                    else paths_item<32, 4>(P, setup, index, lane, ring);
                }
            }
            break;
        }
        case kSelect:
            if (P.setup.paths == 8) select_dispatch<8>(P, item, smem);
            else select_dispatch<3>(P, item, smem);
            break;
        case kCheck: {
            const size_t base = (size_t)item * kPixelsPerItem, pixels = (size_t)W * H;
            for (int i = tid; i < kPixelsPerItem; i += kThreads) {
                const size_t pixel = base + i;
                if (pixel >= pixels) break;
                const int y = (int)(pixel / W), x = (int)(pixel % W);
                P.checked[pixel] = consistent_value<true>(__ldcg(P.raw + pixel), x, W,
                                                          P.right_map + (size_t)y * W);
            }
            break;
        }
        default: {  // kMedian
            const size_t base = (size_t)item * kPixelsPerItem, pixels = (size_t)W * H;
            for (int i = tid; i < kPixelsPerItem; i += kThreads) {
                const size_t pixel = base + i;
                if (pixel >= pixels) break;
                median_at(P.checked, W, H, P.stage_mask, P.disparity, (int)(pixel % W),
                          (int)(pixel / W));
            }
            break;
        }
        }
        __syncthreads();  // every thread's writes, before the item counts as done
        if (tid == 0) {
            __threadfence();
            atomicAdd(done + pair * kPhases + phase, 1u);
            clocks[phase] += clock64() - started;
        }
    }
}

template <bool WIDE>
__global__ void __launch_bounds__(kThreads, WIDE ? 6 : 8)
    batch_kernel(const BatchPair *__restrict__ pairs, const uint2 *__restrict__ queue,
                 unsigned total, unsigned *control, uint64_t limit_ns) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ PathSetup setup;
    __shared__ unsigned long long clocks[kClocks];  // this block's cycle sums (thread 0)
    if (threadIdx.x < kClocks) clocks[threadIdx.x] = 0;
    __syncthreads();
    work<WIDE>(pairs, queue, total, control, smem, setup, clocks, limit_ns);
    __syncthreads();
    if (threadIdx.x < kClocks)
        atomicAdd(reinterpret_cast<unsigned long long *>(control + 4) + threadIdx.x,
                  clocks[threadIdx.x]);
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

void set_error(char *error, size_t error_len, const char *format, ...) {
    if (!error || error_len == 0) return;
    va_list args;
    va_start(args, format);
    vsnprintf(error, error_len, format, args);
    va_end(args);
}

uint64_t wait_limit_ns(const nxs_batch_tuning &t) {
    return t.wait_limit_us ? (uint64_t)t.wait_limit_us * 1000ull : kWaitLimitNs;
}

nxs_status cuda_failed(cudaError_t e, char *error, size_t error_len, const char *what) {
    if (e == cudaSuccess) return NXS_OK;
    set_error(error, error_len, "%s: %s", what, cudaGetErrorString(e));
    return NXS_CUDA_ERROR;
}

// Whole-GPU microseconds of each phase of a 728x544 pair at 128 disparities
// and 8 paths, as the single-pair kernels take them: the weights that
// interleave the queue.
constexpr double kPhaseMicros[kPhases] = {18.0, 38.0, 162.0, 66.0, 7.0, 5.0};
constexpr double kReferencePixels = 728.0 * 544.0, kReferenceDisparities = 128.0;

double phase_micros(const nxs_batch_pair &p, int phase) {
    const double px = (double)p.width * p.height / kReferencePixels;
    const double pd = px * p.params.disparities / kReferenceDisparities;
    const double paths = p.params.paths / 8.0;
    switch (phase) {
    case kCensus: return kPhaseMicros[kCensus] * px;
    case kCosts: return kPhaseMicros[kCosts] * pd;
    case kPaths: return kPhaseMicros[kPaths] * pd * paths;
    case kSelect: return kPhaseMicros[kSelect] * pd * (0.25 + 0.75 * paths);
    default: return kPhaseMicros[phase] * px;
    }
}

}  // namespace
}  // namespace nxs

using namespace nxs;

struct nxs_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    nxs_batch_tuning tuning{};
    std::vector<nxs_batch_pair> specs;
    std::vector<BatchPair> pairs;
    std::vector<size_t> input_offsets, output_offsets;  // left of pair i; its disparity
    unsigned total = 0;  // items in the queue
    int runs = 0;
    int grid = 0;
    bool wide = false;  // some pair's path lanes hold 16 words
    size_t shared_bytes = 0;
    size_t arena_bytes = 0, input_bytes = 0, output_bytes = 0, control_bytes = 0;
    uint8_t *arena = nullptr;    // inputs | control + outputs | everything else
    uint8_t *staging = nullptr;  // pinned mirror of the inputs and of control + outputs
    BatchPair *d_pairs = nullptr;
    uint2 *d_queue = nullptr;  // (pair << 4 | phase, item) of every queue position
    unsigned *d_control = nullptr;
    cudaGraphExec_t graph = nullptr;      // control reset + kernel
    cudaGraphExec_t graph_host = nullptr; // inputs in, reset, kernel, outputs out
    // The streams engine: side streams the pairs' kernel chains fork onto.
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork = nullptr;
    std::mutex lock;
};

namespace {

// A pair's shapes and item counts (no buffers).
void shape_pair(const nxs_batch_pair &s, const nxs_batch_tuning &t, BatchPair *out) {
    BatchPair &P = *out;
    const int W = (int)s.width, H = (int)s.height, D = (int)s.params.disparities;
    const size_t px = (size_t)W * H;
    P.uniqueness = s.params.uniqueness;
    P.stage_mask = s.params.stage_mask ? 1 : 0;
    P.select_lanes = group_lanes(D);
    P.path_words = t.path_words ? t.path_words : path_words(D);
    P.path_lanes = path_lanes(D, P.path_words);
    P.census_columns = (W + kCensus4X - 1) / kCensus4X;
    P.census_tiles = P.census_columns * ((H + kCensusRows - 1) / kCensusRows);
    P.cost_columns = (W + kCostPixels - 1) / kCostPixels;
    P.cost_rows = t.cost_rows;
    P.select_passes = t.select_passes;
    const int warps = path_setup(W, H, D, (int)s.params.paths, (int)s.params.p1,
                                 (int)s.params.p2, P.path_lanes, &P.setup);
    // The path volumes lie 256-aligned apart rather than packed.
    P.setup.volume = align256(px * D);
    P.items[kCensus] = 2 * P.census_tiles;
    P.items[kCosts] = P.cost_columns * ((H + t.cost_rows - 1) / t.cost_rows);
    P.items[kPaths] = (warps + kThreads / 32 - 1) / (kThreads / 32);  // four warps an item
    const size_t per_item = (size_t)(128 / P.select_lanes) * t.select_passes;
    P.items[kSelect] = (int)((px + per_item - 1) / per_item);
    P.items[kCheck] = (int)((px + kPixelsPerItem - 1) / kPixelsPerItem);
    P.items[kMedian] = P.items[kCheck];
}

// A stretch of one phase of one pair in the queue, and its estimated
// whole-GPU time.
struct Chunk {
    int pair, phase, first, count;
    double micros;
};
using Stream = std::vector<Chunk>;

// The steps of the longest scan line of each four-warp path item of a pair.
std::vector<int> path_item_steps(const BatchPair &P) {
    const PathSetup &s = P.setup;
    const int lines_per_warp = 32 / P.path_lanes, warps = s.first_warp[8];
    std::vector<int> steps(P.items[kPaths], 0);
    for (int warp = 0; warp < warps; ++warp) {
        int slot = 0;
        while (warp >= s.first_warp[slot + 1]) ++slot;
        int p, group;
        if (slot < s.straight) {
            p = s.order[slot];
            group = warp - s.first_warp[slot];
        } else {
            const int w = warp - s.first_warp[s.straight];
            p = s.order[s.straight + w % (s.paths - s.straight)];
            group = w / (s.paths - s.straight);
        }
        // ranks are in decreasing length, so the group's first line is its longest
        const int rank = group * lines_per_warp;
        if (rank >= s.lines[p]) continue;
        int y0, x0;
        const int line = ranked_line(rank, s.dy[p], s.dx[p], s.width, s.height);
        const int length = line_start(line, s.dy[p], s.dx[p], s.width, s.height, &y0, &x0);
        int &item = steps[warp / (kThreads / 32)];
        item = std::max(item, length);
    }
    return steps;
}

// Interleaves streams so that each advances in proportion to its estimated
// time: the stream least far along goes next, a run of about `quantum`
// microseconds at a time.
template <typename Emit>
void merge(std::vector<Stream> streams, double quantum, Emit emit) {
    std::vector<double> total(streams.size(), 0.0), done(streams.size(), 0.0);
    std::vector<size_t> at(streams.size(), 0);
    for (size_t i = 0; i < streams.size(); ++i)
        for (const Chunk &c : streams[i]) total[i] += c.micros;
    for (;;) {
        int next = -1;
        double least = 2.0;
        for (size_t i = 0; i < streams.size(); ++i) {
            if (at[i] >= streams[i].size()) continue;
            const double along = total[i] > 0 ? done[i] / total[i] : 0.0;
            if (along < least) {
                least = along;
                next = (int)i;
            }
        }
        if (next < 0) return;
        Chunk &c = streams[next][at[next]];
        const double per_item = c.micros / std::max(c.count, 1);
        int count = (int)std::lround(quantum / std::max(per_item, 1e-9));
        count = std::max(1, std::min(count, c.count));
        emit(c.pair, c.phase, c.first, count);
        c.first += count;
        c.count -= count;
        c.micros -= per_item * count;
        done[next] += per_item * count;
        if (c.count == 0) ++at[next];
    }
}

// The queue. Pairs go in groups of `group_pairs`; with G0, G1, ... the
// groups, the queue alternates two kinds of segment, for i = -2, -1, 0, ...:
//   A(i): census of G(i+2), costs of G(i+1), check of G(i-2), median of G(i-3);
//   B(i): paths of G(i+1) beside the selection of G(i-1),
// the phases of a segment interleaved in proportion to their estimated time.
// Every phase but the paths thus comes at least a whole segment after the
// phase it needs, so its items rarely wait; a group's costs are written just
// before its path items read them (still in L2 for small groups); and the
// path aggregation (integer-pipe bound) runs beside selection (HBM bound).
// Each group's path items are ordered longest first over all its pairs, so a
// group's paths end with short lines. order 1 lays every phase out over all
// pairs in turn instead.
void build_runs(const std::vector<nxs_batch_pair> &specs, const std::vector<BatchPair> &pairs,
                const nxs_batch_tuning &tuning, std::vector<unsigned> &start,
                std::vector<unsigned> &info, std::vector<unsigned> &first) {
    const int n = (int)specs.size();
    const double quantum = tuning.quantum_us > 0 ? tuning.quantum_us : 2.0;
    unsigned position = 0;
    auto emit = [&](int pair, int phase, int item0, int count) {
        const unsigned code = ((unsigned)pair << 4) | (unsigned)phase;
        if (!info.empty() && info.back() == code &&
            first.back() + (position - start.back()) == (unsigned)item0) {
            position += count;  // continues the last run
            return;
        }
        start.push_back(position);
        info.push_back(code);
        first.push_back((unsigned)item0);
        position += count;
    };
    auto whole = [&](int pair, int phase) {
        return Chunk{pair, phase, 0, pairs[pair].items[phase], phase_micros(specs[pair], phase)};
    };
    if (tuning.order == 1) {
        for (int phase = 0; phase < kPhases; ++phase)
            for (int pair = 0; pair < n; ++pair) {
                const Chunk c = whole(pair, phase);
                emit(c.pair, c.phase, c.first, c.count);
            }
        start.push_back(position);
        return;
    }
    const int size = std::max(1, tuning.group_pairs);
    const int groups = (n + size - 1) / size;
    auto members = [&](int g, int *lo, int *hi) {
        *lo = g * size;
        *hi = std::min(n, *lo + size);
    };
    auto one = [&](int phase, int g) {  // one phase of every pair of group g
        Stream st;
        if (g < 0 || g >= groups) return st;
        int lo, hi;
        members(g, &lo, &hi);
        for (int p = lo; p < hi; ++p) st.push_back(whole(p, phase));
        return st;
    };
    auto paths = [&](int g) {  // longest first over the group's pairs
        Stream st;
        if (g < 0 || g >= groups) return st;
        int lo, hi;
        members(g, &lo, &hi);
        struct Item {
            int steps, pair, item;
        };
        std::vector<Item> all;
        for (int p = lo; p < hi; ++p) {
            const std::vector<int> steps = path_item_steps(pairs[p]);
            for (int i = 0; i < (int)steps.size(); ++i) all.push_back({steps[i], p, i});
        }
        std::stable_sort(all.begin(), all.end(),
                         [](const Item &a, const Item &b) { return a.steps > b.steps; });
        for (const Item &it : all) {
            const double micros =
                phase_micros(specs[it.pair], kPaths) / std::max(pairs[it.pair].items[kPaths], 1);
            if (!st.empty() && st.back().pair == it.pair &&
                st.back().first + st.back().count == it.item) {
                st.back().count += 1;
                st.back().micros += micros;
            } else {
                st.push_back({it.pair, kPaths, it.item, 1, micros});
            }
        }
        return st;
    };
    for (int i = -2; i <= groups + 2; ++i) {
        merge({one(kCensus, i + 2), one(kCosts, i + 1), one(kCheck, i - 2), one(kMedian, i - 3)},
              quantum, emit);
        merge({paths(i + 1), one(kSelect, i - 1)}, quantum, emit);
    }
    start.push_back(position);
}

// The streams engine: each pair's single-pair matcher (census, costs, paths,
// selection, check, median: the kernels nxs_sgm runs) as a chain on one of
// the side streams, forked from and joined back to the batch's stream, the
// largest pairs first onto the least loaded stream. Chains of different pairs
// overlap on the device: one pair's path aggregation (integer-pipe bound, with
// few warps per SM) beside others' costs (popcount bound) and selection (HBM
// bound).
// Returns the first launch error of the chains (none: cudaSuccess), with the
// pair it came from in *failed_pair.
cudaError_t fork_chains(nxs_batch *b, int *failed_pair) {
    const int streams = (int)b->side.size();
    cudaEventRecord(b->fork, b->stream);
    for (cudaStream_t side : b->side) cudaStreamWaitEvent(side, b->fork, 0);
    std::vector<int> order(b->specs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    auto work = [&](int i) {
        const nxs_batch_pair &s = b->specs[i];
        return (double)s.width * s.height * s.params.disparities * s.params.paths;
    };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work(x) > work(y); });
    std::vector<double> load(streams, 0.0);
    cudaError_t first = cudaSuccess;
    for (int i : order) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[k] += work(i);
        const nxs_batch_pair &s = b->specs[i];
        const BatchPair &P = b->pairs[i];
        MatcherScratch scratch;
        scratch.costs = P.costs;
        scratch.paths = P.paths;
        scratch.selected = P.raw;
        scratch.keys = P.right_map;
        const cudaError_t e = run_matcher(
            P.left, P.right, (int)s.width, (int)s.height, (int)s.params.disparities,
            (int)s.params.paths, (int)s.params.p1, (int)s.params.p2, s.params.uniqueness,
            s.params.stage_mask ? 1 : 0, scratch, P.disparity, b->side[k], streams > 1);
        if (e != cudaSuccess && first == cudaSuccess) {
            first = e;
            *failed_pair = i;
        }
    }
    for (int k = 0; k < streams; ++k) {
        cudaEventRecord(b->joins[k], b->side[k]);
        cudaStreamWaitEvent(b->stream, b->joins[k], 0);
    }
    return first;
}

nxs_status capture(nxs_batch *b, bool host, cudaGraphExec_t *out, char *error, size_t error_len) {
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e) return cuda_failed(e, error, error_len, "graph capture");
    if (host)
        cudaMemcpyAsync(b->arena, b->staging, b->input_bytes, cudaMemcpyHostToDevice, b->stream);
    cudaMemsetAsync(b->d_control, 0, b->control_bytes, b->stream);
    cudaError_t chains = cudaSuccess;
    int failed_pair = -1;
    if (b->tuning.engine == 1) {
        chains = fork_chains(b, &failed_pair);
    } else {
        auto kernel = b->wide ? batch_kernel<true> : batch_kernel<false>;
        kernel<<<b->grid, kThreads, b->shared_bytes, b->stream>>>(
            b->d_pairs, b->d_queue, b->total, b->d_control, wait_limit_ns(b->tuning));
    }
    if (host)
        cudaMemcpyAsync(b->staging + b->input_bytes, b->arena + b->input_bytes, b->output_bytes,
                        cudaMemcpyDeviceToHost, b->stream);
    const cudaError_t launched = cudaGetLastError();
    e = cudaStreamEndCapture(b->stream, &graph);
    if (chains != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        char where[96];
        snprintf(where, sizeof where, "capturing the kernels of pair %d", failed_pair);
        return cuda_failed(chains, error, error_len, where);
    }
    if (launched) e = launched;
    if (!e) e = cudaGraphInstantiate(out, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    return cuda_failed(e, error, error_len, "graph instantiation");
}

// Shapes every pair for tuning `t`, lays out the queue, uploads the tables
// and captures the two graphs (the buffers stay as they are).
nxs_status prepare(nxs_batch *b, const nxs_batch_tuning &t, char *error, size_t error_len) {
    const size_t n = b->specs.size();
    for (size_t i = 0; i < n; ++i) {
        BatchPair shaped{};
        shape_pair(b->specs[i], t, &shaped);
        BatchPair &P = b->pairs[i];
        const BatchPair buffers = P;
        P = shaped;
        P.left = buffers.left;
        P.right = buffers.right;
        P.left_codes = buffers.left_codes;
        P.right_codes = buffers.right_codes;
        P.costs = buffers.costs;
        P.paths = buffers.paths;
        P.raw = buffers.raw;
        P.right_map = buffers.right_map;
        P.checked = buffers.checked;
        P.disparity = buffers.disparity;
    }
    b->tuning = t;
    std::vector<unsigned> start, info, first;
    build_runs(b->specs, b->pairs, t, start, info, first);
    b->runs = (int)info.size();
    b->total = start.back();
    std::vector<uint2> queue(b->total);
    for (int r = 0; r < b->runs; ++r)
        for (unsigned q = start[r]; q < start[r + 1]; ++q)
            queue[q] = make_uint2(info[r], first[r] + (q - start[r]));

    int max_disparities = 16;
    for (const auto &s : b->specs)
        max_disparities = std::max(max_disparities, (int)s.params.disparities);
    int max_words = 4;
    for (const auto &P : b->pairs) max_words = std::max(max_words, P.path_words);
    b->wide = max_words == 16;
    b->shared_bytes = std::max({costs_shared_bytes(max_disparities),
                                (size_t)(kThreads / 32) * kPrefetch * 32 * 2 * max_words,
                                (size_t)(128 / 4) * 256 * sizeof(uint16_t),
                                (size_t)census4_tile_bytes(kCensusRows)});
    int sms = 0, resident = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    auto kernel = b->wide ? batch_kernel<true> : batch_kernel<false>;
    if (!e) e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)b->shared_bytes);
    if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, kThreads,
                                                              b->shared_bytes);
    if (!e) {
        b->grid = sms * std::max(1, std::min(resident, t.blocks_per_sm));
        b->grid = (int)std::min<size_t>((size_t)b->grid, b->total);
    }
    if (!e && !b->fork) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    while (!e && (int)b->side.size() < t.streams) {
        cudaStream_t side = nullptr;
        cudaEvent_t join = nullptr;
        e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking);
        if (!e) e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
        if (side) b->side.push_back(side);
        if (join) b->joins.push_back(join);
    }
    if (!e && (int)b->side.size() > t.streams) {  // fewer streams than before
        for (size_t k = t.streams; k < b->side.size(); ++k) {
            cudaStreamDestroy(b->side[k]);
            cudaEventDestroy(b->joins[k]);
        }
        b->side.resize(t.streams);
        b->joins.resize(t.streams);
    }
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->graph_host) cudaGraphExecDestroy(b->graph_host);
    b->graph = b->graph_host = nullptr;
    if (b->d_queue) cudaFree(b->d_queue);
    b->d_queue = nullptr;
    if (!e && !b->d_pairs) e = cudaMalloc(&b->d_pairs, sizeof(BatchPair) * n);
    if (!e) e = cudaMalloc(&b->d_queue, sizeof(uint2) * queue.size());
    if (!e) e = cudaMemcpy(b->d_pairs, b->pairs.data(), sizeof(BatchPair) * n,
                           cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(b->d_queue, queue.data(), sizeof(uint2) * queue.size(),
                           cudaMemcpyHostToDevice);
    nxs_status status = cuda_failed(e, error, error_len, "batch set-up");
    if (!status) status = capture(b, false, &b->graph, error, error_len);
    if (!status) status = capture(b, true, &b->graph_host, error, error_len);
    return status;
}

nxs_status check_batch(uint32_t n_pairs, const nxs_batch_pair *specs,
                       const nxs_batch_tuning *tuning, nxs_batch_tuning *chosen, char *error,
                       size_t error_len) {
    if (!specs || n_pairs == 0) {
        set_error(error, error_len, "no pairs");
        return NXS_BAD_ARGUMENT;
    }
    if (n_pairs > (1u << 20)) {
        set_error(error, error_len, "at most %u pairs in a batch, got %u", 1u << 20, n_pairs);
        return NXS_BAD_ARGUMENT;
    }
    nxs_batch_tuning t;
    nxs_batch_default_tuning(&t);
    if (tuning) t = *tuning;
    if (t.blocks_per_sm < 1 || t.blocks_per_sm > 16 || t.cost_rows < 1 || t.cost_rows > 64 ||
        t.select_passes < 1 || t.select_passes > 256 || t.group_pairs < 1 ||
        t.group_pairs > 1024 || !(t.quantum_us > 0.0f && t.quantum_us <= 1000.0f) ||
        (t.order != 0 && t.order != 1) ||
        (t.path_words != 0 && t.path_words != 4 && t.path_words != 8 && t.path_words != 16) ||
        (t.engine != 0 && t.engine != 1) || t.streams < 1 || t.streams > 64 ||
        t.wait_limit_us > 60000000u) {
        set_error(error, error_len,
                  "tuning out of range: blocks_per_sm 1..16, cost_rows 1..64, select_passes "
                  "1..256, group_pairs 1..1024, quantum_us in (0, 1000], order 0 or 1, "
                  "path_words 0, 4, 8 or 16, engine 0 or 1, streams 1..64, wait_limit_us "
                  "0..60000000");
        return NXS_BAD_ARGUMENT;
    }
    for (uint32_t i = 0; i < n_pairs; ++i) {
        char reason[200];
        if (nxs_sgm_check(&specs[i].params, specs[i].width, specs[i].height, reason,
                          sizeof reason)) {
            set_error(error, error_len, "pair %u: %s", i, reason);
            return NXS_BAD_ARGUMENT;
        }
    }
    *chosen = t;
    return NXS_OK;
}

}  // namespace

extern "C" void nxs_batch_default_tuning(nxs_batch_tuning *t) {
    if (!t) return;
    t->blocks_per_sm = 8;
    t->cost_rows = 4;
    t->select_passes = 16;
    t->group_pairs = 16;
    t->quantum_us = 2.0f;
    t->order = 1;
    t->path_words = 0;
    t->engine = 0;
    t->streams = 8;
    t->wait_limit_us = 0;
}

extern "C" nxs_status nxs_batch_create(nxs_context *context, uint32_t n_pairs,
                                       const nxs_batch_pair *specs,
                                       const nxs_batch_tuning *tuning, nxs_batch **out,
                                       char *error, size_t error_len) {
    if (!context || !out) {
        set_error(error, error_len, "a NULL context or result");
        return NXS_BAD_ARGUMENT;
    }
    *out = nullptr;
    nxs_batch_tuning t;
    nxs_status status = check_batch(n_pairs, specs, tuning, &t, error, error_len);
    if (status) return status;
    auto b = new nxs_batch();
    b->device = context_device(context);
    b->tuning = t;
    b->specs.assign(specs, specs + n_pairs);
    cudaSetDevice(b->device);

    // Layout: inputs (both images of every pair), then the control words and
    // every pair's output, then the intermediates; each buffer 256-aligned.
    size_t at = 0;
    for (const auto &s : b->specs) {
        const size_t px = (size_t)s.width * s.height;
        b->input_offsets.push_back(at);
        at += 2 * align256(px);
    }
    b->input_bytes = at;
    b->control_bytes = align256(sizeof(unsigned) * (kControlWords + (size_t)kPhases * n_pairs));
    at += b->control_bytes;
    for (const auto &s : b->specs) {
        b->output_offsets.push_back(at);
        at += align256(sizeof(float) * s.width * s.height);
    }
    b->output_bytes = at - b->input_bytes;
    std::vector<size_t> scratch_offsets;
    for (const auto &s : b->specs) {
        const size_t px = (size_t)s.width * s.height, volume = px * s.params.disparities;
        scratch_offsets.push_back(at);
        at += 2 * align256(8 * px) + align256(volume) + s.params.paths * align256(volume) +
              3 * align256(4 * px);
    }
    b->arena_bytes = at;

    size_t free_bytes = 0, total_bytes = 0;
    cudaMemGetInfo(&free_bytes, &total_bytes);
    if (b->arena_bytes + (512ull << 20) > free_bytes) {
        set_error(error, error_len,
                  "the batch needs %.2f GB of device memory and %.2f GB are free",
                  b->arena_bytes / 1e9, free_bytes / 1e9);
        delete b;
        return NXS_BAD_ARGUMENT;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (!e) e = cudaMalloc(&b->arena, b->arena_bytes);
    if (!e) e = cudaHostAlloc(&b->staging, b->input_bytes + b->output_bytes, cudaHostAllocDefault);
    if (e) {
        status = cuda_failed(e, error, error_len, "batch allocation");
        nxs_batch_destroy(b);
        return status;
    }
    b->d_control = reinterpret_cast<unsigned *>(b->arena + b->input_bytes);

    for (uint32_t i = 0; i < n_pairs; ++i) {
        const nxs_batch_pair &s = b->specs[i];
        const size_t px = (size_t)s.width * s.height, volume = px * s.params.disparities;
        BatchPair P{};
        shape_pair(s, t, &P);
        P.left = b->arena + b->input_offsets[i];
        P.right = P.left + align256(px);
        P.disparity = reinterpret_cast<float *>(b->arena + b->output_offsets[i]);
        uint8_t *p = b->arena + scratch_offsets[i];
        auto take = [&](size_t bytes) {
            uint8_t *r = p;
            p += align256(bytes);
            return r;
        };
        P.left_codes = reinterpret_cast<uint64_t *>(take(8 * px));
        P.right_codes = reinterpret_cast<uint64_t *>(take(8 * px));
        P.costs = take(volume);
        P.paths = p;
        p += s.params.paths * align256(volume);
        P.raw = reinterpret_cast<float *>(take(4 * px));
        P.right_map = reinterpret_cast<uint32_t *>(take(4 * px));
        P.checked = reinterpret_cast<float *>(take(4 * px));
        b->pairs.push_back(P);
    }

    status = prepare(b, t, error, error_len);
    if (status) {
        nxs_batch_destroy(b);
        return status;
    }
    std::memset(b->staging, 0, b->input_bytes + b->output_bytes);
    *out = b;
    return NXS_OK;
}

extern "C" nxs_status nxs_batch_retune(nxs_batch *b, const nxs_batch_tuning *tuning,
                                       char *error, size_t error_len) {
    if (!b) {
        set_error(error, error_len, "a NULL batch");
        return NXS_BAD_ARGUMENT;
    }
    nxs_batch_tuning t;
    nxs_status status = check_batch((uint32_t)b->specs.size(), b->specs.data(), tuning, &t, error,
                                    error_len);
    if (status) return status;
    std::lock_guard<std::mutex> g(b->lock);
    cudaSetDevice(b->device);
    status = cuda_failed(cudaStreamSynchronize(b->stream), error, error_len, "batch retune");
    if (!status) status = prepare(b, t, error, error_len);
    return status;
}

extern "C" nxs_status nxs_batch_queue(uint32_t n_pairs, const nxs_batch_pair *specs,
                                      const nxs_batch_tuning *tuning, uint32_t *items,
                                      uint32_t *runs, uint32_t capacity, uint32_t *n_runs,
                                      char *error, size_t error_len) {
    nxs_batch_tuning t;
    nxs_status status = check_batch(n_pairs, specs, tuning, &t, error, error_len);
    if (status) return status;
    std::vector<nxs_batch_pair> list(specs, specs + n_pairs);
    std::vector<BatchPair> pairs(n_pairs);
    for (uint32_t i = 0; i < n_pairs; ++i) shape_pair(list[i], t, &pairs[i]);
    std::vector<unsigned> start, info, first;
    build_runs(list, pairs, t, start, info, first);
    if (n_runs) *n_runs = (uint32_t)info.size();
    if (items)
        for (uint32_t i = 0; i < n_pairs; ++i)
            for (int k = 0; k < kPhases; ++k) items[i * kPhases + k] = (uint32_t)pairs[i].items[k];
    if (runs && capacity >= info.size())
        for (size_t r = 0; r < info.size(); ++r) {
            runs[4 * r + 0] = start[r];
            runs[4 * r + 1] = info[r] >> 4;
            runs[4 * r + 2] = info[r] & 15u;
            runs[4 * r + 3] = first[r];
        }
    return NXS_OK;
}

extern "C" nxs_status nxs_batch_buffers(nxs_batch *b, uint32_t pair, int device_side,
                                        uint8_t **left, uint8_t **right, float **disparity) {
    if (!b || pair >= b->specs.size()) return NXS_BAD_ARGUMENT;
    uint8_t *base = device_side ? b->arena : b->staging;
    const size_t px = (size_t)b->specs[pair].width * b->specs[pair].height;
    if (left) *left = base + b->input_offsets[pair];
    if (right) *right = base + b->input_offsets[pair] + align256(px);
    if (disparity) *disparity = reinterpret_cast<float *>(base + b->output_offsets[pair]);
    return NXS_OK;
}

extern "C" nxs_status nxs_batch_launch(nxs_batch *b, int host_buffers, void *stream,
                                       char *error, size_t error_len) {
    if (!b) {
        set_error(error, error_len, "a NULL batch");
        return NXS_BAD_ARGUMENT;
    }
    cudaSetDevice(b->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
    return cuda_failed(cudaGraphLaunch(host_buffers ? b->graph_host : b->graph, s), error,
                       error_len, "batch launch");
}

extern "C" nxs_status nxs_batch_run(nxs_batch *b, char *error, size_t error_len) {
    if (!b) {
        set_error(error, error_len, "a NULL batch");
        return NXS_BAD_ARGUMENT;
    }
    std::lock_guard<std::mutex> g(b->lock);
    nxs_status s = nxs_batch_launch(b, 1, nullptr, error, error_len);
    if (s) return s;
    s = cuda_failed(cudaStreamSynchronize(b->stream), error, error_len, "batch run");
    if (s) return s;
    const unsigned *control = reinterpret_cast<const unsigned *>(b->staging + b->input_bytes);
    if (control[1]) {
        set_error(error, error_len, "a batch item waited more than %.6f s for the phase before it",
                  wait_limit_ns(b->tuning) / 1e9);
        return NXS_TIMEOUT;
    }
    return NXS_OK;
}

extern "C" nxs_status nxs_batch_check(nxs_batch *b, char *error, size_t error_len) {
    if (!b) {
        set_error(error, error_len, "a NULL batch");
        return NXS_BAD_ARGUMENT;
    }
    cudaSetDevice(b->device);
    unsigned status = 0;
    nxs_status s = cuda_failed(cudaMemcpy(&status, b->d_control + 1, sizeof status,
                                          cudaMemcpyDeviceToHost),
                               error, error_len, "batch status");
    if (s) return s;
    if (status) {
        set_error(error, error_len, "a batch item waited more than %.6f s for the phase before it",
                  wait_limit_ns(b->tuning) / 1e9);
        return NXS_TIMEOUT;
    }
    return NXS_OK;
}

extern "C" nxs_status nxs_batch_hold_phase(nxs_batch *b, uint32_t pair, uint32_t phase,
                                           char *error, size_t error_len) {
    if (!b || pair >= b->specs.size() || phase < 1 || phase >= (uint32_t)kPhases) {
        set_error(error, error_len, "a NULL batch, or a pair or phase (1..%d) out of range",
                  kPhases - 1);
        return NXS_BAD_ARGUMENT;
    }
    std::lock_guard<std::mutex> g(b->lock);
    cudaSetDevice(b->device);
    BatchPair held = b->pairs[pair];
    held.items[phase - 1] += 1;  // one item more than the phase before has: never reached
    // Only the `items` entry of the device copy changes; the host plan stays.
    const size_t offset = sizeof(BatchPair) * pair + offsetof(BatchPair, items) +
                          sizeof(int) * (phase - 1);
    return cuda_failed(cudaMemcpy(reinterpret_cast<char *>(b->d_pairs) + offset,
                                  &held.items[phase - 1], sizeof(int), cudaMemcpyHostToDevice),
                       error, error_len, "batch hold");
}

extern "C" nxs_status nxs_batch_clocks(nxs_batch *b, uint64_t *cycles) {
    if (!b || !cycles) return NXS_BAD_ARGUMENT;
    cudaSetDevice(b->device);
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (!e) e = cudaMemcpy(cycles, b->d_control + 4, kClocks * sizeof(uint64_t),
                           cudaMemcpyDeviceToHost);
    return e ? NXS_CUDA_ERROR : NXS_OK;
}

extern "C" nxs_status nxs_batch_info(const nxs_batch *b, nxs_batch_stats *stats) {
    if (!b || !stats) return NXS_BAD_ARGUMENT;
    stats->pairs = (uint32_t)b->specs.size();
    stats->items = b->total;
    stats->runs = (uint32_t)b->runs;
    stats->blocks = (uint32_t)b->grid;
    stats->shared_bytes = b->shared_bytes;
    stats->device_bytes = b->arena_bytes;
    stats->input_bytes = b->input_bytes;
    stats->output_bytes = b->output_bytes;
    return NXS_OK;
}

extern "C" void nxs_batch_destroy(nxs_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->graph_host) cudaGraphExecDestroy(b->graph_host);
    if (b->d_queue) cudaFree(b->d_queue);
    if (b->d_pairs) cudaFree(b->d_pairs);
    if (b->arena) cudaFree(b->arena);
    if (b->staging) cudaFreeHost(b->staging);
    for (cudaStream_t side : b->side) cudaStreamDestroy(side);
    for (cudaEvent_t join : b->joins) cudaEventDestroy(join);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}
