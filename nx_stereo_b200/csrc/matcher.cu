// The full-search matcher of NxStereo.sgm/3 on B200: census, the u8 Hamming
// cost volume, the path recurrence along every scan line, selection, the
// left-right check and the median.
//
// Layout in HBM for a W x H pair and D disparities (D a multiple of 16):
//   costs      u8  [H][W][D]     Hamming costs, 0..48 (the census codes of both
//                                images stay in the census + costs kernel's
//                                shared memory)
//   paths      u8  [P][H][W][D]  each direction's path costs, 0..p2+48 <= 127
//   selected   f32 [H][W], keys u32 [H][W]
// Disparities are the fastest axis so that one scan-line step reads and
// writes D contiguous bytes: one coalesced 128-byte transaction per warp at
// D = 128.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <type_traits>

#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

#include "nxs_kernels.h"
#include "nxs_matcher.cuh"

namespace nxs {

// ---------------------------------------------------------------- census
// A block of 256 threads takes 128 x 8 pixels of one image (blockIdx.z), four
// pixels a thread.
constexpr int kCensus4Rows = 8, kCensus4Threads = 256;

__global__ void __launch_bounds__(kCensus4Threads)
    census_kernel(const uint8_t *__restrict__ left, const uint8_t *__restrict__ right, int width,
                  int height, uint64_t *__restrict__ left_codes,
                  uint64_t *__restrict__ right_codes) {
    __shared__ __align__(16) uint8_t tile[census4_tile_bytes(kCensus4Rows)];
    follow_previous_grid();
    census4_tile<kCensus4Rows, kCensus4Threads>(
        blockIdx.z == 0 ? left : right, width, height,
        blockIdx.z == 0 ? left_codes : right_codes, blockIdx.x * kCensus4X,
        blockIdx.y * kCensus4Rows, threadIdx.x, tile);
}

cudaError_t launch_census(const uint8_t *left, const uint8_t *right, int width, int height,
                          uint64_t *left_codes, uint64_t *right_codes, cudaStream_t stream) {
    dim3 grid((width + kCensus4X - 1) / kCensus4X, (height + kCensus4Rows - 1) / kCensus4Rows,
              right ? 2 : 1);
    return launch_after(census_kernel, grid, dim3(kCensus4Threads), 0, stream, left, right,
                        width, height, left_codes, right_codes);
}

// ---------------------------------------------------------------- costs
template <int SPAN>
__global__ void __launch_bounds__(128)
    costs_kernel(const uint64_t *__restrict__ left_codes, const uint64_t *__restrict__ right_codes,
                 int width, int disparities, uint8_t *__restrict__ costs) {
    follow_previous_grid();
    extern __shared__ __align__(16) uint8_t staged[];
    costs_tile<SPAN>(left_codes, right_codes, width, disparities, costs,
                     blockIdx.x * kCostPixels, blockIdx.y, staged);
}

cudaError_t launch_costs(const uint64_t *left_codes, const uint64_t *right_codes, int width,
                         int height, int disparities, uint8_t *costs, cudaStream_t stream,
                         int span) {
    dim3 grid((width + kCostPixels - 1) / kCostPixels, height);
    const size_t shared = costs_shared_bytes(disparities);
#define NXS_COSTS(S)                                                                          \
    launch_after(costs_kernel<S>, grid, dim3(128), shared, stream, left_codes, right_codes,   \
                 width, disparities, costs)
    if (span == 16) NXS_COSTS(16);
    else if (span == 8) NXS_COSTS(8);
    else NXS_COSTS(0);
#undef NXS_COSTS
    return cudaGetLastError();
}

// ---------------------------------------------------------------- census + costs
// A block of 128 threads takes kCensusCostPixels pixels of one row: the
// census of both images around them and their costs (census_costs_tile).
template <int SPAN>
__global__ void __launch_bounds__(128)
    census_costs_kernel(const uint8_t *__restrict__ left, const uint8_t *__restrict__ right,
                        int width, int height, int disparities, uint8_t *__restrict__ costs) {
    follow_previous_grid();
    extern __shared__ __align__(16) uint8_t staged[];
    census_costs_tile<SPAN, kCensusCostPixels, 128>(left, right, width, height, disparities,
                                                    costs, blockIdx.x * kCensusCostPixels,
                                                    blockIdx.y, staged, threadIdx.x);
}

cudaError_t launch_census_costs(const uint8_t *left, const uint8_t *right, int width, int height,
                                int disparities, uint8_t *costs, cudaStream_t stream, int span) {
    if (disparities < 16 || disparities > 256 || disparities % 16) return cudaErrorInvalidValue;
    dim3 grid((width + kCensusCostPixels - 1) / kCensusCostPixels, height);
    const size_t shared = census_costs_shared_bytes(kCensusCostPixels, disparities);
#define NXS_CENSUS_COSTS(S)                                                                   \
    launch_after(census_costs_kernel<S>, grid, dim3(128), shared, stream, left, right, width, \
                 height, disparities, costs)
    if (span == 16) NXS_CENSUS_COSTS(16);
    else if (span == 8) NXS_CENSUS_COSTS(8);
    else NXS_CENSUS_COSTS(0);
#undef NXS_CENSUS_COSTS
    return cudaGetLastError();
}

// ---------------------------------------------------------------- paths
// One warp per block, so blocks go to SMs as they free up, longest lines first.
// SUMS: every direction adds into one u16 aggregate volume (follow_lines).
// TILES: the blocks of steps every line of a warp covers take their costs by
// bulk tensor copies of `maps` into kTileStages stages of 8 steps x 32 lanes
// x 16 bytes; the per-lane ring of the other steps shares the first stage.
template <int G, int WORDS, bool FULL, int SPAN, bool SUMS = false, bool TILES = false>
__global__ void __launch_bounds__(32)
    paths_kernel(const uint8_t *__restrict__ costs, uint8_t *__restrict__ paths_out,
                 const PathSetup s, const __grid_constant__ CostMaps maps) {
    using Piece = typename std::conditional<WORDS == 4, uint2, uint4>::type;
    constexpr int PIECES = WORDS == 16 ? 2 : 1;
    constexpr int RING_BYTES = kPrefetch * PIECES * 32 * (int)sizeof(Piece);
    constexpr int TILE_BYTES = kTileStages * kPrefetch * 32 * 16;
    static_assert(!TILES || RING_BYTES <= TILE_BYTES / kTileStages, "the ring fits one stage");
    __shared__ __align__(128) uint8_t room[TILES ? TILE_BYTES : RING_BYTES];
    __shared__ __align__(8) uint64_t bars[TILES ? kTileStages : 1];
    if constexpr (TILES) {
        if (threadIdx.x == 0) {
            for (int k = 0; k < kTileStages; ++k) barrier_init(&bars[k], 32 / G);
            barrier_init_fence();
        }
        __syncwarp();
    }
    follow_previous_grid();
    path_warp<G, WORDS, FULL, SPAN, SUMS, TILES>(costs, paths_out, s, blockIdx.x, threadIdx.x,
                                                 reinterpret_cast<Piece *>(room) + threadIdx.x,
                                                 &maps, room, bars);
}

// ---- the cost volume's tensor maps (cuTensorMapEncodeTiled, from the driver) ----
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult found;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &found) ==
                cudaSuccess &&
            found == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    return encode;
}

// The four views of a [H][W][D] u8 cost volume that CostMaps describes; false
// where the driver refuses one (then the scan takes the per-lane copies).
static bool encode_cost_maps(const uint8_t *costs, int width, int height, int disparities,
                             CostMaps *maps) {
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode || width < 2 || height < 2) return false;
    const cuuint64_t D = (cuuint64_t)disparities;
    const cuuint64_t pixels = (cuuint64_t)width * (cuuint64_t)height;
    auto view = [&](CUtensorMap *map, cuuint64_t step_pixels) {
        const cuuint64_t dims[3] = {D, (cuuint64_t)kPrefetch, pixels};
        const cuuint64_t strides[2] = {step_pixels * D, D};  // bytes, of dimensions 1 and 2
        const cuuint32_t box[3] = {(cuuint32_t)D, (cuuint32_t)kPrefetch, 1};
        const cuuint32_t element_strides[3] = {1, 1, 1};
        return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t *>(costs), dims,
                      strides, box, element_strides, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    const cuuint64_t W = (cuuint64_t)width;
    return view(&maps->row, 1) && view(&maps->column, W) && view(&maps->diagonal, W + 1) &&
           view(&maps->anti, W - 1);
}

// Whether the path scans take their full blocks' costs by tensor copies: 0
// never, 2 always, 1 (the default) from kTilesFrom pixel-disparities on,
// where they measured faster (1280x720x128: 295 against 300 us, 1920x1080x256:
// 1329 against 1360 us); below it the per-lane copies were (728x544x128: 121
// against 129 us, 364x272x64: 40 against 53 us). Results do not depend on it.
static std::atomic<int> g_path_tiles{1};
constexpr size_t kTilesFrom = (size_t)96 << 20;
void set_path_tiles(int mode) { g_path_tiles = mode < 0 || mode > 2 ? 1 : mode; }
int path_tiles() { return g_path_tiles; }
static bool tiles_wanted(int width, int height, int disparities) {
    return g_path_tiles == 2 ||
           (g_path_tiles == 1 && (size_t)width * height * disparities >= kTilesFrom);
}

unsigned path_wait_failures() {
    unsigned n = 0;
    if (cudaMemcpyFromSymbol(&n, g_path_wait_failures, sizeof n) != cudaSuccess) return ~0u;
    return n;
}

// Zeroes `chunks` 16-byte chunks (the aggregate volume before the summing scan).
__global__ void __launch_bounds__(256) clear_kernel(uint4 *__restrict__ to, size_t chunks) {
    follow_previous_grid();
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < chunks; i += stride)
        to[i] = make_uint4(0, 0, 0, 0);
}

// Words a path lane holds at each disparity count (4, 8 or 16), the tunable
// shape of the path kernels; words_slot maps 64..256 to the table.
static std::atomic<int> g_path_words[5] = {8, 8, 8, 8, 8};
static int words_slot(int disparities) {
    return disparities <= 64 ? 0 : disparities <= 96 ? 1 : disparities <= 128 ? 2
                                   : disparities <= 192 ? 3 : 4;
}
int path_words(int disparities) { return g_path_words[words_slot(disparities)]; }
void set_path_words(int disparities, int words) {
    g_path_words[words_slot(disparities)] = words == 4 ? 4 : (words == 16 ? 16 : 8);
}

int path_setup(int width, int height, int disparities, int paths, int p1, int p2, int lanes,
               PathSetup *setup) {
    PathSetup &s = *setup;
    s = PathSetup{};
    s.width = width;
    s.height = height;
    s.disparities = disparities;
    s.p1 = p1;
    s.p2 = p2;
    s.paths = paths;
    s.volume = (size_t)width * height * disparities;
    s.one = 1u;
    const int lines_per_warp = 32 / lanes;
    // Rows, then columns, then diagonals.
    int n = 0;
    for (int pass = 0; pass < 3; ++pass) {
        for (int p = 0; p < paths; ++p) {
            const int dy = kDirections[p][0], dx = kDirections[p][1];
            const int kind = dy == 0 ? 0 : (dx == 0 ? 1 : 2);
            if (kind == pass) s.order[n++] = p;
        }
        if (pass == 1) s.straight = n;
    }
    for (int p = 0; p < paths; ++p) {
        s.dy[p] = kDirections[p][0];
        s.dx[p] = kDirections[p][1];
        s.lines[p] = s.dy[p] == 0 ? height : (s.dx[p] == 0 ? width : width + height - 1);
    }
    int total = 0;
    for (int slot = 0; slot < s.straight; ++slot) {
        s.first_warp[slot] = total;
        total += (s.lines[s.order[slot]] + lines_per_warp - 1) / lines_per_warp;
    }
    // The diagonals share one range of warps starting at slot `straight`;
    // every later slot starts at the end, so the slot search stops in range.
    const int diagonals = paths - s.straight;
    s.first_warp[s.straight] = total;
    if (diagonals) total += (width + height - 1 + lines_per_warp - 1) / lines_per_warp * diagonals;
    for (int slot = s.straight + 1; slot <= 8; ++slot) s.first_warp[slot] = total;
    return total;
}

// The path kernel is one wave of one-warp blocks whose time is set by the most
// loaded SM. launch_after starts it as the costs kernel's last block exits, so
// its blocks spread over idle SMs; with an early signal from every costs block
// (griddepcontrol.launch_dependents at their start) they landed unevenly beside
// the costs kernel's last wave and a pair took 525 us instead of 290.
template <int WORDS, bool PERMUTED>
static void launch_paths_in(const uint8_t *costs, uint8_t *paths_out, const PathSetup &s,
                            int total, int g, cudaStream_t stream) {
    constexpr int SPAN = PERMUTED ? (WORDS == 4 ? 8 : 16) : 0;
    const bool full = g * 2 * WORDS == s.disparities;
    CostMaps maps{};
    if constexpr (WORDS == 8 && PERMUTED) {
        if (full && tiles_wanted(s.width, s.height, s.disparities) &&
            encode_cost_maps(costs, s.width, s.height, s.disparities, &maps)) {
#define NXS_TILED(G)                                                                           \
    launch_after(paths_kernel<G, 8, true, 16, false, true>, dim3(total), dim3(32), 0, stream,  \
                 costs, paths_out, s, maps)
            if (g == 4) NXS_TILED(4);
            else if (g == 8) NXS_TILED(8);
            else NXS_TILED(16);
#undef NXS_TILED
            return;
        }
    }
#define NXS_PATHS(G, F)                                                                        \
    launch_after(paths_kernel<G, WORDS, F, SPAN>, dim3(total), dim3(32), 0, stream, costs,    \
                 paths_out, s, maps)
    if constexpr (WORDS == 16) {
        if (g == 2) full ? NXS_PATHS(2, true) : NXS_PATHS(2, false);
        else if (g == 4) full ? NXS_PATHS(4, true) : NXS_PATHS(4, false);
        else full ? NXS_PATHS(8, true) : NXS_PATHS(8, false);
    } else if constexpr (WORDS == 8) {
        if (g == 4) full ? NXS_PATHS(4, true) : NXS_PATHS(4, false);
        else if (g == 8) full ? NXS_PATHS(8, true) : NXS_PATHS(8, false);
        else full ? NXS_PATHS(16, true) : NXS_PATHS(16, false);
    } else {
        if (g == 8) full ? NXS_PATHS(8, true) : NXS_PATHS(8, false);
        else if (g == 16) full ? NXS_PATHS(16, true) : NXS_PATHS(16, false);
        else full ? NXS_PATHS(32, true) : NXS_PATHS(32, false);
    }
#undef NXS_PATHS
}

int matcher_span(int disparities) { return path_words(disparities) == 4 ? 8 : 16; }

cudaError_t launch_paths(const uint8_t *costs, int width, int height, int disparities, int paths,
                         int p1, int p2, uint8_t *paths_out, cudaStream_t stream, int span) {
    // Words a lane holds: the tuned count, unless the order needs another.
    int words = path_words(disparities);
    if (span == 8) words = 4;
    else if (span == 16 && words == 4) words = 8;
    const bool permuted = span != 0;
    const int g = path_lanes(disparities, words);
    // The kernels take 2..8 lanes a line at 16 words, 4..16 at 8 and 8..32 at
    // 4 (64 to 256 disparities); fewer would be launched with the wrong shape.
    if (g < (words == 16 ? 2 : words == 8 ? 4 : 8) || g > 256 / (2 * words))
        return cudaErrorInvalidValue;
    PathSetup s;
    const int total = path_setup(width, height, disparities, paths, p1, p2, g, &s);
    if (words == 16) {
        if (permuted) launch_paths_in<16, true>(costs, paths_out, s, total, g, stream);
        else launch_paths_in<16, false>(costs, paths_out, s, total, g, stream);
    } else if (words == 8) {
        if (permuted) launch_paths_in<8, true>(costs, paths_out, s, total, g, stream);
        else launch_paths_in<8, false>(costs, paths_out, s, total, g, stream);
    } else {
        if (permuted) launch_paths_in<4, true>(costs, paths_out, s, total, g, stream);
        else launch_paths_in<4, false>(costs, paths_out, s, total, g, stream);
    }
    return cudaGetLastError();
}

// How the matcher aggregates: 0 (the default) the path volumes, then
// selection over all of them; 1 the summing scan into one aggregate volume,
// then selection over it. The reductions run at a few TB/s in L2, below what
// the path volumes' plain stores reach, so 1 measured slower at every size
// from 364x272x64 to 1920x1080x256 and is kept as a knob, not a default.
static std::atomic<int> g_path_sums{0};
void set_path_sums(int mode) { g_path_sums = mode == 1 ? 1 : 0; }
int path_sums_mode() { return g_path_sums; }

bool path_sums_wanted(int width, int height, int disparities) {
    (void)width;
    (void)height;
    return g_path_sums == 1 && disparities % 16 == 0 && path_words(disparities) == 8;
}

cudaError_t launch_paths_sums(const uint8_t *costs, int width, int height, int disparities,
                              int paths, int p1, int p2, uint16_t *sums, cudaStream_t stream) {
    if (disparities % 16 != 0) return cudaErrorInvalidValue;
    const int g = path_lanes(disparities, 8);
    if (g < 4 || g > 16) return cudaErrorInvalidValue;
    const size_t chunks = (size_t)width * height * disparities * 2 / 16;
    cudaError_t e = launch_after(clear_kernel, dim3(4 * 148), dim3(256), 0, stream,
                                 reinterpret_cast<uint4 *>(sums), chunks);
    if (e != cudaSuccess) return e;
    PathSetup s;
    const int total = path_setup(width, height, disparities, paths, p1, p2, g, &s);
    const bool full = g * 16 == disparities;
    uint8_t *out = reinterpret_cast<uint8_t *>(sums);
    const CostMaps maps{};
#define NXS_SUMS(G, F)                                                                         \
    launch_after(paths_kernel<G, 8, F, 16, true>, dim3(total), dim3(32), 0, stream, costs, out, s, \
                 maps)
    if (g == 4) full ? NXS_SUMS(4, true) : NXS_SUMS(4, false);
    else if (g == 8) full ? NXS_SUMS(8, true) : NXS_SUMS(8, false);
    else full ? NXS_SUMS(16, true) : NXS_SUMS(16, false);
#undef NXS_SUMS
    return cudaGetLastError();
}

// sums[y][x][d] = sum of the P path volumes, u16 (at most 8 x 127 = 1016).
__global__ void sum_paths_kernel(const uint8_t *__restrict__ paths_in, size_t volume, int paths,
                                 uint16_t *__restrict__ sums) {
    follow_previous_grid();
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t quads = volume / 4;
    if (i >= quads) return;
    uint32_t lo = 0, hi = 0;
    for (int p = 0; p < paths; ++p) {
        uint32_t c = __ldg(reinterpret_cast<const uint32_t *>(paths_in + p * volume) + i);
        lo += __byte_perm(c, 0, 0x4140);
        hi += __byte_perm(c, 0, 0x4342);
    }
    reinterpret_cast<uint2 *>(sums)[i] = make_uint2(lo, hi);
}

cudaError_t launch_sum_paths(const uint8_t *paths_in, int width, int height, int disparities,
                             int paths, uint16_t *sums, cudaStream_t stream) {
    size_t volume = (size_t)width * height * disparities;
    size_t quads = volume / 4;
    return launch_after(sum_paths_kernel, dim3((unsigned)((quads + 255) / 256)), dim3(256), 0,
                        stream, paths_in, volume, paths, sums);
}

// ---------------------------------------------------------------- select
// `one` is 1, given at run time (select_pixels adds by multiply-adds).
template <int G, int PATHS, int SPAN>
__global__ void __launch_bounds__(128)
    select_kernel(const void *__restrict__ source, int width, int height, int disparities,
                  size_t volume, float uniqueness, float *__restrict__ disparity,
                  uint32_t *__restrict__ keys, uint32_t one) {
    follow_previous_grid();
    __shared__ __align__(16) uint16_t values_of[128 / G][256];
    select_pixels<G, PATHS, SPAN>(source, width, height, disparities, volume, uniqueness,
                                  disparity, keys, nullptr, blockIdx.x, values_of, one);
}

// select_kernel with a grid of `resident` blocks that step through the
// pixel blocks: a selection run beside another stream's path scan holds
// fewer warps a SM while it streams the path volumes.
template <int G, int PATHS, int SPAN>
__global__ void __launch_bounds__(128)
    select_lean_kernel(const void *__restrict__ source, int width, int height, int disparities,
                       size_t volume, float uniqueness, float *__restrict__ disparity,
                       uint32_t *__restrict__ keys, uint32_t one, size_t blocks) {
    follow_previous_grid();
    __shared__ __align__(16) uint16_t values_of[128 / G][256];
    for (size_t block = blockIdx.x; block < blocks; block += gridDim.x) {
        __syncwarp();  // the group's row of values_of is read before it is rewritten
        select_pixels<G, PATHS, SPAN>(source, width, height, disparities, volume, uniqueness,
                                      disparity, keys, nullptr, block, values_of, one);
    }
}

// Blocks a SM of the lean selection the split segments run beside a path scan
// (0: one block for each pixel block). 8 measured best end to end on the
// 728x544x128 chain: 2% above the full grid, 16 (above the 12 that fit a SM at
// 39 registers) 7% below it.
static std::atomic<int> g_lean_select{8};
void set_lean_select(int blocks_per_sm) { g_lean_select = blocks_per_sm < 0 ? 0 : blocks_per_sm; }
int lean_select() { return g_lean_select.load(); }

template <int PATHS, int SPAN = 0>
static cudaError_t launch_select(const void *source, int width, int height, int disparities,
                                 float uniqueness, float *disparity, uint32_t *keys,
                                 cudaStream_t stream, int lean = 0) {
    const size_t pixels = (size_t)width * height;
    const size_t volume = pixels * disparities;
    const int g = group_lanes(disparities);
    const unsigned blocks = (unsigned)((pixels + 128 / g - 1) / (128 / g));
    if (lean > 0) {
        int device = 0, sms = 148;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const unsigned grid = std::min<unsigned>(blocks, (unsigned)(lean * sms));
#define NXS_LEAN(G)                                                                            \
    launch_after(select_lean_kernel<G, PATHS, SPAN>, dim3(grid), dim3(128), 0, stream, source,  \
                 width, height, disparities, volume, uniqueness, disparity, keys, 1u,           \
                 (size_t)blocks)
        if (g == 4) NXS_LEAN(4);
        else if (g == 8) NXS_LEAN(8);
        else NXS_LEAN(16);
#undef NXS_LEAN
        return cudaGetLastError();
    }
#define NXS_SELECT(G)                                                                         \
    launch_after(select_kernel<G, PATHS, SPAN>, dim3(blocks), dim3(128), 0, stream, source,   \
                 width, height, disparities, volume, uniqueness, disparity, keys, 1u)
    if (g == 4) NXS_SELECT(4);
    else if (g == 8) NXS_SELECT(8);
    else NXS_SELECT(16);
#undef NXS_SELECT
    return cudaGetLastError();
}

cudaError_t launch_select_paths(const uint8_t *paths_in, int width, int height, int disparities,
                                int paths, float uniqueness, float *disparity, uint32_t *keys,
                                cudaStream_t stream, int span, int lean) {
#define NXS_SELECT_SPAN(S)                                                                     \
    return paths == 8 ? launch_select<8, S>(paths_in, width, height, disparities, uniqueness,   \
                                            disparity, keys, stream, lean)                     \
                      : launch_select<3, S>(paths_in, width, height, disparities, uniqueness,   \
                                            disparity, keys, stream, lean)
    if (span == 16) NXS_SELECT_SPAN(16);
    if (span == 8) NXS_SELECT_SPAN(8);
#undef NXS_SELECT_SPAN
    return paths == 8 ? launch_select<8>(paths_in, width, height, disparities, uniqueness,
                                         disparity, keys, stream)
                      : launch_select<3>(paths_in, width, height, disparities, uniqueness,
                                         disparity, keys, stream);
}

cudaError_t launch_select_sums(const uint16_t *sums, int width, int height, int disparities,
                               float uniqueness, float *disparity, uint32_t *keys,
                               cudaStream_t stream) {
    return launch_select<0>(sums, width, height, disparities, uniqueness, disparity, keys,
                            stream);
}

cudaError_t launch_select_path_sums(const uint16_t *sums, int width, int height,
                                    int disparities, float uniqueness, float *disparity,
                                    uint32_t *keys, cudaStream_t stream) {
    return launch_select<-1, 16>(sums, width, height, disparities, uniqueness, disparity, keys,
                                 stream);
}

// ---------------------------------------------------------------- check
__global__ void __launch_bounds__(256)
    consistency_kernel(const float *__restrict__ disparity, const uint32_t *__restrict__ keys,
                       int width, float *__restrict__ checked) {
    follow_previous_grid();
    extern __shared__ uint32_t right[];
    consistency_row(disparity, keys, width, checked, blockIdx.x, right);
}

cudaError_t launch_consistency(const float *disparity, const uint32_t *keys, int width,
                               int height, float *checked, cudaStream_t stream) {
    return launch_after(consistency_kernel, dim3(height), dim3(256), sizeof(uint32_t) * width,
                        stream, disparity, keys, width, checked);
}

// ---------------------------------------------------------------- median
__global__ void median3_kernel(const float *__restrict__ image, int width, int height,
                               int stage_mask, float *__restrict__ filtered) {
    follow_previous_grid();
    median_at(image, width, height, stage_mask, filtered, blockIdx.x * blockDim.x + threadIdx.x,
              blockIdx.y);
}

cudaError_t launch_median3(const float *image, int width, int height, int stage_mask,
                           float *filtered, cudaStream_t stream) {
    dim3 grid((width + 127) / 128, height);
    return launch_after(median3_kernel, grid, dim3(128), 0, stream, image, width, height,
                        stage_mask, filtered);
}

// ---------------------------------------------------------------- check + median
// The left-right check and the median in one pass over bands of kBandRows
// rows: a block builds, in shared memory, the right maps and the checked
// disparities of its band's rows and of the row above and below (rows
// clamped at the image's edges, as the median replicates them), then filters
// its rows. The per-pixel steps are consistency_row's and median_at's.
constexpr int kBandRows = 1;

size_t check_median_shared_bytes(int width) {
    return (size_t)(kBandRows + 2) * width * (sizeof(uint32_t) + sizeof(float));
}

__global__ void __launch_bounds__(256)
    check_median_kernel(const float *__restrict__ disparity, const uint32_t *__restrict__ keys,
                        int width, int height, int stage_mask, float *__restrict__ filtered) {
    follow_previous_grid();
    extern __shared__ uint32_t band[];
    constexpr int ROWS = kBandRows + 2;
    uint32_t *right = band;                                     // [ROWS][width]
    float *checked = reinterpret_cast<float *>(band + ROWS * width);  // [ROWS][width]
    const int y0 = blockIdx.x * kBandRows;
    for (int i = threadIdx.x; i < ROWS * width; i += blockDim.x) right[i] = kInvalidKey;
    __syncthreads();
    // Keys into the right maps, the disparities kept raw in `checked`: the
    // loads of kCheckChunk columns of every row a thread are issued together,
    // then used. Loops run over rows and columns (no division by the width).
    constexpr int kCheckChunk = 3;
    for (int xb = threadIdx.x; xb < width; xb += kCheckChunk * blockDim.x) {
        uint32_t key[ROWS][kCheckChunk];
        float value[ROWS][kCheckChunk];
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            const size_t row = (size_t)min(max(y0 - 1 + r, 0), height - 1) * width;
#pragma unroll
            for (int k = 0; k < kCheckChunk; ++k) {
                const int x = xb + k * blockDim.x;
                if (x < width) {
                    key[r][k] = __ldcg(keys + row + x);
                    value[r][k] = __ldcg(disparity + row + x);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
#pragma unroll
            for (int k = 0; k < kCheckChunk; ++k) {
                const int x = xb + k * blockDim.x;
                if (x >= width) continue;
                checked[r * width + x] = value[r][k];
                const uint32_t found = key[r][k];
                if (found == kInvalidKey) continue;
                const int winner = (int)(found & 0xFFFFu);
                if (x - winner < 0) continue;  // a winner is at most x (past-edge costs lose)
                atomicMin(&right[r * width + x - winner],
                          (found & 0xFFFF0000u) | (65535u - (uint32_t)winner));
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < ROWS; ++r)
        for (int x = threadIdx.x; x < width; x += blockDim.x)
            checked[r * width + x] =
                consistent_value<false>(checked[r * width + x], x, width, right + r * width);
    __syncthreads();
#pragma unroll
    for (int ry = 0; ry < kBandRows; ++ry) {
        const int y = y0 + ry;
        if (y >= height) break;
        for (int x = threadIdx.x; x < width; x += blockDim.x) {
            float v[9];
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    const int sx = min(max(x + dx, 0), width - 1);
                    v[(dy + 1) * 3 + dx + 1] = checked[(ry + 1 + dy) * width + sx];
                }
            filtered[(size_t)y * width + x] = median_of_nine(v, stage_mask);
        }
    }
}

// cudaFuncSetAttribute on the current device, once per device ordinal.
static cudaError_t allow_check_median_shared() {
    constexpr int kDevices = 64;
    static std::mutex lock;
    static bool allowed[kDevices] = {};
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device < 0 || device >= kDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> guard(lock);
    if (allowed[device]) return cudaSuccess;
    e = cudaFuncSetAttribute(check_median_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)check_median_shared_bytes(4096));
    if (e == cudaSuccess) allowed[device] = true;
    return e;
}

cudaError_t launch_check_median(const float *disparity, const uint32_t *keys, int width,
                                int height, int stage_mask, float *filtered,
                                cudaStream_t stream) {
    const size_t shared = check_median_shared_bytes(width);
    // Wide images need more than the default 48 KB: allowed once per device
    // (the attribute belongs to the device current when it is set), for the widest.
    if (shared > 48 * 1024) {
        const cudaError_t allowed = allow_check_median_shared();
        if (allowed != cudaSuccess) return allowed;
    }
    return launch_after(check_median_kernel, dim3((height + kBandRows - 1) / kBandRows),
                        dim3(256), shared, stream, disparity, keys, width, height, stage_mask,
                        filtered);
}

// ---------------------------------------------------------------- the matcher
static size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

size_t matcher_scratch_bytes(int width, int height, int disparities) {
    const size_t pixels = (size_t)width * height, volume = pixels * disparities;
    return align256(volume) + 8 * align256(volume) + 2 * align256(4 * pixels);
}

MatcherScratch carve_matcher_scratch(void *base, int width, int height, int disparities) {
    const size_t pixels = (size_t)width * height, volume = pixels * disparities;
    char *at = static_cast<char *>(base);
    MatcherScratch s;
    s.costs = reinterpret_cast<uint8_t *>(at);
    at += align256(volume);
    s.paths = reinterpret_cast<uint8_t *>(at);
    at += 8 * align256(volume);
    s.selected = reinterpret_cast<float *>(at);
    at += align256(4 * pixels);
    s.keys = reinterpret_cast<uint32_t *>(at);
    return s;
}

cudaError_t run_matcher_front(const uint8_t *left, const uint8_t *right, int width, int height,
                              int disparities, int paths, int p1, int p2,
                              const MatcherScratch &s, cudaStream_t stream) {
    cudaError_t e;
    // The intermediates are in the permuted order of the path lanes' span
    // (span_disparity).
    const int span = matcher_span(disparities);
    if ((e = launch_census_costs(left, right, width, height, disparities, s.costs, stream, span)))
        return e;
    if (path_sums_wanted(width, height, disparities))  // the aggregate in the path volumes' room
        return launch_paths_sums(s.costs, width, height, disparities, paths, p1, p2,
                                 reinterpret_cast<uint16_t *>(s.paths), stream);
    return launch_paths(s.costs, width, height, disparities, paths, p1, p2, s.paths, stream,
                        span);
}

cudaError_t run_matcher_back(int width, int height, int disparities, int paths,
                             float uniqueness, int stage_mask, const MatcherScratch &s,
                             float *disparity, cudaStream_t stream, bool beside) {
    cudaError_t e;
    if (path_sums_wanted(width, height, disparities))
        e = launch_select_path_sums(reinterpret_cast<const uint16_t *>(s.paths), width, height,
                                    disparities, uniqueness, s.selected, s.keys, stream);
    else
        e = launch_select_paths(s.paths, width, height, disparities, paths, uniqueness,
                                s.selected, s.keys, stream, matcher_span(disparities),
                                beside ? g_lean_select.load() : 0);
    if (e) return e;
    return launch_check_median(s.selected, s.keys, width, height, stage_mask, disparity, stream);
}

cudaError_t run_matcher(const uint8_t *left, const uint8_t *right, int width, int height,
                        int disparities, int paths, int p1, int p2, float uniqueness,
                        int stage_mask, const MatcherScratch &s, float *disparity,
                        cudaStream_t stream, bool beside) {
    const cudaError_t e =
        run_matcher_front(left, right, width, height, disparities, paths, p1, p2, s, stream);
    if (e) return e;
    return run_matcher_back(width, height, disparities, paths, uniqueness, stage_mask, s,
                            disparity, stream, beside);
}

}  // namespace nxs
