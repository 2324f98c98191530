// NxStereo's coarse-to-fine search on B200 (lib/nx_stereo.ex:138-471):
// sgm_coarse_to_fine/3 is sgm/3 on the pair shrunk 2x with 64 disparities,
// each full-size pixel's band base from that coarse match, then sgm_band/4:
// the full-search pipeline with each pixel's candidates limited to the BAND
// disparities base .. base + BAND - 1.
//
// Layout in HBM for a W x H pair (B = BAND):
//   half images  u8  [2][H/2][W/2]  the rounded 2x2 means
//   coarse       f32 [H/2][W/2]     sgm/3 of the half pair (the full-search kernels)
//   base         s32 [H][W]         each pixel's band base, -1 without an estimate
//   codes        u64 [2][H][W]      the fine census of both images
//   costs        u8  [H][W][B]      candidate k = disparity base + k
//   paths        u8  [P][H][W][B]   each direction's band path costs, <= p2 + 48
//   selected f32 [H][W], keys u32 [H][W]; the check and median write the output.
//
// The band path scan keeps, per scan line, the previous pixel's normalised
// costs as u16 values in a row of shared memory padded with p2 on both sides:
// moving them to this pixel's band (by base - previous base) is a read of the
// row at that offset, and candidates outside the previous band read p2.
#include <algorithm>
#include <cstdio>

#include "nxs_kernels.h"
#include "nxs_matcher.cuh"

namespace nxs {

// ---------------------------------------------------------------- shrink
// Both images' rounded 2x2 means, (sum + 2) / 4 (lib/nx_stereo.ex:227-238).
__global__ void shrink_pair_kernel(const uint8_t *__restrict__ left,
                                   const uint8_t *__restrict__ right, int width, int height,
                                   uint8_t *__restrict__ left_half,
                                   uint8_t *__restrict__ right_half) {
    follow_previous_grid();
    const int hw = width / 2, hh = height / 2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hw * hh) return;
    const int x = i % hw, y = i / hw;
    const size_t at = (size_t)(2 * y) * width + 2 * x;
    for (int image = 0; image < 2; ++image) {
        const uint8_t *src = image ? right : left;
        const int sum = src[at] + src[at + 1] + src[at + width] + src[at + width + 1];
        (image ? right_half : left_half)[i] = (uint8_t)((sum + 2) / 4);
    }
}

// ---------------------------------------------------------------- band bases
// A thread per coarse pixel: the lowest match (>= 0) in its 3x3
// neighbourhood, doubled, floored, less the margin, clipped to
// 0..128 - band, written to its 2x2 block; -1 where there is none
// (lib/nx_stereo.ex:240-254). f32 steps as the reference's: exact here.
__global__ void band_base_kernel(const float *__restrict__ coarse, int coarse_width,
                                 int coarse_height, int band, int margin,
                                 int32_t *__restrict__ base) {
    follow_previous_grid();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= coarse_width * coarse_height) return;
    const int cx = i % coarse_width, cy = i / coarse_width;
    const float none = 1.0e9f;
    float lowest = none;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const int x = cx + dx, y = cy + dy;
            if (x < 0 || x >= coarse_width || y < 0 || y >= coarse_height) continue;
            const float v = coarse[y * coarse_width + x];
            if (v >= 0.0f && v < lowest) lowest = v;
        }
    const float start = fsub(floorf(fmul(lowest, 2.0f)), (float)margin);
    const int value = lowest < none ? min(max((int)start, 0), 128 - band) : -1;
    const int width = 2 * coarse_width;
    const size_t at = (size_t)(2 * cy) * width + 2 * cx;
    base[at] = value;
    base[at + 1] = value;
    base[at + width] = value;
    base[at + width + 1] = value;
}

// ---------------------------------------------------------------- dense census
// The dense 9x5 window (dy -2..2, dx -4..4 but the centre, row-major bit
// order), its anchor the centre or, BLEND, the centre's rounded average with
// its 3x3 Gaussian mean: (1-2-1 x 1-2-1 weighted sum + 16 centre + 24) / 32
// (lib/nx_stereo.ex:491-526). A block of 128 threads takes 128 pixels of a
// row from a staged window of 5 rows x 136 columns (borders replicated).
template <bool BLEND>
__global__ void __launch_bounds__(128)
    census_dense_kernel(const uint8_t *__restrict__ left, const uint8_t *__restrict__ right,
                        int width, int height, uint64_t *__restrict__ left_codes,
                        uint64_t *__restrict__ right_codes) {
    constexpr int PITCH = 128 + 8, ROWS = 5;
    __shared__ uint8_t window[ROWS][PITCH];
    follow_previous_grid();
    const uint8_t *image = blockIdx.z ? right : left;
    uint64_t *codes = blockIdx.z ? right_codes : left_codes;
    const int x0 = blockIdx.x * 128, y = blockIdx.y;
    for (int i = threadIdx.x; i < ROWS * PITCH; i += 128) {
        const int r = i / PITCH, c = i % PITCH;
        const int sy = min(max(y + r - 2, 0), height - 1);
        const int sx = min(max(x0 + c - 4, 0), width - 1);
        window[r][c] = __ldg(image + (size_t)sy * width + sx);
    }
    __syncthreads();
    const int x = x0 + threadIdx.x;
    if (x >= width) return;
    const int c = threadIdx.x + 4;
    int anchor = window[2][c];
    if (BLEND) {
        const int weighted = window[1][c - 1] + 2 * window[1][c] + window[1][c + 1] +
                             2 * window[2][c - 1] + 4 * window[2][c] + 2 * window[2][c + 1] +
                             window[3][c - 1] + 2 * window[3][c] + window[3][c + 1];
        anchor = (weighted + 16 * anchor + 24) / 32;
    }
    uint64_t code = 0;
    int bit = 0;
#pragma unroll
    for (int r = 0; r < ROWS; ++r)
#pragma unroll
        for (int dx = -4; dx <= 4; ++dx) {
            if (r == 2 && dx == 0) continue;
            if ((int)window[r][c + dx] + 1 < anchor) code |= (uint64_t)1 << bit;
            ++bit;
        }
    codes[(size_t)y * width + x] = code;
}

// ---------------------------------------------------------------- band costs
// A thread per pixel: costs[y][x][k] = popcount(left[y][x] ^ right[y][x - b - k])
// with b = max(base, 0) and right codes left of the image zero
// (lib/nx_stereo.ex:362-383), written BAND bytes at a time in 16-byte stores.
template <int BAND>
__global__ void __launch_bounds__(128)
    band_costs_kernel(const uint64_t *__restrict__ left_codes,
                      const uint64_t *__restrict__ right_codes, const int32_t *__restrict__ base,
                      int width, int height, uint8_t *__restrict__ costs) {
    follow_previous_grid();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= width) return;
    const size_t pixel = (size_t)y * width + x;
    const int b = max(__ldg(base + pixel), 0);
    const uint64_t code = __ldg(left_codes + pixel);
    const uint64_t *row = right_codes + (size_t)y * width;
    uint32_t packed[BAND / 4];
#pragma unroll
    for (int w = 0; w < BAND / 4; ++w) {
        uint32_t word = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int column = x - b - (4 * w + j);
            const uint64_t feature = column >= 0 ? __ldg(row + column) : 0ull;
            word |= (uint32_t)__popcll(code ^ feature) << (8 * j);
        }
        packed[w] = word;
    }
    uint4 *out = reinterpret_cast<uint4 *>(costs + pixel * BAND);
    if constexpr (BAND >= 16) {
#pragma unroll
        for (int q = 0; q < BAND / 16; ++q)
            out[q] = make_uint4(packed[4 * q], packed[4 * q + 1], packed[4 * q + 2],
                                packed[4 * q + 3]);
    } else {
        *reinterpret_cast<uint2 *>(costs + pixel * BAND) = make_uint2(packed[0], packed[1]);
    }
}

// ---------------------------------------------------------------- band paths
// The band recurrence along every scan line (lib/nx_stereo.ex:385-454): at
// pixel (y, x) with base b, continuing from the pixel before with base b',
// window[j] = the previous normalised cost of candidate j - 1 + b - b', p2
// where the previous band lacks it; L[k] = min(min(window[k + 1], p2),
// min(window[k], window[k + 2]) + p1) + C[k]. A line entering the image
// starts from zero in its own band. G = BAND / V lanes follow a line, each
// with V candidates as V / 2 u16x2 words; a warp follows 32 / G lines.
template <int BAND, int V>
struct BandRow {
    static constexpr int PAD = BAND + 4;             // u16 values of p2 each side
    static constexpr int ELEMENTS = BAND + 2 * PAD;  // of a line's row
    static constexpr int WORDS = ELEMENTS / 2;       // u32 words of a row
};

template <int BAND, int V>
__global__ void __launch_bounds__(32)
    band_paths_kernel(const uint8_t *__restrict__ costs, const int32_t *__restrict__ base,
                      uint8_t *__restrict__ out, const PathSetup s) {
    constexpr int G = BAND / V, WORDS = V / 2, LINES = 32 / G;
    using Row = BandRow<BAND, V>;
    static_assert(Row::PAD % 2 == 0 && V % 4 == 0, "rows of whole words");
    __shared__ uint32_t rows[LINES][Row::WORDS];
    follow_previous_grid();
    const int lane = threadIdx.x, member = lane % G, slot_line = lane / G;
    uint32_t *row = rows[slot_line];
    const uint32_t p1x2 = (uint32_t)s.p1 * 0x10001u, p2x2 = (uint32_t)s.p2 * 0x10001u;
    // pads of p2, the band's middle zero (a line starts from zero)
    for (int w = member; w < Row::WORDS; w += G) {
        const int e = 2 * w;
        row[w] = (e >= Row::PAD && e < Row::PAD + BAND) ? 0u : p2x2;
    }

    // this warp's direction and line, as the full search assigns them
    const int warp = blockIdx.x;
    int slot = 0;
    while (warp >= s.first_warp[slot + 1]) ++slot;
    int p, group;
    if (slot < s.straight) {
        p = s.order[slot];
        group = warp - s.first_warp[slot];
    } else {
        const int w = warp - s.first_warp[s.straight];
        const int diagonals = s.paths - s.straight;
        p = s.order[s.straight + w % diagonals];
        group = w / diagonals;
    }
    const int dy = s.dy[p], dx = s.dx[p], W = s.width, H = s.height;
    const int rank = group * LINES + slot_line;
    int y0 = 0, x0 = 0, length = 0;
    if (rank < s.lines[p]) length = line_start(ranked_line(rank, dy, dx, W, H), dy, dx, W, H, &y0, &x0);
    const int steps = (int)__reduce_max_sync(kFullMask, (unsigned)length);
    const ptrdiff_t step_pixels = (ptrdiff_t)dy * W + dx;
    size_t pixel = (size_t)y0 * W + x0;
    uint8_t *const volume = out + (size_t)p * s.volume;

    uint32_t r[WORDS];
#pragma unroll
    for (int k = 0; k < WORDS; ++k) r[k] = 0u;
    uint32_t m2 = 0;
    int previous_base = 0;
    // the first step's base and costs
    int b = length > 0 ? max(__ldg(base + pixel), 0) : 0;
    using Chunk = typename std::conditional<V == 16, uint4,
                                            typename std::conditional<V == 8, uint2, uint32_t>::type>::type;
    Chunk cost_chunk{};
    if (length > 0) cost_chunk = __ldg(reinterpret_cast<const Chunk *>(costs + pixel * BAND + member * V));
    __syncwarp();
    for (int step = 0; step < steps; ++step) {
        const bool valid = step < length;
        // prefetch the next step's base and costs
        const size_t next_pixel = pixel + step_pixels;
        int next_b = 0;
        Chunk next_chunk{};
        if (step + 1 < length) {
            next_b = max(__ldg(base + next_pixel), 0);
            next_chunk = __ldg(reinterpret_cast<const Chunk *>(costs + next_pixel * BAND + member * V));
        }
        const int delta = step == 0 ? 0 : min(max(b - previous_base, -(BAND + 1)), BAND + 1);
        // the window: row elements from PAD + member * V - 1 + delta, V + 2 of them
        const int first = Row::PAD + member * V - 1 + delta;
        const int word0 = first >> 1;
        const unsigned shift = (unsigned)(first & 1) * 16u;
        uint32_t loaded[WORDS + 2];
#pragma unroll
        for (int i = 0; i < WORDS + 2; ++i) loaded[i] = row[word0 + i];
        uint32_t even[WORDS + 1];  // even[m] = (window[2m], window[2m + 1])
#pragma unroll
        for (int i = 0; i < WORDS + 1; ++i) even[i] = __funnelshift_r(loaded[i], loaded[i + 1], shift);
        uint32_t cost[WORDS];
        {
            const uint32_t *c = reinterpret_cast<const uint32_t *>(&cost_chunk);
#pragma unroll
            for (int i = 0; i < V / 4; ++i) {
                cost[2 * i] = __byte_perm(c[i], 0, 0x4140);
                cost[2 * i + 1] = __byte_perm(c[i], 0, 0x4342);
            }
        }
#pragma unroll
        for (int k = 0; k < WORDS; ++k) {
            const uint32_t own = __byte_perm(even[k], even[k + 1], 0x5432);  // (window[2k+1], window[2k+2])
            const uint32_t neighbour = vmin2(even[k], even[k + 1]) + p1x2;
            r[k] = __vimin3_u16x2(own, p2x2, neighbour) + cost[k];
        }
        if (valid) {
            Chunk packed;
            uint32_t *words = reinterpret_cast<uint32_t *>(&packed);
#pragma unroll
            for (int i = 0; i < V / 4; ++i) words[i] = __byte_perm(r[2 * i], r[2 * i + 1], 0x6420);
            *reinterpret_cast<Chunk *>(volume + pixel * BAND + member * V) = packed;
        }
        // the line's lowest cost, then its normalised costs into the row
        uint32_t lowest = r[0];
#pragma unroll
        for (int k = 1; k < WORDS; ++k) lowest = vmin2(lowest, r[k]);
        lowest = vmin2(lowest, __byte_perm(lowest, 0, 0x1032));
        m2 = line_minimum<G>(lowest);
        __syncwarp();  // every lane has read the row
#pragma unroll
        for (int k = 0; k < WORDS; ++k) row[(Row::PAD + member * V) / 2 + k] = r[k] - m2;
        __syncwarp();
        previous_base = b;
        b = next_b;
        cost_chunk = next_chunk;
        pixel = next_pixel;
    }
}

// ---------------------------------------------------------------- band select
// A thread per pixel: the sum of the path volumes over the pixel's band, the
// winner (ties low) with disparities past x raised by 0x8000, the second best
// outside k - 1..k + 1, acceptance (a base >= 0, winner base + k <= x, the
// uniqueness test) and the subpixel step in the reference's f32 order
// (lib/nx_stereo.ex:429-469); keys (cost << 16) | (base + k).
template <int BAND, int PATHS>
__global__ void __launch_bounds__(128)
    band_select_kernel(const uint8_t *__restrict__ paths_in, const int32_t *__restrict__ base,
                       int width, int height, int disparities, size_t volume, float uniqueness,
                       float *__restrict__ disparity, uint32_t *__restrict__ keys) {
    follow_previous_grid();
    const size_t pixel = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= (size_t)width * height) return;
    const int x = (int)(pixel % (size_t)width);
    const int raw_base = __ldg(base + pixel);
    const int b = max(raw_base, 0);
    uint32_t sums[BAND / 2];  // (k, k + 1) pairs
#pragma unroll
    for (int i = 0; i < BAND / 2; ++i) sums[i] = 0;
#pragma unroll
    for (int p = 0; p < PATHS; ++p) {
        const uint8_t *at = paths_in + p * volume + pixel * BAND;
#pragma unroll
        for (int q = 0; q < BAND / 8; ++q) {
            const uint2 c = __ldcs(reinterpret_cast<const uint2 *>(at + 8 * q));
            sums[4 * q] += __byte_perm(c.x, 0, 0x4140);
            sums[4 * q + 1] += __byte_perm(c.x, 0, 0x4342);
            sums[4 * q + 2] += __byte_perm(c.y, 0, 0x4140);
            sums[4 * q + 3] += __byte_perm(c.y, 0, 0x4342);
        }
    }
    uint32_t values[BAND];
#pragma unroll
    for (int k = 0; k < BAND; ++k)
        values[k] = ((k % 2) ? (sums[k / 2] >> 16) : (sums[k / 2] & 0xFFFFu)) +
                    (b + k > x ? 0x8000u : 0u);
    uint32_t minimum = values[0];
    int winner = 0;
#pragma unroll
    for (int k = 1; k < BAND; ++k)
        if (values[k] < minimum) {
            minimum = values[k];
            winner = k;
        }
    uint32_t second = 0xFFFFFFFFu;
    uint32_t lower = 0, upper = 0;
#pragma unroll
    for (int k = 0; k < BAND; ++k) {
        if (k < winner - 1 || k > winner + 1) second = min(second, values[k]);
        if (k == max(winner - 1, 0)) lower = values[k];
        if (k == min(winner + 1, BAND - 1)) upper = values[k];
    }
    const float lower_f = (float)lower, upper_f = (float)upper, minimum_f = (float)minimum;
    const float second_f = second == 0xFFFFFFFFu ? 2147483647.0f : (float)second;
    const int winner_d = b + winner;
    const bool accepted = raw_base >= 0 && winner_d <= x && second_f > fmul(minimum_f, uniqueness);
    const float denominator = fsub(fadd(lower_f, upper_f), fmul(2.0f, minimum_f));
    const float bounded = denominator > 1.0f ? denominator : 1.0f;
    float correction = fdiv(fsub(lower_f, upper_f), fmul(2.0f, bounded));
    correction = correction < -0.5f ? -0.5f : (correction > 0.5f ? 0.5f : correction);
    const bool refine = denominator > 0.0f && winner > 0 && winner < BAND - 1 &&
                        winner_d < min(disparities - 1, x);
    const float value = fadd((float)winner_d, refine ? correction : 0.0f);
    disparity[pixel] = accepted ? value : -1.0f;
    keys[pixel] = accepted ? ((minimum << 16) | (uint32_t)winner_d) : kInvalidKey;
}

// ---------------------------------------------------------------- launchers
cudaError_t launch_shrink_pair(const uint8_t *left, const uint8_t *right, int width, int height,
                               uint8_t *left_half, uint8_t *right_half, cudaStream_t stream) {
    const int n = (width / 2) * (height / 2);
    return launch_after(shrink_pair_kernel, dim3((n + 255) / 256), dim3(256), 0, stream, left,
                        right, width, height, left_half, right_half);
}

cudaError_t launch_band_base(const float *coarse, int coarse_width, int coarse_height, int band,
                             int margin, int32_t *base, cudaStream_t stream) {
    const int n = coarse_width * coarse_height;
    return launch_after(band_base_kernel, dim3((n + 255) / 256), dim3(256), 0, stream, coarse,
                        coarse_width, coarse_height, band, margin, base);
}

cudaError_t launch_census_window(const uint8_t *left, const uint8_t *right, int width,
                                 int height, int window, uint64_t *left_codes,
                                 uint64_t *right_codes, cudaStream_t stream) {
    if (window == 0)
        return launch_census(left, right, width, height, left_codes, right_codes, stream);
    const dim3 grid((width + 127) / 128, height, 2);
    return window == 2 ? launch_after(census_dense_kernel<true>, grid, dim3(128), 0, stream, left,
                                      right, width, height, left_codes, right_codes)
                       : launch_after(census_dense_kernel<false>, grid, dim3(128), 0, stream,
                                      left, right, width, height, left_codes, right_codes);
}

cudaError_t launch_band_costs(const uint64_t *left_codes, const uint64_t *right_codes,
                              const int32_t *base, int width, int height, int band,
                              uint8_t *costs, cudaStream_t stream) {
    const dim3 grid((width + 127) / 128, height);
#define NXS_BAND_COSTS(B)                                                                      \
    launch_after(band_costs_kernel<B>, grid, dim3(128), 0, stream, left_codes, right_codes,   \
                 base, width, height, costs)
    switch (band) {
    case 8: return NXS_BAND_COSTS(8);
    case 16: return NXS_BAND_COSTS(16);
    case 32: return NXS_BAND_COSTS(32);
    case 64: return NXS_BAND_COSTS(64);
    default: return cudaErrorInvalidValue;
    }
#undef NXS_BAND_COSTS
}

// Candidates a lane of the band scan holds: 4 for bands 8 and 16, 8 above.
int band_lane_values(int band) { return band <= 16 ? 4 : 8; }

cudaError_t launch_band_paths(const uint8_t *costs, const int32_t *base, int width, int height,
                              int band, int paths, int p1, int p2, uint8_t *out,
                              cudaStream_t stream) {
    const int v = band_lane_values(band);
    PathSetup s;
    const int total = path_setup(width, height, band, paths, p1, p2, band / v, &s);
#define NXS_BAND_PATHS(B, VV)                                                                  \
    launch_after(band_paths_kernel<B, VV>, dim3(total), dim3(32), 0, stream, costs, base, out, s)
    switch (band) {
    case 8: return NXS_BAND_PATHS(8, 4);
    case 16: return NXS_BAND_PATHS(16, 4);
    case 32: return NXS_BAND_PATHS(32, 8);
    case 64: return NXS_BAND_PATHS(64, 8);
    default: return cudaErrorInvalidValue;
    }
#undef NXS_BAND_PATHS
}

cudaError_t launch_band_select(const uint8_t *paths_in, const int32_t *base, int width,
                               int height, int band, int paths, int disparities, float uniqueness,
                               float *disparity, uint32_t *keys, cudaStream_t stream) {
    const size_t pixels = (size_t)width * height, volume = pixels * band;
    const dim3 grid((unsigned)((pixels + 127) / 128));
#define NXS_BAND_SELECT(B, P)                                                                  \
    launch_after(band_select_kernel<B, P>, grid, dim3(128), 0, stream, paths_in, base, width,   \
                 height, disparities, volume, uniqueness, disparity, keys)
#define NXS_BAND_SELECT_PATHS(B) return paths == 8 ? NXS_BAND_SELECT(B, 8) : NXS_BAND_SELECT(B, 3)
    switch (band) {
    case 8: NXS_BAND_SELECT_PATHS(8);
    case 16: NXS_BAND_SELECT_PATHS(16);
    case 32: NXS_BAND_SELECT_PATHS(32);
    case 64: NXS_BAND_SELECT_PATHS(64);
    default: return cudaErrorInvalidValue;
    }
#undef NXS_BAND_SELECT_PATHS
#undef NXS_BAND_SELECT
}

// ---------------------------------------------------------------- the searches
namespace {
size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }
}  // namespace

size_t band_scratch_bytes(int width, int height, int band) {
    const size_t px = (size_t)width * height;
    return 2 * align256(8 * px) + align256(4 * px) + align256(px * band) +
           8 * align256(px * band) + 2 * align256(4 * px);
}

BandScratch carve_band_scratch(void *base_ptr, int width, int height, int band) {
    const size_t px = (size_t)width * height;
    char *at = static_cast<char *>(base_ptr);
    BandScratch s;
    s.left_codes = reinterpret_cast<uint64_t *>(at);
    at += align256(8 * px);
    s.right_codes = reinterpret_cast<uint64_t *>(at);
    at += align256(8 * px);
    s.base = reinterpret_cast<int32_t *>(at);
    at += align256(4 * px);
    s.costs = reinterpret_cast<uint8_t *>(at);
    at += align256(px * band);
    s.paths = reinterpret_cast<uint8_t *>(at);
    at += 8 * align256(px * band);
    s.selected = reinterpret_cast<float *>(at);
    at += align256(4 * px);
    s.keys = reinterpret_cast<uint32_t *>(at);
    return s;
}

size_t coarse_to_fine_scratch_bytes(int width, int height, int band) {
    const int hw = width / 2, hh = height / 2;
    const size_t half = (size_t)hw * hh;
    return band_scratch_bytes(width, height, band) + 2 * align256(half) + align256(4 * half) +
           matcher_scratch_bytes(hw, hh, 64);
}

cudaError_t run_band_matcher(const uint8_t *left, const uint8_t *right, const int32_t *base,
                             int width, int height, int disparities, int paths, int band,
                             int window, int p1, int p2, float uniqueness, int stage_mask,
                             const BandScratch &s, float *disparity, cudaStream_t stream) {
    cudaError_t e;
    if ((e = launch_census_window(left, right, width, height, window, s.left_codes,
                                  s.right_codes, stream)) ||
        (e = launch_band_costs(s.left_codes, s.right_codes, base, width, height, band, s.costs,
                               stream)) ||
        (e = launch_band_paths(s.costs, base, width, height, band, paths, p1, p2, s.paths,
                               stream)) ||
        (e = launch_band_select(s.paths, base, width, height, band, paths, disparities,
                                uniqueness, s.selected, s.keys, stream)))
        return e;
    return launch_check_median(s.selected, s.keys, width, height, stage_mask, disparity, stream);
}

cudaError_t run_coarse_to_fine(const uint8_t *left, const uint8_t *right, int width, int height,
                               int paths, int coarse_paths, int band, int margin, int window,
                               int p1, int p2, float uniqueness, int stage_mask, void *scratch,
                               float *disparity, int32_t *base_out, cudaStream_t stream) {
    const int hw = width / 2, hh = height / 2;
    const size_t half = (size_t)hw * hh;
    BandScratch s = carve_band_scratch(scratch, width, height, band);
    char *at = static_cast<char *>(scratch) + band_scratch_bytes(width, height, band);
    uint8_t *left_half = reinterpret_cast<uint8_t *>(at);
    at += align256(half);
    uint8_t *right_half = reinterpret_cast<uint8_t *>(at);
    at += align256(half);
    float *coarse = reinterpret_cast<float *>(at);
    at += align256(4 * half);
    MatcherScratch coarse_scratch = carve_matcher_scratch(at, hw, hh, 64);
    int32_t *base = base_out ? base_out : s.base;
    cudaError_t e;
    if ((e = launch_shrink_pair(left, right, width, height, left_half, right_half, stream)) ||
        (e = run_matcher(left_half, right_half, hw, hh, 64, coarse_paths, p1, p2, uniqueness, 0,
                         coarse_scratch, coarse, stream)) ||
        (e = launch_band_base(coarse, hw, hh, band, margin, base, stream)))
        return e;
    return run_band_matcher(left, right, base, width, height, 128, paths, band, window, p1, p2,
                            uniqueness, stage_mask, s, disparity, stream);
}

}  // namespace nxs
