// The full-search matcher of NxStereo.sgm/3 on B200: census, the u8 Hamming
// cost volume, the path recurrence along every scan line, selection, the
// left-right check and the median.
//
// Layout in HBM for a W x H pair and D disparities (D a multiple of 16):
//   codes      u64 [2][H][W]     48-bit census codes of both images
//   costs      u8  [H][W][D]     Hamming costs, 0..48
//   paths      u8  [P][H][W][D]  each direction's path costs, 0..p2+48 <= 127
//   selected   f32 [H][W], keys u32 [H][W], checked f32 [H][W]
// Disparities are the fastest axis so that one scan-line step reads and
// writes D contiguous bytes: one coalesced 128-byte transaction per warp at
// D = 128.
#include <algorithm>

#include "nxs_device.cuh"
#include "nxs_kernels.h"

namespace nxs {

// ---------------------------------------------------------------- census
// 9x7 sparse census (lib/nx_stereo.ex:491-505): bit i for the i-th neighbour
// in row-major order over dy in -3..3, dx in -4..4, both non-zero, set where
// neighbour + 1 < centre; borders replicated (lib/nx_stereo/image.ex:508-537).
// A 32x8 block stages its window of 40x14 pixels in shared memory.
constexpr int kCensusX = 32, kCensusY = 8;

__global__ void __launch_bounds__(kCensusX *kCensusY)
    census_kernel(const uint8_t *__restrict__ left, const uint8_t *__restrict__ right, int width,
                  int height, uint64_t *__restrict__ left_codes,
                  uint64_t *__restrict__ right_codes) {
    __shared__ uint8_t tile[kCensusY + 6][kCensusX + 8];
    const uint8_t *image = blockIdx.z == 0 ? left : right;
    uint64_t *codes = blockIdx.z == 0 ? left_codes : right_codes;
    const int x0 = blockIdx.x * kCensusX, y0 = blockIdx.y * kCensusY;
    const int tid = threadIdx.y * kCensusX + threadIdx.x;
    for (int i = tid; i < (kCensusY + 6) * (kCensusX + 8); i += kCensusX * kCensusY) {
        int ty = i / (kCensusX + 8), tx = i % (kCensusX + 8);
        int sy = min(max(y0 + ty - 3, 0), height - 1);
        int sx = min(max(x0 + tx - 4, 0), width - 1);
        tile[ty][tx] = image[(size_t)sy * width + sx];
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= width || y >= height) return;
    const int centre = tile[threadIdx.y + 3][threadIdx.x + 4];
    uint64_t code = 0;
    int bit = 0;
#pragma unroll
    for (int dy = -3; dy <= 3; ++dy) {
        if (dy == 0) continue;
#pragma unroll
        for (int dx = -4; dx <= 4; ++dx) {
            if (dx == 0) continue;
            int n = tile[threadIdx.y + 3 + dy][threadIdx.x + 4 + dx];
            code |= (uint64_t)(n + 1 < centre) << bit;
            ++bit;
        }
    }
    codes[(size_t)y * width + x] = code;
}

cudaError_t launch_census(const uint8_t *left, const uint8_t *right, int width, int height,
                          uint64_t *left_codes, uint64_t *right_codes, cudaStream_t stream) {
    dim3 block(kCensusX, kCensusY);
    dim3 grid((width + kCensusX - 1) / kCensusX, (height + kCensusY - 1) / kCensusY,
              right ? 2 : 1);
    census_kernel<<<grid, block, 0, stream>>>(left, right, width, height, left_codes,
                                              right_codes);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- costs
// costs[y][x][d] = popcount(left[y][x] ^ right[y][x - d]), right codes left of
// the image zero (lib/nx_stereo.ex:528-542). A block covers 32 pixels of a
// row; it stages their left codes and the D + 31 right codes they reach, then
// writes the block's 32 x D bytes with 16-byte stores.
constexpr int kCostPixels = 32;

__global__ void __launch_bounds__(128)
    costs_kernel(const uint64_t *__restrict__ left_codes, const uint64_t *__restrict__ right_codes,
                 int width, int disparities, uint8_t *__restrict__ costs) {
    extern __shared__ uint64_t staged[];
    uint64_t *lefts = staged;
    uint64_t *rights = staged + kCostPixels;
    const int x0 = blockIdx.x * kCostPixels, y = blockIdx.y;
    const size_t row = (size_t)y * width;
    for (int i = threadIdx.x; i < kCostPixels; i += blockDim.x)
        lefts[i] = x0 + i < width ? left_codes[row + x0 + i] : 0;
    for (int i = threadIdx.x; i < kCostPixels + disparities - 1; i += blockDim.x) {
        int x = x0 - (disparities - 1) + i;
        rights[i] = (x >= 0 && x < width) ? right_codes[row + x] : 0;
    }
    __syncthreads();
    const int pixels = min(kCostPixels, width - x0);
    const int chunks = disparities / 16;
    for (int c = threadIdx.x; c < pixels * chunks; c += blockDim.x) {
        const int p = c / chunks, d0 = (c % chunks) * 16;
        const uint64_t l = lefts[p];
        // right code of pixel x0 + p at disparity d: rights[p - d + D - 1]
        const uint64_t *r = rights + p + disparities - 1 - d0;
        uint32_t words[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t b0 = __popcll(l ^ r[-(4 * q + 0)]);
            uint32_t b1 = __popcll(l ^ r[-(4 * q + 1)]);
            uint32_t b2 = __popcll(l ^ r[-(4 * q + 2)]);
            uint32_t b3 = __popcll(l ^ r[-(4 * q + 3)]);
            words[q] = b0 | (b1 << 8) | (b2 << 16) | (b3 << 24);
        }
        *reinterpret_cast<uint4 *>(costs + (row + x0 + p) * disparities + d0) =
            make_uint4(words[0], words[1], words[2], words[3]);
    }
}

cudaError_t launch_costs(const uint64_t *left_codes, const uint64_t *right_codes, int width,
                         int height, int disparities, uint8_t *costs, cudaStream_t stream) {
    dim3 grid((width + kCostPixels - 1) / kCostPixels, height);
    size_t shared = sizeof(uint64_t) * (2 * kCostPixels + disparities - 1);
    costs_kernel<<<grid, 128, shared, stream>>>(left_codes, right_codes, width, disparities,
                                                costs);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- paths
// libSGM's normalised recurrence (lib/nx_stereo.ex:575-606) along every scan
// line of every direction, one warp per line. Lane l holds disparities
// l*DPL .. l*DPL + DPL - 1 as u16x2 words, unnormalised:
//   L[d] = min(prev[d], prev[d-1] + p1, prev[d+1] + p1, m + p2) - m + C[d],
//   m = min over d of prev,
// which equals the reference's min(min(a, p2), min(a[d-1], a[d+1]) + p1) + C
// with a = prev - m; its out-of-range neighbours (p2 - p1, so p2 once p1 is
// added) never beat m + p2, so they read as +inf here. Lanes past D hold +inf.
// A path starts from zero where it enters the image, so its first step is C.
// The costs of the next kPrefetch steps are in flight while a step computes.
constexpr int kPrefetch = 4;

struct PathSetup {
    int width, height, disparities, p1, p2, paths;
    int first_warp[9];  // first warp of each direction; first_warp[paths] = total
    int dy[8], dx[8];
    size_t volume;      // bytes of one direction's volume
};

template <int DPL>
struct Chunk;
template <>
struct Chunk<2> {
    using T = uint16_t;
    static __device__ __forceinline__ void unpack(T c, uint32_t *w) {
        w[0] = __byte_perm((uint32_t)c, 0, 0x4140);
    }
    static __device__ __forceinline__ T pack(const uint32_t *w) {
        return (T)__byte_perm(w[0], 0, 0x4420);
    }
    static __device__ __forceinline__ T zero() { return 0; }
};
template <>
struct Chunk<4> {
    using T = uint32_t;
    static __device__ __forceinline__ void unpack(T c, uint32_t *w) {
        w[0] = __byte_perm(c, 0, 0x4140);
        w[1] = __byte_perm(c, 0, 0x4342);
    }
    static __device__ __forceinline__ T pack(const uint32_t *w) {
        return __byte_perm(w[0], w[1], 0x6420);
    }
    static __device__ __forceinline__ T zero() { return 0; }
};
template <>
struct Chunk<8> {
    using T = uint2;
    static __device__ __forceinline__ void unpack(T c, uint32_t *w) {
        w[0] = __byte_perm(c.x, 0, 0x4140);
        w[1] = __byte_perm(c.x, 0, 0x4342);
        w[2] = __byte_perm(c.y, 0, 0x4140);
        w[3] = __byte_perm(c.y, 0, 0x4342);
    }
    static __device__ __forceinline__ T pack(const uint32_t *w) {
        return make_uint2(__byte_perm(w[0], w[1], 0x6420), __byte_perm(w[2], w[3], 0x6420));
    }
    static __device__ __forceinline__ T zero() { return make_uint2(0, 0); }
};

template <int DPL>
__global__ void __launch_bounds__(128)
    paths_kernel(const uint8_t *__restrict__ costs, uint8_t *__restrict__ paths_out,
                 const PathSetup s) {
    using C = Chunk<DPL>;
    using T = typename C::T;
    constexpr int R = DPL / 2;  // u16x2 words per lane
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= s.first_warp[s.paths]) return;  // the whole warp leaves together
    int p = 0;
    while (warp >= s.first_warp[p + 1]) ++p;
    const int line = warp - s.first_warp[p];
    const int dy = s.dy[p], dx = s.dx[p];
    const int W = s.width, H = s.height;
    int y0, x0, length;
    if (dy == 0) {  // along a row
        y0 = line;
        x0 = dx > 0 ? 0 : W - 1;
        length = W;
    } else if (dx == 0) {  // down or up a column
        x0 = line;
        y0 = dy > 0 ? 0 : H - 1;
        length = H;
    } else {  // a diagonal, entering from the first row it meets or from a side
        if (line < W) {
            x0 = line;
            y0 = dy > 0 ? 0 : H - 1;
        } else {
            x0 = dx > 0 ? 0 : W - 1;
            int k = line - W + 1;
            y0 = dy > 0 ? k : H - 1 - k;
        }
        int rows = dy > 0 ? H - y0 : y0 + 1;
        int columns = dx > 0 ? W - x0 : x0 + 1;
        length = min(rows, columns);
    }
    const int D = s.disparities;
    const bool active = lane * DPL < D;
    const ptrdiff_t stride = ((ptrdiff_t)dy * W + dx) * D;
    const uint8_t *src = costs + ((size_t)y0 * W + x0) * D + lane * DPL;
    uint8_t *dst = paths_out + (size_t)p * s.volume + ((size_t)y0 * W + x0) * D + lane * DPL;

    uint32_t r[R];
#pragma unroll
    for (int k = 0; k < R; ++k) r[k] = active ? 0u : kInf2;
    uint32_t m2 = 0, j2 = (uint32_t)s.p2 * 0x10001u;
    const uint32_t p1x2 = (uint32_t)s.p1 * 0x10001u;

    T ring[kPrefetch];
#pragma unroll
    for (int i = 0; i < kPrefetch; ++i)
        ring[i] = (active && i < length) ? __ldg(reinterpret_cast<const T *>(src + i * stride))
                                         : C::zero();

    for (int base = 0; base < length; base += kPrefetch) {
#pragma unroll
        for (int i = 0; i < kPrefetch; ++i) {
            const int step = base + i;
            if (step >= length) break;  // uniform across the warp
            const T c = ring[i];
            const int ahead = step + kPrefetch;
            ring[i] = (active && ahead < length)
                          ? __ldg(reinterpret_cast<const T *>(src + ahead * stride))
                          : C::zero();
            uint32_t cost[R];
            C::unpack(c, cost);
            uint32_t from_left = __shfl_up_sync(kFullMask, r[R - 1], 1);
            uint32_t from_right = __shfl_down_sync(kFullMask, r[0], 1);
            if (lane == 0) from_left = kInf2;
            if (lane == 31) from_right = kInf2;
            uint32_t shifted[R + 1];  // shifted[k] = (d-1) values of word k
            shifted[0] = __byte_perm(from_left, r[0], 0x5432);
#pragma unroll
            for (int k = 1; k < R; ++k) shifted[k] = __byte_perm(r[k - 1], r[k], 0x5432);
            shifted[R] = __byte_perm(r[R - 1], from_right, 0x5432);
            uint32_t lowest = kInf2;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                uint32_t neighbour = vmin2(shifted[k], shifted[k + 1]);
                uint32_t t = vmin2(r[k], j2);
                t = __viaddmin_u16x2(neighbour, p1x2, t);
                // t >= m in both halves, so the subtraction borrows nowhere.
                uint32_t value = t - m2 + cost[k];
                r[k] = active ? value : kInf2;
                lowest = vmin2(lowest, r[k]);
            }
            if (active) *reinterpret_cast<T *>(dst + step * stride) = C::pack(r);
            uint32_t m = min(lowest & 0xFFFFu, lowest >> 16);
            m = __reduce_min_sync(kFullMask, m);
            m2 = m * 0x10001u;
            j2 = (m + (uint32_t)s.p2) * 0x10001u;
        }
    }
}

static int lanes_disparities(int disparities) {
    // Disparities per lane: a warp of 32 lanes covers up to 32 * DPL.
    return disparities <= 64 ? 2 : (disparities <= 128 ? 4 : 8);
}

cudaError_t launch_paths(const uint8_t *costs, int width, int height, int disparities, int paths,
                         int p1, int p2, uint8_t *paths_out, cudaStream_t stream) {
    PathSetup s{};
    s.width = width;
    s.height = height;
    s.disparities = disparities;
    s.p1 = p1;
    s.p2 = p2;
    s.paths = paths;
    s.volume = (size_t)width * height * disparities;
    int total = 0;
    for (int p = 0; p < paths; ++p) {
        s.first_warp[p] = total;
        s.dy[p] = kDirections[p][0];
        s.dx[p] = kDirections[p][1];
        total += s.dy[p] == 0 ? height : (s.dx[p] == 0 ? width : width + height - 1);
    }
    s.first_warp[paths] = total;
    const int threads = 128, warps_per_block = threads / 32;
    const int blocks = (total + warps_per_block - 1) / warps_per_block;
    switch (lanes_disparities(disparities)) {
    case 2: paths_kernel<2><<<blocks, threads, 0, stream>>>(costs, paths_out, s); break;
    case 4: paths_kernel<4><<<blocks, threads, 0, stream>>>(costs, paths_out, s); break;
    default: paths_kernel<8><<<blocks, threads, 0, stream>>>(costs, paths_out, s); break;
    }
    return cudaGetLastError();
}

// sums[y][x][d] = sum of the P path volumes, u16 (at most 8 x 127 = 1016).
__global__ void sum_paths_kernel(const uint8_t *__restrict__ paths_in, size_t volume, int paths,
                                 uint16_t *__restrict__ sums) {
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
    sum_paths_kernel<<<(unsigned)((quads + 255) / 256), 256, 0, stream>>>(paths_in, volume, paths,
                                                                          sums);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- select
// Winner, uniqueness and subpixel (lib/nx_stereo.ex:608-641), one warp per
// pixel, lanes over disparities. values = sums + 0x8000 past x; the winner is
// the lowest (value << 16 | d), so ties go to the lowest d; `second` is the
// lowest value more than one disparity from the winner; the f32 steps are
// rounded one at a time in the reference's order.
template <int DPL, bool FROM_SUMS>
__global__ void __launch_bounds__(128)
    select_kernel(const void *__restrict__ source, int width, int height, int disparities,
                  int paths, size_t volume, float uniqueness, float *__restrict__ disparity,
                  uint32_t *__restrict__ keys) {
    const size_t pixel = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (pixel >= (size_t)width * height) return;
    const int x = (int)(pixel % width);
    const int D = disparities;
    const bool active = lane * DPL < D;
    uint32_t sum[DPL];
#pragma unroll
    for (int i = 0; i < DPL; ++i) sum[i] = 0;
    if (active) {
        const size_t at = pixel * D + lane * DPL;
        if (FROM_SUMS) {
            const uint16_t *sums = static_cast<const uint16_t *>(source) + at;
#pragma unroll
            for (int i = 0; i < DPL; ++i) sum[i] = sums[i];
        } else {
            const uint8_t *volumes = static_cast<const uint8_t *>(source) + at;
            uint32_t packed[DPL / 2];
#pragma unroll
            for (int k = 0; k < DPL / 2; ++k) packed[k] = 0;
            for (int p = 0; p < paths; ++p) {
                uint32_t words[DPL / 2];
                Chunk<DPL>::unpack(
                    __ldg(reinterpret_cast<const typename Chunk<DPL>::T *>(volumes + p * volume)),
                    words);
#pragma unroll
                for (int k = 0; k < DPL / 2; ++k) packed[k] += words[k];
            }
#pragma unroll
            for (int k = 0; k < DPL / 2; ++k) {
                sum[2 * k] = packed[k] & 0xFFFFu;
                sum[2 * k + 1] = packed[k] >> 16;
            }
        }
    }
    uint32_t value[DPL];
    uint32_t best = 0xFFFFFFFFu;
#pragma unroll
    for (int i = 0; i < DPL; ++i) {
        const int d = lane * DPL + i;
        value[i] = sum[i] + (d > x ? 0x8000u : 0u);
        if (active) best = min(best, (value[i] << 16) | (uint32_t)d);
    }
    best = __reduce_min_sync(kFullMask, best);
    const uint32_t minimum = best >> 16;
    const int winner = (int)(best & 0xFFFFu);
    const int below = max(winner - 1, 0), above = min(winner + 1, D - 1);
    uint32_t second = 0xFFFFFFFFu, lower = 0xFFFFFFFFu, upper = 0xFFFFFFFFu;
#pragma unroll
    for (int i = 0; i < DPL; ++i) {
        const int d = lane * DPL + i;
        if (!active) continue;
        if (d < winner - 1 || d > winner + 1) second = min(second, value[i]);
        if (d == below) lower = value[i];
        if (d == above) upper = value[i];
    }
    second = __reduce_min_sync(kFullMask, second);
    lower = __reduce_min_sync(kFullMask, lower);
    upper = __reduce_min_sync(kFullMask, upper);
    if (lane != 0) return;
    const float lower_f = (float)lower, upper_f = (float)upper, minimum_f = (float)minimum;
    // With no disparity outside the winner's neighbours the reference's
    // minimum is i32::MAX (lib/nx_stereo.ex:620-622).
    const float second_f = second == 0xFFFFFFFFu ? 2147483647.0f : (float)second;
    const bool accepted = second_f > fmul(minimum_f, uniqueness);
    const float denominator = fsub(fadd(lower_f, upper_f), fmul(2.0f, minimum_f));
    const float bounded = denominator > 1.0f ? denominator : 1.0f;
    float correction = fdiv(fsub(lower_f, upper_f), fmul(2.0f, bounded));
    correction = correction < -0.5f ? -0.5f : (correction > 0.5f ? 0.5f : correction);
    const bool refine = denominator > 0.0f && winner > 0 && winner < min(D - 1, x);
    const float value_f = refine ? fadd((float)winner, correction) : (float)winner;
    disparity[pixel] = accepted ? value_f : -1.0f;
    keys[pixel] = accepted ? ((minimum << 16) | (uint32_t)winner) : kInvalidKey;
}

template <bool FROM_SUMS>
static cudaError_t launch_select(const void *source, int width, int height, int disparities,
                                 int paths, float uniqueness, float *disparity, uint32_t *keys,
                                 cudaStream_t stream) {
    const size_t pixels = (size_t)width * height;
    const size_t volume = pixels * disparities;
    const unsigned blocks = (unsigned)((pixels * 32 + 127) / 128);
    switch (lanes_disparities(disparities)) {
    case 2:
        select_kernel<2, FROM_SUMS><<<blocks, 128, 0, stream>>>(
            source, width, height, disparities, paths, volume, uniqueness, disparity, keys);
        break;
    case 4:
        select_kernel<4, FROM_SUMS><<<blocks, 128, 0, stream>>>(
            source, width, height, disparities, paths, volume, uniqueness, disparity, keys);
        break;
    default:
        select_kernel<8, FROM_SUMS><<<blocks, 128, 0, stream>>>(
            source, width, height, disparities, paths, volume, uniqueness, disparity, keys);
        break;
    }
    return cudaGetLastError();
}

cudaError_t launch_select_paths(const uint8_t *paths_in, int width, int height, int disparities,
                                int paths, float uniqueness, float *disparity, uint32_t *keys,
                                cudaStream_t stream) {
    return launch_select<false>(paths_in, width, height, disparities, paths, uniqueness,
                                disparity, keys, stream);
}

cudaError_t launch_select_sums(const uint16_t *sums, int width, int height, int disparities,
                               float uniqueness, float *disparity, uint32_t *keys,
                               cudaStream_t stream) {
    return launch_select<true>(sums, width, height, disparities, 0, uniqueness, disparity, keys,
                               stream);
}

// ---------------------------------------------------------------- check
// OpenCV's left-right check (lib/nx_stereo.ex:643-683), one block per row:
// the right map is the per-row atomicMin of (key & 0xFFFF0000) | (65535 - d)
// at x - d, so the cheapest match wins and ties go to the larger d.
__global__ void __launch_bounds__(256)
    consistency_kernel(const float *__restrict__ disparity, const uint32_t *__restrict__ keys,
                       int width, float *__restrict__ checked) {
    extern __shared__ uint32_t right[];
    const size_t row = (size_t)blockIdx.x * width;
    for (int x = threadIdx.x; x < width; x += blockDim.x) right[x] = kInvalidKey;
    __syncthreads();
    for (int x = threadIdx.x; x < width; x += blockDim.x) {
        uint32_t key = keys[row + x];
        if (key == kInvalidKey) continue;
        int winner = (int)(key & 0xFFFFu);
        if (x - winner < 0) continue;  // a winner is at most x (past-edge costs lose)
        atomicMin(&right[x - winner], (key & 0xFFFF0000u) | (65535u - (uint32_t)winner));
    }
    __syncthreads();
    for (int x = threadIdx.x; x < width; x += blockDim.x) {
        float value = disparity[row + x];
        int low = (int)floorf(value), high = (int)ceilf(value);
        bool rejected = true;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            int d = k == 0 ? low : high;
            int rx = x - d;
            bool inside = rx >= 0 && rx < width;
            uint32_t found = right[min(max(rx, 0), width - 1)];
            int right_d = 65535 - (int)(found & 0xFFFFu);
            bool disagrees = inside && found != kInvalidKey && abs(right_d - d) > 1;
            rejected = rejected && disagrees;
        }
        checked[row + x] = (value >= 0.0f && !rejected) ? value : -1.0f;
    }
}

cudaError_t launch_consistency(const float *disparity, const uint32_t *keys, int width,
                               int height, float *checked, cudaStream_t stream) {
    consistency_kernel<<<height, 256, sizeof(uint32_t) * width, stream>>>(disparity, keys, width,
                                                                         checked);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- median
// Devillard's 9-element network (lib/nx_stereo/image.ex:272, 483-505): the
// median ends in slot 4; borders replicated. Then, for Stage.Disparity,
// disparity <= 0 becomes -1 (lib/nx_stereo/stage/disparity.ex:162).
__device__ __forceinline__ void exchange(float &a, float &b) {
    const float lo = fminf(a, b), hi = fmaxf(a, b);
    a = lo;
    b = hi;
}

__global__ void median3_kernel(const float *__restrict__ image, int width, int height,
                               int stage_mask, float *__restrict__ filtered) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= width) return;
    float v[9];
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            int sy = min(max(y + dy, 0), height - 1), sx = min(max(x + dx, 0), width - 1);
            v[(dy + 1) * 3 + dx + 1] = image[(size_t)sy * width + sx];
        }
    exchange(v[1], v[2]); exchange(v[4], v[5]); exchange(v[7], v[8]);
    exchange(v[0], v[1]); exchange(v[3], v[4]); exchange(v[6], v[7]);
    exchange(v[1], v[2]); exchange(v[4], v[5]); exchange(v[7], v[8]);
    exchange(v[0], v[3]); exchange(v[5], v[8]); exchange(v[4], v[7]);
    exchange(v[3], v[6]); exchange(v[1], v[4]); exchange(v[2], v[5]);
    exchange(v[4], v[7]); exchange(v[4], v[2]); exchange(v[6], v[4]);
    exchange(v[4], v[2]);
    float out = v[4];
    if (stage_mask && !(out > 0.0f)) out = -1.0f;
    filtered[(size_t)y * width + x] = out;
}

cudaError_t launch_median3(const float *image, int width, int height, int stage_mask,
                           float *filtered, cudaStream_t stream) {
    dim3 grid((width + 127) / 128, height);
    median3_kernel<<<grid, 128, 0, stream>>>(image, width, height, stage_mask, filtered);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- the matcher
static size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

size_t matcher_scratch_bytes(int width, int height, int disparities) {
    const size_t pixels = (size_t)width * height, volume = pixels * disparities;
    return 2 * align256(8 * pixels) + align256(volume) + 8 * align256(volume) +
           3 * align256(4 * pixels);
}

MatcherScratch carve_matcher_scratch(void *base, int width, int height, int disparities) {
    const size_t pixels = (size_t)width * height, volume = pixels * disparities;
    char *at = static_cast<char *>(base);
    MatcherScratch s;
    s.left_codes = reinterpret_cast<uint64_t *>(at);
    at += align256(8 * pixels);
    s.right_codes = reinterpret_cast<uint64_t *>(at);
    at += align256(8 * pixels);
    s.costs = reinterpret_cast<uint8_t *>(at);
    at += align256(volume);
    s.paths = reinterpret_cast<uint8_t *>(at);
    at += 8 * align256(volume);
    s.selected = reinterpret_cast<float *>(at);
    at += align256(4 * pixels);
    s.checked = reinterpret_cast<float *>(at);
    at += align256(4 * pixels);
    s.keys = reinterpret_cast<uint32_t *>(at);
    return s;
}

cudaError_t run_matcher(const uint8_t *left, const uint8_t *right, int width, int height,
                        int disparities, int paths, int p1, int p2, float uniqueness,
                        int stage_mask, const MatcherScratch &s, float *disparity,
                        cudaStream_t stream) {
    cudaError_t e;
    if ((e = launch_census(left, right, width, height, s.left_codes, s.right_codes, stream)))
        return e;
    if ((e = launch_costs(s.left_codes, s.right_codes, width, height, disparities, s.costs,
                          stream)))
        return e;
    if ((e = launch_paths(s.costs, width, height, disparities, paths, p1, p2, s.paths, stream)))
        return e;
    if ((e = launch_select_paths(s.paths, width, height, disparities, paths, uniqueness,
                                 s.selected, s.keys, stream)))
        return e;
    if ((e = launch_consistency(s.selected, s.keys, width, height, s.checked, stream))) return e;
    return launch_median3(s.checked, width, height, stage_mask, disparity, stream);
}

}  // namespace nxs
