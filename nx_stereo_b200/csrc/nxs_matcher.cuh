// Device building blocks of the matcher, shared by the single-pair kernels
// (matcher.cu) and the batched ones (batch.cu): each takes the pair's buffers
// and sizes as arguments and the position of its block within the pair.
#pragma once

#include <cstddef>
#include <cstdint>
#include <type_traits>

#include <cuda.h>  // CUtensorMap

#include "nxs_device.cuh"

namespace nxs {

// ---------------------------------------------------------------- census
// 9x7 sparse census (lib/nx_stereo.ex:491-505): bit i for the i-th neighbour
// in row-major order over dy in -3..3, dx in -4..4, both non-zero, set where
// neighbour + 1 < centre; borders replicated (lib/nx_stereo/image.ex:508-537).

// Four pixels' codes at once, as packed bytes. `window` holds the pixels'
// 9x7 neighbourhoods in rows `pitch` bytes apart (pitch a multiple of 4);
// the first pixel's centre is at row `centre_row`, column `col` (a multiple
// of 4). The six neighbour rows give the code's six bytes: for each row, the
// eight neighbours at dx -4..-1, 1..4 enter each pixel's byte from the top
// (acc >> 1, the new bit at bit 7), so after eight the first is bit 0, as in
// census_code. n + 1 < c is n < t with t = c - 1 (0 where c is 0: then no
// neighbour is below it), compared four bytes at a time: bit 7 of
// d = (n | 0x80) - (t & 0x7F) says low7(n) >= low7(t), and
// n < t = (!n7 & t7) | (n7 == t7 & !d7).
__device__ __forceinline__ void census4(const uint8_t *window, int pitch, int col,
                                        int centre_row, uint64_t *codes) {
    const uint32_t c =
        *reinterpret_cast<const uint32_t *>(window + (size_t)centre_row * pitch + col);
    const uint32_t zero = ~(((c & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | c | 0x7F7F7F7Fu);  // bit 7: c == 0
    const uint32_t t = (c | (zero >> 7)) - 0x01010101u;
    const uint32_t t_low = t & 0x7F7F7F7Fu;
    uint32_t acc[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        const int dy = r < 3 ? r - 3 : r - 2;
        const uint32_t *w =
            reinterpret_cast<const uint32_t *>(window + (size_t)(centre_row + dy) * pitch + col - 4);
        const uint32_t w0 = w[0], w1 = w[1], w2 = w[2];  // columns col - 4 .. col + 7
        uint32_t a = 0;
#pragma unroll
        for (int dx = -4; dx <= 4; ++dx) {
            if (dx == 0) continue;
            // the four pixels' neighbours at dx: bytes col + dx .. col + dx + 3
            const int o = dx + 4;  // offset from column col - 4
            const uint32_t n = o == 0 ? w0 : o == 4 ? w1 : o == 8 ? w2
                               : o < 4 ? __byte_perm(w0, w1, (o) | (o + 1) << 4 | (o + 2) << 8 | (o + 3) << 12)
                                       : __byte_perm(w1, w2, (o - 4) | (o - 3) << 4 | (o - 2) << 8 | (o - 1) << 12);
            const uint32_t d = (n | 0x80808080u) - t_low;
            const uint32_t below = (~n & t) | (~(n ^ t) & ~d);  // bit 7 of each byte
            a = ((a >> 1) & 0x7F7F7F7Fu) | (below & 0x80808080u);
        }
        acc[r] = a;
    }
    // pixel i: byte r of its code is byte i of acc[r]
    const uint32_t lo01 = __byte_perm(acc[0], acc[1], 0x5140), lo23 = __byte_perm(acc[2], acc[3], 0x5140);
    const uint32_t hi01 = __byte_perm(acc[0], acc[1], 0x7362), hi23 = __byte_perm(acc[2], acc[3], 0x7362);
    const uint32_t top01 = __byte_perm(acc[4], acc[5], 0x5140), top23 = __byte_perm(acc[4], acc[5], 0x7362);
    // lo01 = (a0.b0, a1.b0, a0.b1, a1.b1): pixel 0's bytes 0-1 in its low half, pixel 1's in its high
    codes[0] = (uint64_t)__byte_perm(lo01, lo23, 0x5410) | (uint64_t)(top01 & 0xFFFFu) << 32;
    codes[1] = (uint64_t)__byte_perm(lo01, lo23, 0x7632) | (uint64_t)(top01 >> 16) << 32;
    codes[2] = (uint64_t)__byte_perm(hi01, hi23, 0x5410) | (uint64_t)(top23 & 0xFFFFu) << 32;
    codes[3] = (uint64_t)__byte_perm(hi01, hi23, 0x7632) | (uint64_t)(top23 >> 16) << 32;
}

// The census of a tile of kCensus4X x ROWS pixels with census4: THREADS
// threads, each 4 pixels of a row at a time; `tile` holds the window of
// (kCensus4X + 8) x (ROWS + 6) bytes (census4_tile_bytes).
constexpr int kCensus4X = 128;
__host__ __device__ constexpr int census4_tile_bytes(int rows) { return (rows + 6) * (kCensus4X + 8); }

// Copies rows y0 - 3 .. of `image` (clamped), columns x0 - 4 .. x0 - 4 + pitch - 1
// (clamped), into `window` ([rows][pitch]): every thread's loads first, in
// flight together (at most MAX_PER a thread), then the shared stores.
template <int THREADS, int MAX_PER>
__device__ __forceinline__ void stage_window(const uint8_t *__restrict__ image, int width,
                                             int height, int x0, int y0, int rows, int pitch,
                                             uint8_t *window, int tid) {
    const int cells = rows * pitch;
    uint8_t v[MAX_PER];
#pragma unroll
    for (int k = 0; k < MAX_PER; ++k) {
        const int i = tid + k * THREADS;
        if (i < cells) {
            const int sy = min(max(y0 + i / pitch - 3, 0), height - 1);
            const int sx = min(max(x0 + i % pitch - 4, 0), width - 1);
            v[k] = __ldg(image + (size_t)sy * width + sx);
        }
    }
#pragma unroll
    for (int k = 0; k < MAX_PER; ++k) {
        const int i = tid + k * THREADS;
        if (i < cells) window[i] = v[k];
    }
}

// stage_window for a pitch known only at run time (at most MAX_PITCH): ROWS
// rows, each thread columns tid, tid + THREADS, ... of every row, all loads
// in flight together, with no division by the pitch.
template <int THREADS, int ROWS, int MAX_PITCH>
__device__ __forceinline__ void stage_rows(const uint8_t *__restrict__ image, int width,
                                           int height, int x0, int y0, int pitch,
                                           uint8_t *window, int tid) {
    constexpr int PER_ROW = (MAX_PITCH + THREADS - 1) / THREADS;
    uint8_t v[ROWS][PER_ROW];
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        const uint8_t *row = image + (size_t)min(max(y0 + r - 3, 0), height - 1) * width;
#pragma unroll
        for (int k = 0; k < PER_ROW; ++k) {
            const int c = tid + k * THREADS;
            if (c < pitch) v[r][k] = __ldg(row + min(max(x0 + c - 4, 0), width - 1));
        }
    }
#pragma unroll
    for (int r = 0; r < ROWS; ++r)
#pragma unroll
        for (int k = 0; k < PER_ROW; ++k) {
            const int c = tid + k * THREADS;
            if (c < pitch) window[r * pitch + c] = v[r][k];
        }
}

// n / d for 0 <= n < 2^16 and 0 < d <= 16 by a multiply-high of 16 n with
// magic = 0x0FFFFFFF / d + 1 (ceil(2^28 / d), which fits 32 bits for every d
// including 1): the rounding error 16 n / 2^32 stays below 1 / d.
__host__ __device__ constexpr uint32_t small_divisor_magic(uint32_t d) {
    return 0x0FFFFFFFu / d + 1u;
}
__device__ __forceinline__ uint32_t divide_small(uint32_t n, uint32_t magic) {
    return __umulhi(n << 4, magic);
}

template <int ROWS, int THREADS>
__device__ __forceinline__ void census4_tile(const uint8_t *__restrict__ image, int width,
                                             int height, uint64_t *__restrict__ codes, int x0,
                                             int y0, int tid, uint8_t *tile) {
    constexpr int PITCH = kCensus4X + 8;
    stage_window<THREADS, ((ROWS + 6) * PITCH + THREADS - 1) / THREADS>(
        image, width, height, x0, y0, ROWS + 6, PITCH, tile, tid);
    __syncthreads();
    for (int g = tid; g < (kCensus4X / 4) * ROWS; g += THREADS) {
        const int tx = 4 * (g % (kCensus4X / 4)), ty = g / (kCensus4X / 4);
        const int x = x0 + tx, y = y0 + ty;
        if (x >= width || y >= height) continue;
        uint64_t four[4];
        census4(tile, PITCH, tx + 4, ty + 3, four);
        uint64_t *out = codes + (size_t)y * width + x;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (x + i < width) out[i] = four[i];
    }
}

// ---------------------------------------------------------------- costs
// costs[y][x][d] = popcount(left[y][x] ^ right[y][x - d]), right codes left of
// the image zero (lib/nx_stereo.ex:528-542). SPAN 8 or 16 stores each run of
// SPAN disparities in the permuted order of span_disparity, the order the
// matcher's own path and selection kernels work in. A block of 128 threads covers 64
// pixels of a row. It stages their left codes and the D + 64 right codes from
// x0 - D on; a thread computes 4 neighbouring pixels x 16 disparities, whose
// right codes are 19 consecutive ones held in registers, into a shared tile,
// and the block then writes its 64 x D bytes out contiguously with 16-byte
// stores.
constexpr int kCostPixels = 64;

// The permuted disparity order: a path lane holding a run of SPAN
// disparities keeps them as u16x2 words, word k holding (k, k + SPAN / 2), so
// the neighbours of both halves at d - 1 and at d + 1 are the whole words
// k - 1 and k + 1. In memory each 4 bytes 4q .. 4q + 3 of a run hold words
// 2q and 2q + 1 interleaved: disparities 2q, 2q + 1, 2q + SPAN / 2 and
// 2q + 1 + SPAN / 2, so a lane packs two words into one u32 with one
// multiply-add (w[2q] + 256 w[2q + 1]) and unpacks them with two byte
// permutes. SPAN 0 is the natural order. span_disparity: the disparity at
// byte j; span_position: the byte that holds disparity d.
__host__ __device__ constexpr int span_disparity(int span, int j) {
    return span == 0 ? j
                     : (j / span) * span + 2 * ((j % span) / 4) + (j % 2) +
                           (span / 2) * (((j % span) / 2) % 2);
}
__host__ __device__ constexpr int span_position(int span, int d) {
    return span == 0 ? d
                     : (d / span) * span + 4 * (((d % span) % (span / 2)) / 2) + (d % 2) +
                           2 * ((d % span) / (span / 2));
}

// Where code j of a staged code array (lefts, rights below) lies: within each
// 128-byte block of 8 code pairs, an odd block swaps neighbouring pairs, so that
// the 16-byte pair reads of eight threads whose windows start 4 codes apart fall
// in 8 different bank quads (checked on the CPU for 16..256 disparities).
__host__ __device__ constexpr int code_slot(int j) { return j ^ ((j >> 3) & 2); }
__host__ __device__ constexpr int pair_slot(int pair) { return pair ^ ((pair >> 3) & 1); }

__host__ __device__ inline size_t costs_shared_bytes(int disparities) {
    return sizeof(uint64_t) * (2 * kCostPixels + disparities) + (size_t)kCostPixels * disparities;
}

// Costs of PIXELS pixels of row y from x0 on, from codes staged in shared
// memory (16-byte aligned): lefts[code_slot(i)] the code of x0 + i (0 past the
// image), rights[code_slot(i)] that of x0 - D + i (0 outside it), PIXELS + D of
// them; `tile` (16-byte aligned) takes PIXELS x D bytes.
//
// Shared-memory banks: a warp's threads take neighbouring groups of 4 pixels at
// one run of 16 disparities. Their code windows start 4 codes (32 bytes) apart
// and are read as 16-byte pairs, which code_slot's layout spreads over all bank
// quads. Each tile row is D bytes with its 16-byte runs rotated by the pixel's
// group (run q of pixel p at (q + p / 4) mod D / 16), so a warp's 16-byte stores
// to four pixel rows fall in 8 different bank quads; the write-out undoes the
// rotation.
// 256^b for the byte b of a word of costs, read at run time so that the
// packing below stays multiply-adds (FMA pipe) beside the popcounts (XU) and
// the XORs (integer pipe).
__constant__ uint32_t g_byte_scale[4] = {1u, 256u, 65536u, 16777216u};

template <int SPAN, int PIXELS>
__device__ __forceinline__ void costs_from_codes(const uint64_t *lefts, const uint64_t *rights,
                                                 int width, int disparities,
                                                 uint8_t *__restrict__ costs, int x0, int y,
                                                 uint8_t *tile) {
    const int D = disparities;
    const size_t row = (size_t)y * width;
    const int groups = PIXELS / 4, chunks = D / 16;
    const uint32_t magic = small_divisor_magic((uint32_t)chunks);  // divide_small by chunks
    for (int t = threadIdx.x; t < groups * chunks; t += blockDim.x) {
        const int group = t % groups, q = t / groups;
        const int p0 = 4 * group, d0 = 16 * q;
        // pixel p0 + i at disparity d0 + k reads rights[p0 + i - d0 - k + D]
        //   = window[16 + i - k], window[m] = rights[p0 - d0 + D - 16 + m]
        // (m = 1..19; the first of the 20 is read for the 16-byte alignment)
        const uint4 *pairs = reinterpret_cast<const uint4 *>(rights);
        const int first = (p0 - d0 + D - 16) / 2;  // the window's first pair
        uint64_t window[20];
#pragma unroll
        for (int j = 0; j < 10; ++j) {
            const uint4 two = pairs[pair_slot(first + j)];
            window[2 * j] = (uint64_t)two.x | (uint64_t)two.y << 32;
            window[2 * j + 1] = (uint64_t)two.z | (uint64_t)two.w << 32;
        }
        const uint4 *left_pairs = reinterpret_cast<const uint4 *>(lefts);
        const uint4 l01 = left_pairs[pair_slot(2 * group)];
        const uint4 l23 = left_pairs[pair_slot(2 * group + 1)];
        const uint64_t l4[4] = {(uint64_t)l01.x | (uint64_t)l01.y << 32,
                                (uint64_t)l01.z | (uint64_t)l01.w << 32,
                                (uint64_t)l23.x | (uint64_t)l23.y << 32,
                                (uint64_t)l23.z | (uint64_t)l23.w << 32};
        int rotated = q + group - chunks * (int)divide_small(group, magic);  // q + group % chunks
        if (rotated >= chunks) rotated -= chunks;
        uint32_t scale[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) scale[b] = g_byte_scale[b];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            uint32_t words[4];
#pragma unroll
            for (int w4 = 0; w4 < 4; ++w4) {
                // Byte b of the word: the popcounts of the XOR's two halves, each
                // added as count x 256^b (a cost is at most 48, so no byte carries).
                uint32_t w = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int k = span_disparity(SPAN, 4 * w4 + b);
                    const uint64_t x = l4[i] ^ window[16 + i - k];
                    uint32_t low;
                    asm("mad.lo.u32 %0, %1, %2, %3;"
                        : "=r"(low)
                        : "r"((uint32_t)__popc((uint32_t)x)), "r"(scale[b]), "r"(w));
                    asm("mad.lo.u32 %0, %1, %2, %3;"
                        : "=r"(w)
                        : "r"((uint32_t)__popc((uint32_t)(x >> 32))), "r"(scale[b]), "r"(low));
                }
                words[w4] = w;
            }
            *reinterpret_cast<uint4 *>(tile + (p0 + i) * D + 16 * rotated) =
                make_uint4(words[0], words[1], words[2], words[3]);
        }
    }
    __syncthreads();
    const int pixels = min(PIXELS, width - x0);
    uint4 *out = reinterpret_cast<uint4 *>(costs + (row + x0) * D);
    for (int c = threadIdx.x; c < pixels * chunks; c += blockDim.x) {
        const int p = (int)divide_small(c, magic), g = p / 4;
        int rotated = c - p * chunks + g - chunks * (int)divide_small(g, magic);
        if (rotated >= chunks) rotated -= chunks;
        out[c] = *reinterpret_cast<const uint4 *>(tile + p * D + 16 * rotated);
    }
}

template <int SPAN = 0>
__device__ __forceinline__ void costs_tile(const uint64_t *__restrict__ left_codes,
                                           const uint64_t *__restrict__ right_codes, int width,
                                           int disparities, uint8_t *__restrict__ costs, int x0,
                                           int y, uint8_t *staged) {
    const int D = disparities;
    uint64_t *lefts = reinterpret_cast<uint64_t *>(staged);
    uint64_t *rights = lefts + kCostPixels;
    uint8_t *tile = staged + sizeof(uint64_t) * (2 * kCostPixels + D);
    const size_t row = (size_t)y * width;
    for (int i = threadIdx.x; i < kCostPixels; i += blockDim.x)
        lefts[code_slot(i)] = x0 + i < width ? __ldcg(left_codes + row + x0 + i) : 0;
    for (int i = threadIdx.x; i < kCostPixels + D; i += blockDim.x) {
        const int x = x0 - D + i;
        rights[code_slot(i)] = (x >= 0 && x < width) ? __ldcg(right_codes + row + x) : 0;
    }
    __syncthreads();
    costs_from_codes<SPAN, kCostPixels>(lefts, rights, width, D, costs, x0, y, tile);
}

// ---------------------------------------------------------------- census + costs
// Both steps for PIXELS pixels of row y from x0 on, in one block of THREADS
// threads: the block stages the 7 rows of both images around row y that the
// pixels' census windows reach (the left image's columns x0 - 4 .. x0 +
// PIXELS + 3, the right image's x0 - D - 4 .. x0 + PIXELS + 3, clamped as the
// census clamps), takes census4 of the PIXELS left pixels and of the PIXELS + D
// right pixels from x0 - D on into shared memory (0 outside the image), and
// forms the costs from them with costs_from_codes. The codes never reach
// global memory; each right code is formed by up to (PIXELS + D) / PIXELS
// blocks, which is integer work beside the popcounts that bound the costs.
constexpr int kCensusCostPixels = 128;

__host__ __device__ constexpr int census_costs_window_bytes(int pixels, int disparities) {
    return (7 * (pixels + 8) + 7 * (pixels + disparities + 8) + 15) / 16 * 16;
}

__host__ __device__ inline size_t census_costs_shared_bytes(int pixels, int disparities) {
    return sizeof(uint64_t) * (2 * pixels + disparities) +
           census_costs_window_bytes(pixels, disparities) + (size_t)pixels * disparities;
}

template <int SPAN, int PIXELS, int THREADS, int MAX_DISPARITIES = 256>
__device__ __forceinline__ void census_costs_tile(const uint8_t *__restrict__ left_image,
                                                  const uint8_t *__restrict__ right_image,
                                                  int width, int height, int disparities,
                                                  uint8_t *__restrict__ costs, int x0, int y,
                                                  uint8_t *staged, int tid) {
    static_assert(PIXELS % 4 == 0, "census4 takes four pixels at once");
    const int D = disparities;
    const int left_pitch = PIXELS + 8, right_pitch = PIXELS + D + 8;
    uint64_t *lefts = reinterpret_cast<uint64_t *>(staged);   // x0 ..
    uint64_t *rights = lefts + PIXELS;                         // x0 - D ..
    uint8_t *left_window = reinterpret_cast<uint8_t *>(rights + PIXELS + D);
    uint8_t *right_window = left_window + 7 * left_pitch;
    uint8_t *tile = left_window + census_costs_window_bytes(PIXELS, D);
    stage_rows<THREADS, 7, PIXELS + 8>(left_image, width, height, x0, y, left_pitch, left_window,
                                       tid);
    stage_rows<THREADS, 7, PIXELS + MAX_DISPARITIES + 8>(right_image, width, height, x0 - D, y,
                                                         right_pitch, right_window, tid);
    __syncthreads();
    constexpr int kLeftGroups = PIXELS / 4;
    const int groups = kLeftGroups + (PIXELS + D) / 4;
    for (int g = tid; g < groups; g += THREADS) {
        uint64_t four[4];
        if (g < kLeftGroups) {
            census4(left_window, left_pitch, 4 * g + 4, 3, four);
#pragma unroll
            for (int i = 0; i < 4; ++i)
                lefts[code_slot(4 * g + i)] = x0 + 4 * g + i < width ? four[i] : 0;
        } else {
            const int r = g - kLeftGroups;
            census4(right_window, right_pitch, 4 * r + 4, 3, four);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int x = x0 - D + 4 * r + i;
                rights[code_slot(4 * r + i)] = (x >= 0 && x < width) ? four[i] : 0;
            }
        }
    }
    __syncthreads();
    costs_from_codes<SPAN, PIXELS>(lefts, rights, width, D, costs, x0, y, tile);
}

// ---------------------------------------------------------------- paths
// libSGM's normalised recurrence (lib/nx_stereo.ex:575-606) along every scan
// line of every direction, unnormalised:
//   L[d] = min(prev[d], prev[d-1] + p1, prev[d+1] + p1, m + p2) - m + C[d],
//   m = min over d of prev,
// which equals the reference's min(min(a, p2), min(a[d-1], a[d+1]) + p1) + C
// with a = prev - m; its out-of-range neighbours (p2 - p1, so p2 once p1 is
// added) never beat m + p2, so they read as +inf. Lanes past D hold +inf.
// A path starts from zero where it enters the image, so its first step is C.
//
// A group of G lanes follows one line, each lane holding 2 * WORDS
// disparities as u16x2 words (five integer instructions per word and step),
// and a warp follows 32 / G lines in lockstep. Each lane copies its costs for the next kPrefetch - 1 steps into a shared
// ring with cp.async while a step computes, and stores its path costs with
// 16-byte stores.
constexpr int kPrefetch = 8;

struct PathSetup {
    int width, height, disparities, p1, p2, paths;
    int first_warp[9];  // first warp of each direction; first_warp[paths] = total
    int lines[8];       // scan lines of each direction
    int dy[8], dx[8];
    int order[8];       // direction of each slot: rows first, then columns, then diagonals
    int straight;       // slots of rows and columns
    // 1, given at run time so that some of the recurrence's adds and the
    // pointer steps are issued as multiply-adds on the FMA pipe (follow_lines).
    unsigned one;
    size_t volume;      // bytes of one direction's volume
};

// a * b + c (mod 2^32) as a multiply-add.
__device__ __forceinline__ uint32_t mad_lo(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// The u16x2 minimum over each aligned group of G lanes (a scan line's lanes):
// rounds of three shuffles (xor s, 2s, 3s) and one three-way min cover four
// lanes at once, so 8 lanes take two dependent shuffle rounds instead of three
// (728x544x128: 118.8 against 122.9 us); 16 lanes keep the four pairwise rounds
// (1920x1080x256: six shuffles in two rounds measured 1.4% slower).
template <int G>
__device__ __forceinline__ uint32_t line_minimum(uint32_t v) {
    if constexpr (G >= 16) {
#pragma unroll
        for (int offset = G / 2; offset >= 1; offset /= 2)
            v = vmin2(v, __shfl_xor_sync(kFullMask, v, offset));
    } else {
#pragma unroll
        for (int span = 1; span < G; span *= 4) {
            if (span * 2 == G) {
                v = vmin2(v, __shfl_xor_sync(kFullMask, v, span));
            } else {
                const uint32_t a = __shfl_xor_sync(kFullMask, v, span);
                const uint32_t b = __shfl_xor_sync(kFullMask, v, 2 * span);
                const uint32_t c = __shfl_xor_sync(kFullMask, v, 3 * span);
                v = vmin2(__vimin3_u16x2(v, a, b), c);
            }
        }
    }
    return v;
}

// p + a * b bytes for a pointer p and 32-bit a, b, as one wide multiply-add.
template <typename T>
__device__ __forceinline__ T *advance(T *p, int a, unsigned b) {
    uint64_t d;
    asm("mad.wide.s32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"((int)b), "l"((uint64_t)p));
    return reinterpret_cast<T *>(d);
}

// The words of a permuted run (span_disparity) from its bytes, and back.
__device__ __forceinline__ void unpack_run16(const uint4 c, uint32_t *w) {
    w[0] = __byte_perm(c.x, 0, 0x4240);
    w[1] = __byte_perm(c.x, 0, 0x4341);
    w[2] = __byte_perm(c.y, 0, 0x4240);
    w[3] = __byte_perm(c.y, 0, 0x4341);
    w[4] = __byte_perm(c.z, 0, 0x4240);
    w[5] = __byte_perm(c.z, 0, 0x4341);
    w[6] = __byte_perm(c.w, 0, 0x4240);
    w[7] = __byte_perm(c.w, 0, 0x4341);
}
__device__ __forceinline__ void unpack_run8(const uint2 c, uint32_t *w) {
    w[0] = __byte_perm(c.x, 0, 0x4240);
    w[1] = __byte_perm(c.x, 0, 0x4341);
    w[2] = __byte_perm(c.y, 0, 0x4240);
    w[3] = __byte_perm(c.y, 0, 0x4341);
}
// Halves below 256: w[2q] + 256 w[2q + 1] interleaves their bytes (a
// multiply-add by a run-time 256, on the FMA pipe).
__device__ __forceinline__ uint4 pack_run16(const uint32_t *w, uint32_t byte) {
    return make_uint4(mad_lo(w[1], byte, w[0]), mad_lo(w[3], byte, w[2]),
                      mad_lo(w[5], byte, w[4]), mad_lo(w[7], byte, w[6]));
}
__device__ __forceinline__ uint2 pack_run8(const uint32_t *w, uint32_t byte) {
    return make_uint2(mad_lo(w[1], byte, w[0]), mad_lo(w[3], byte, w[2]));
}

__device__ __forceinline__ void unpack16(const uint4 c, uint32_t *w) {
    w[0] = __byte_perm(c.x, 0, 0x4140);
    w[1] = __byte_perm(c.x, 0, 0x4342);
    w[2] = __byte_perm(c.y, 0, 0x4140);
    w[3] = __byte_perm(c.y, 0, 0x4342);
    w[4] = __byte_perm(c.z, 0, 0x4140);
    w[5] = __byte_perm(c.z, 0, 0x4342);
    w[6] = __byte_perm(c.w, 0, 0x4140);
    w[7] = __byte_perm(c.w, 0, 0x4342);
}

__device__ __forceinline__ void unpack8(const uint2 c, uint32_t *w) {
    w[0] = __byte_perm(c.x, 0, 0x4140);
    w[1] = __byte_perm(c.x, 0, 0x4342);
    w[2] = __byte_perm(c.y, 0, 0x4140);
    w[3] = __byte_perm(c.y, 0, 0x4342);
}

__device__ __forceinline__ uint2 pack8(const uint32_t *w) {
    return make_uint2(__byte_perm(w[0], w[1], 0x6420), __byte_perm(w[2], w[3], 0x6420));
}

__device__ __forceinline__ uint4 pack16(const uint32_t *w) {
    return make_uint4(__byte_perm(w[0], w[1], 0x6420), __byte_perm(w[2], w[3], 0x6420),
                      __byte_perm(w[4], w[5], 0x6420), __byte_perm(w[6], w[7], 0x6420));
}

// The start and length of scan line `line` of direction (dy, dx): rows run
// along x, columns along y, and a diagonal enters from the first row it meets
// (line < W) or from the side column it meets.
__host__ __device__ __forceinline__ int line_start(int line, int dy, int dx, int W, int H, int *y0,
                                          int *x0) {
    if (dy == 0) {
        *y0 = line;
        *x0 = dx > 0 ? 0 : W - 1;
        return W;
    }
    if (dx == 0) {
        *x0 = line;
        *y0 = dy > 0 ? 0 : H - 1;
        return H;
    }
    if (line < W) {
        *x0 = line;
        *y0 = dy > 0 ? 0 : H - 1;
    } else {
        *x0 = dx > 0 ? 0 : W - 1;
        const int k = line - W + 1;
        *y0 = dy > 0 ? k : H - 1 - k;
    }
    const int rows = dy > 0 ? H - *y0 : *y0 + 1;
    const int columns = dx > 0 ? W - *x0 : *x0 + 1;
    return min(rows, columns);
}

// 16-byte global -> shared copies that complete asynchronously (cp.async);
// src_size 0 zero-fills without reading.
__device__ __forceinline__ void copy16_async(void *shared, const void *global, bool valid) {
    const unsigned address = (unsigned)__cvta_generic_to_shared(shared);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(address), "l"(global),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void copy8_async(void *shared, const void *global, bool valid) {
    const unsigned address = (unsigned)__cvta_generic_to_shared(shared);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(address), "l"(global),
                 "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void copy_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void copy_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Adds four u16x2 words (eight u16 values below 1024) into 16 bytes of an
// aggregate volume in L2: a vector f16x2 reduction on their bit patterns,
// which for subnormals kept as such (.noftz) is the integer add.
__device__ __forceinline__ void add_sums16(void *global, uint32_t a, uint32_t b, uint32_t c,
                                           uint32_t d) {
    asm volatile("red.relaxed.gpu.global.add.noftz.v4.f16x2 [%0], {%1, %2, %3, %4};\n" ::"l"(global),
                 "r"(a), "r"(b), "r"(c), "r"(d)
                 : "memory");
}

// ---- bulk tensor copies of the cost stream ----
// The cost volume [H][W][D] bytes seen four ways, one per kind of scan line:
// a 3-D tensor map of (d, s, q) at byte q D + s S + d, S the line's step in
// bytes (D for rows, W D for columns, (W + 1) D and (W - 1) D for the two
// diagonals), s < 8 and q < W H a pixel index. A box of (D, 8, 1) at (0, 0,
// q) is the [8][D] tile of the 8 steps of a line from pixel q on, in
// ascending pixel order: a line going forward (dx > 0 on rows, dy > 0 on the
// others) has step base + i in row i from the pixel of step base, one going
// back row 7 - i from the pixel of step base + 7. A copy is only issued for 8
// steps that all lie on the line, so every byte it reads is the volume's.
// The maps are encoded on the host for each launch.
struct CostMaps {
    CUtensorMap row, column, diagonal, anti;
};

// Waits of the path scan on its copies that gave up (after kTileWaitNs of
// the global timer): 0 unless a copy never landed.
static __device__ unsigned int g_path_wait_failures;
constexpr uint64_t kTileWaitNs = 1000000000ull;
// Tiles in flight or being read, a line (2 and 3 measured no faster).
constexpr int kTileStages = 4;

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned shared_address(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void barrier_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(shared_address(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void barrier_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void barrier_expect(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(shared_address(bar)),
                 "r"(bytes)
                 : "memory");
}
// True once the barrier has completed the phase of `parity`; false when it
// has not after kTileWaitNs (the clock is read every 256 tries).
__device__ __forceinline__ bool barrier_wait(uint64_t *bar, unsigned parity) {
    const unsigned address = shared_address(bar);
    uint64_t start = 0;
    for (unsigned i = 0;; ++i) {
        unsigned done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            "selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(address), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255u) == 0) {
            const uint64_t now = global_ns();
            if (i == 0) start = now;
            else if (now - start > kTileWaitNs) return false;
        }
    }
}
// The tile of a map at (0, 0, pixel) into this CTA's shared memory,
// completing on `bar` (no multicast: the volume is this GPU's own memory).
__device__ __forceinline__ void tile_copy(void *to, const CUtensorMap *map, int pixel,
                                          uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(shared_address(to)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(0), "r"(pixel), "r"(shared_address(bar))
        : "memory");
}

// Where the aggregate volume of the summing path scan keeps disparity
// position j of a pixel (j in the span-16 permuted order of span_disparity,
// lane j / 16 holding positions 16 * lane ..): the lane's words 0-3 (positions
// 0-7 of its run) at u16 8 * lane + (j % 8), its words 4-7 at D / 2 + 8 * lane
// + (j % 8).
__host__ __device__ constexpr int sum_position(int disparities, int j) {
    return (j % 16 < 8 ? 0 : disparities / 2) + 8 * (j / 16) + j % 8;
}

// The lines of one warp: G lanes per line, WORDS (4, 8 or 16) u16x2 words,
// so 2 x WORDS disparities, per lane. `ring` is this thread's first slot of
// the warp's kPrefetch x THREADS slots of 2 x WORDS bytes. SPAN (8 or 16, at
// most 2 x WORDS): costs and path costs are in the permuted order of
// span_disparity, so within each run of SPAN disparities word k holds
// disparities (k, k + SPAN / 2) and its neighbours at d - 1 and d + 1 are the
// words k - 1 and k + 1, but for the first and last word of a run, whose
// outer neighbour lies in the next run (one byte permute each); SPAN 0:
// word k holds (2k, 2k + 1) and every neighbour is made by a byte permute.
//
// SUMS: instead of its own u8 volume, each direction adds its path costs into
// one u16 aggregate volume (zeroed before the launch) in the lane-split
// layout of sum_position, with 16-byte reductions: every direction's lane
// sends its words 0-3 and 4-7 as two reductions, so G lanes cover two runs of
// 16 * G contiguous bytes. The reductions are f16x2 adds on the u16 bit
// patterns: an integer n < 1024 is the f16 subnormal n * 2^-24, and the sum
// of subnormals below 2^-14 is exact with subnormals kept (.noftz), so the
// adds are the integer adds (8 directions x at most 127 = 1016).
//
// TILES (8 words a lane, span 16, every lane active): the blocks of 8 steps
// that every line of the warp covers take their costs from bulk tensor copies
// (CostMaps) instead of per-lane copies: one lane of each line asks for a
// block's [8][D] tile kTileStages - 1 blocks ahead into a stage of `tiles`,
// each stage completing on its own barrier of `bars` (LINES arrivals a
// phase); the other blocks (each line's last ones) keep the per-lane copies,
// their ring in the first stage's room once every tile has been read.
template <int G, int WORDS, bool FULL, int THREADS, int SPAN = 0, bool SUMS = false,
          bool TILES = false>
__device__ __forceinline__ void follow_lines(const uint8_t *__restrict__ costs,
                                             uint8_t *__restrict__ out, const PathSetup &s,
                                             int p, int line, int member, void *ring_base,
                                             const CostMaps *maps = nullptr,
                                             uint8_t *tiles = nullptr, uint64_t *bars = nullptr) {
    static_assert(WORDS == 4 || WORDS == 8 || WORDS == 16, "4, 8 or 16 words a lane");
    static_assert(SPAN == 0 || (SPAN >= 8 && SPAN <= 2 * WORDS && (2 * WORDS) % SPAN == 0),
                  "a lane holds whole permuted runs");
    static_assert(!SUMS || WORDS == 8, "the aggregate layout has 16 disparities a lane");
    static_assert(!TILES || (WORDS == 8 && SPAN == 16 && FULL), "tiles of 16 bytes a lane");
    constexpr int BYTES = 2 * WORDS;             // a lane's disparities, one byte each
    constexpr int PIECE = BYTES < 16 ? BYTES : 16;  // bytes of one async copy
    constexpr int PIECES = BYTES / PIECE;
    constexpr int RUN = SPAN / 2;                // words of a permuted run
    constexpr int LINES = 32 / G;                // lines of a warp
    using Piece = typename std::conditional<PIECE == 16, uint4, uint2>::type;
    Piece *ring = static_cast<Piece *>(ring_base);
    const int dy = s.dy[p], dx = s.dx[p];
    const int W = s.width, H = s.height, D = s.disparities;
    int y0 = 0, x0 = 0, length = 0;
    if (line < s.lines[p]) length = line_start(line, dy, dx, W, H, &y0, &x0);
    const bool active = FULL || member * BYTES < D;
    const ptrdiff_t stride = ((ptrdiff_t)dy * W + dx) * D;  // |stride| <= 4097 x 256
    const int stride32 = (int)stride;
    const size_t at = ((size_t)y0 * W + x0) * D + member * BYTES;
    const uint8_t *ahead = costs + at;
    // SUMS: lane `member`'s words 0-3 at u16 (pixel * D + 8 * member), 4-7 D bytes on.
    uint8_t *dst = SUMS ? out + 2 * (((size_t)y0 * W + x0) * D + 8 * member)
                        : out + (size_t)p * s.volume + at;
    const int steps = (int)__reduce_max_sync(kFullMask, (unsigned)length);
    const int shortest = (int)__reduce_min_sync(kFullMask, (unsigned)length);
    // Blocks all of whose steps every line of the warp has, with the copies they
    // start (kPrefetch - 1 steps ahead), run without the checks: all blocks of the
    // rows and columns but the last, most of each diagonal's.
    auto unchecked_at = [&](int base) { return FULL && base + 2 * kPrefetch - 1 <= shortest; };

    uint32_t r[WORDS];
#pragma unroll
    for (int k = 0; k < WORDS; ++k) r[k] = active ? 0u : kInf2;
    uint32_t m2 = 0, j2 = (uint32_t)s.p2 * 0x10001u;
    const uint32_t p1x2 = (uint32_t)s.p1 * 0x10001u, p2x2 = (uint32_t)s.p2 * 0x10001u;
    const uint32_t keep_left = member == 0 ? 0u : s.one, edge_left = member == 0 ? kInf2 : 0u;
    const uint32_t keep_right = member == G - 1 ? 0u : s.one;
    const uint32_t edge_right = member == G - 1 ? kInf2 : 0u;
    const uint32_t byte = s.one << 8;  // 256, at run time (pack_run16)

    auto fetch = [&](int slot, bool valid) {
#pragma unroll
        for (int c = 0; c < PIECES; ++c) {
            Piece *to = ring + (slot * PIECES + c) * THREADS;
            const uint8_t *from = valid ? ahead + PIECE * c : costs;
            if (PIECE == 16) copy16_async(to, from, valid);
            else copy8_async(to, from, valid);
        }
        copy_commit();
        ahead = advance(ahead, stride32, s.one);
    };
    // The ring's first kPrefetch - 1 slots take steps base .. base + kPrefetch - 2.
    auto prime = [&](int base) {
        ahead = costs + at + (ptrdiff_t)base * stride;
#pragma unroll
        for (int i = 0; i < kPrefetch - 1; ++i) fetch(i, active && base + i < length);
    };
    if (!(TILES && unchecked_at(0))) prime(0);

    // One step from this step's costs: the recurrence on every word, the
    // store (or reduction) of the path costs where `store`, the line's minimum.
    auto advance_step = [&](const uint32_t(&cost)[WORDS], bool store) {
        // The line's first and last lanes see +inf past the ends: x keep + edge
        // as multiply-adds (keep 0 and edge kInf2 there, 1 and 0 elsewhere).
        const uint32_t from_left =
            mad_lo(__shfl_up_sync(kFullMask, r[WORDS - 1], 1), keep_left, edge_left);
        const uint32_t from_right =
            mad_lo(__shfl_down_sync(kFullMask, r[0], 1), keep_right, edge_right);
        const uint32_t negm2 = 0u - m2;
        uint32_t below[WORDS], above[WORDS];  // word k's values at d - 1 and at d + 1
        if constexpr (SPAN != 0) {
#pragma unroll
            for (int k = 0; k < WORDS; ++k) {
                const int first = k - k % RUN, last = first + RUN - 1;
                if (k == first)  // (the run before's last disparity, this run's middle - 1)
                    below[k] = __byte_perm(first ? r[first - 1] : from_left, r[last], 0x5432);
                else
                    below[k] = r[k - 1];
                if (k == last)  // (this run's middle, the next run's first disparity)
                    above[k] = __byte_perm(r[first], last + 1 < WORDS ? r[last + 1] : from_right,
                                           0x5432);
                else
                    above[k] = r[k + 1];
            }
        } else {
            uint32_t shifted[WORDS + 1];  // shifted[k]: the (d - 1) values of word k
            shifted[0] = __byte_perm(from_left, r[0], 0x5432);
#pragma unroll
            for (int k = 1; k < WORDS; ++k) shifted[k] = __byte_perm(r[k - 1], r[k], 0x5432);
            shifted[WORDS] = __byte_perm(r[WORDS - 1], from_right, 0x5432);
#pragma unroll
            for (int k = 0; k < WORDS; ++k) {
                below[k] = shifted[k];
                above[k] = shifted[k + 1];
            }
        }
#pragma unroll
        for (int k = 0; k < WORDS; ++k) {
            // min(prev, neighbours + p1, m + p2) - m + cost: neighbours + p1
            // (a multiply-add by a run-time 1, on the FMA pipe beside the
            // integer pipe's min and permute work) <= 0x7FFF + 79 stays in its
            // half; t + cost + (-m) is one three-input add taken mod 2^32,
            // which equals t - m + cost, whose halves neither borrow nor carry
            // (t >= m in both). It measured 3% faster than two multiply-adds.
            const uint32_t neighbour = vmin2(below[k], above[k]);
            const uint32_t raised = mad_lo(neighbour, s.one, p1x2);
            const uint32_t t = __vimin3_u16x2(r[k], j2, raised);
            const uint32_t value = t + cost[k] + negm2;
            r[k] = (FULL || active) ? value : kInf2;
        }
        if (store) {
            if constexpr (SUMS) {
                add_sums16(dst, r[0], r[1], r[2], r[3]);
                add_sums16(dst + D, r[4], r[5], r[6], r[7]);
            } else {
#pragma unroll
                for (int c = 0; c < PIECES; ++c) {
                    if constexpr (PIECE == 16)
                        __stcs(reinterpret_cast<uint4 *>(dst + 16 * c),
                               SPAN ? pack_run16(r + 8 * c, byte) : pack16(r + 8 * c));
                    else
                        __stcs(reinterpret_cast<uint2 *>(dst + 8 * c),
                               SPAN ? pack_run8(r + 4 * c, byte) : pack8(r + 4 * c));
                }
            }
        }
        dst = advance(dst, SUMS ? 2 * stride32 : stride32, s.one);
        // The lowest path cost over the line's disparities: a shallow tree
        // over the lane's words, both halves folded into each half, then
        // over the line's G lanes a shuffle tree (one warp-wide reduction
        // when the line has the whole warp; a reduction under each group's
        // own mask measured slower than the shuffles).
        constexpr int PARTS = (WORDS + 2) / 3;
        uint32_t part[PARTS];
#pragma unroll
        for (int k = 0; k < WORDS; k += 3)
            part[k / 3] = k + 2 < WORDS ? __vimin3_u16x2(r[k], r[k + 1], r[k + 2])
                                        : (k + 1 < WORDS ? vmin2(r[k], r[k + 1]) : r[k]);
        uint32_t lowest = part[0];
#pragma unroll
        for (int k = 1; k < PARTS; k += 2)
            lowest = k + 1 < PARTS ? __vimin3_u16x2(lowest, part[k], part[k + 1])
                                   : vmin2(lowest, part[k]);
        lowest = vmin2(lowest, __byte_perm(lowest, 0, 0x1032));
        if constexpr (G == 32) {
            m2 = __reduce_min_sync(kFullMask, lowest);
        } else {
            lowest = line_minimum<G>(lowest);
            m2 = lowest;
        }
        j2 = m2 + p2x2;
    };
    // One block of kPrefetch steps from `base` from the ring. CHECKED: the steps
    // test the warp's last step and each line's end; without, every line of the
    // warp covers the block and the copies it starts (FULL: every lane active).
    auto block = [&](const int base, auto checked) {
        constexpr bool CHECKED = decltype(checked)::value;
#pragma unroll
        for (int i = 0; i < kPrefetch; ++i) {
            const int step = base + i;
            if (CHECKED && step >= steps) break;  // uniform across the warp
            // the copy of step + kPrefetch - 1 goes to the slot read last step
            fetch((i + kPrefetch - 1) % kPrefetch,
                  !CHECKED || (active && step + kPrefetch - 1 < length));
            copy_wait<kPrefetch - 1>();
            uint32_t cost[WORDS];
#pragma unroll
            for (int c = 0; c < PIECES; ++c) {
                if constexpr (PIECE == 16) {
                    if constexpr (SPAN != 0) unpack_run16(ring[(i * PIECES + c) * THREADS], cost + 8 * c);
                    else unpack16(ring[(i * PIECES + c) * THREADS], cost + 8 * c);
                } else {
                    if constexpr (SPAN != 0) unpack_run8(ring[(i * PIECES + c) * THREADS], cost + 4 * c);
                    else unpack8(ring[(i * PIECES + c) * THREADS], cost + 4 * c);
                }
            }
            advance_step(cost, !CHECKED || (active && step < length));
        }
    };

    if constexpr (TILES) {
        // Tile rows ascend in pixel index: step base + i is row i going
        // forward, row 7 - i going back. The unchecked blocks are the first
        // `tiled` ones; block b's tile is in stage b % kTileStages, asked for
        // kTileStages - 1 blocks ahead.
        const bool forward = dy > 0 || (dy == 0 && dx > 0);
        const int slot_line = (threadIdx.x % 32) / G;
        const CUtensorMap *map = dy == 0 ? &maps->row
                                 : dx == 0 ? &maps->column
                                 : dx == dy ? &maps->diagonal : &maps->anti;
        const int start = y0 * W + x0, step_pixels = dy * W + dx;  // pixel indices < 2^31
        const int tiled = shortest >= 2 * kPrefetch - 1 ? (shortest - (2 * kPrefetch - 1)) / kPrefetch + 1 : 0;
        auto tile_of = [&](int stage) { return tiles + (stage * LINES + slot_line) * kPrefetch * D; };
        auto issue = [&](int b) {  // block b into its stage
            if (member == 0) {
                const int first = forward ? b * kPrefetch : b * kPrefetch + kPrefetch - 1;
                uint64_t *bar = bars + b % kTileStages;
                barrier_expect(bar, (unsigned)(kPrefetch * D));
                tile_copy(tile_of(b % kTileStages), map, start + first * step_pixels, bar);
            }
        };
        auto wait_block = [&](int b) {
            return barrier_wait(bars + b % kTileStages, (unsigned)(b / kTileStages) & 1u);
        };
        for (int b = 0; b < tiled && b < kTileStages - 1; ++b) issue(b);
        for (int b = 0; b < tiled; ++b) {
            __syncwarp();  // every lane has read block b - 1's stage
            if (b + kTileStages - 1 < tiled) issue(b + kTileStages - 1);
            if (!__all_sync(kFullMask, wait_block(b))) {
                // A copy that never landed: count it, give the others in
                // flight the same time, and leave this warp's lines unfinished.
                if ((threadIdx.x % 32) == 0) atomicAdd(&g_path_wait_failures, 1u);
                for (int k = b + 1; k < tiled && k < b + kTileStages; ++k) wait_block(k);
                return;
            }
            const uint4 *tile = reinterpret_cast<const uint4 *>(tile_of(b % kTileStages)) + member;
            if (forward) {
#pragma unroll
                for (int i = 0; i < kPrefetch; ++i) {
                    uint32_t cost[WORDS];
                    unpack_run16(tile[i * G], cost);
                    advance_step(cost, true);
                }
            } else {
#pragma unroll
                for (int i = 0; i < kPrefetch; ++i) {
                    uint32_t cost[WORDS];
                    unpack_run16(tile[(kPrefetch - 1 - i) * G], cost);
                    advance_step(cost, true);
                }
            }
        }
        // The rest from the ring, which shares the first stage's room: every
        // tile has landed and been read (the barrier below) before it refills.
        __syncwarp();
        for (int base = tiled * kPrefetch; base < steps; base += kPrefetch) {
            if (base == tiled * kPrefetch && tiled > 0) prime(base);
            block(base, std::true_type());
        }
    } else {
        for (int base = 0; base < steps; base += kPrefetch) {
            if (unchecked_at(base)) block(base, std::false_type());
            else block(base, std::true_type());
        }
    }
    copy_wait<0>();
}

// The scan line of direction (dy, dx) with rank `rank` when the lines are
// ordered by length, longest first, so the lines a warp follows together are
// alike in length. Rows and columns are all alike. A diagonal line either
// starts on the first row it meets, at a distance j = 1..W from the side it
// runs away from (length min(H, j)), or on a side column at row offset
// k = 1..H-1 (length min(H - k, W)).
__host__ __device__ __forceinline__ int ranked_line(int rank, int dy, int dx, int W, int H) {
    if (dy == 0 || dx == 0) return rank;
    const int full = (W > H ? W - H : H - W) + 1;  // lines of the greatest length
    int j = 0, k = 0;                              // first-row distance, or side offset
    if (rank < full) {
        if (W >= H) j = W - rank;
        else if (rank < full - 1) k = rank + 1;
        else j = W;
    } else {
        const int q = rank - full;
        const int len = min(W, H) - 1 - q / 2;
        if (q % 2 == 0) j = len;
        else k = H - len;
    }
    if (j > 0) return dx > 0 ? W - j : j - 1;
    return W - 1 + k;
}


// One warp's lines: warp `warp` of the pair's path launch, lane `lane`.
// Rows, then columns, then the diagonals of all four directions by rank.
// `ring`: this lane's first slot of the warp's kPrefetch x 32 slots of
// 2 x WORDS bytes (in pieces of at most 16 bytes, strided by 32 lanes).
template <int G, int WORDS, bool FULL, int SPAN = 0, bool SUMS = false, bool TILES = false>
__device__ __forceinline__ void path_warp(const uint8_t *__restrict__ costs,
                                          uint8_t *__restrict__ paths_out, const PathSetup &s,
                                          int warp, int lane, void *ring,
                                          const CostMaps *maps = nullptr, uint8_t *tiles = nullptr,
                                          uint64_t *bars = nullptr) {
    int slot = 0;
    while (warp >= s.first_warp[slot + 1]) ++slot;
    int p, group;
    if (slot < s.straight) {  // rows and columns, direction by direction
        p = s.order[slot];
        group = warp - s.first_warp[slot];
    } else {                  // diagonals interleaved, longest first
        const int w = warp - s.first_warp[s.straight];
        const int diagonals = s.paths - s.straight;
        p = s.order[s.straight + w % diagonals];
        group = w / diagonals;
    }
    const int rank = group * (32 / G) + lane / G;
    const int line =
        rank < s.lines[p] ? ranked_line(rank, s.dy[p], s.dx[p], s.width, s.height) : rank;
    follow_lines<G, WORDS, FULL, 32, SPAN, SUMS, TILES>(costs, paths_out, s, p, line, lane % G,
                                                        ring, maps, tiles, bars);
}

// Lanes per pixel (selection) or per line (paths with 16 disparities a lane),
// 16 disparities each: a power of two.
__host__ __device__ inline int group_lanes(int disparities) {
    return disparities <= 64 ? 4 : (disparities <= 128 ? 8 : 16);
}

// Lanes per scan line with `words` u16x2 words (2 x words disparities) a
// lane: the power of two that covers the disparities.
__host__ __device__ inline int path_lanes(int disparities, int words) {
    int g = 1;
    while (g * 2 * words < disparities) g *= 2;
    return g;
}

// ---------------------------------------------------------------- select
// Which disparity half h of word k of a selection lane's 16 holds (j = 2k +
// h): the volumes' bytes 2k and 2k + 1 (span_disparity), or for the summing
// scan's aggregate (PATHS -1) the scan lane's word k, (k, k + 8); and where
// disparity d lies in the per-pixel row of 16-value runs.
template <int PATHS, int SPAN>
__host__ __device__ constexpr int select_disparity(int j) {
    return PATHS == -1 ? (j % 16) / 2 + 8 * (j % 2) + 16 * (j / 16) : span_disparity(SPAN, j);
}
template <int PATHS, int SPAN>
__host__ __device__ constexpr int select_position(int d) {
    return PATHS == -1 ? 16 * (d / 16) + 2 * (d % 8) + (d % 16) / 8 : span_position(SPAN, d);
}
// Winner, uniqueness and subpixel (lib/nx_stereo.ex:608-641). A group of G
// lanes takes one pixel, each lane 16 disparities, so a warp takes 32 / G
// pixels. values = sum of the path costs + 0x8000 past x; the winner is the
// lowest (value << 16 | d), so ties go to the lowest d; `second` is the
// lowest value more than one disparity from the winner; the f32 steps are
// rounded one at a time in the reference's order. Two path volumes add as
// bytes without carry (127 + 127 < 256) before widening to u16x2.
//
// Either `keys` receives each pixel's key (0xFFFFFFFF where rejected) for the
// per-row check, or, with `right_map`, each accepted match goes straight into
// the right image's map: right_map[y][x - d] = min of (key & 0xFFFF0000) |
// (65535 - d) (lib/nx_stereo.ex:646-664). `values_of` is 128 / G rows of 256
// values in shared memory.
// SPAN: the path volumes' disparity order (span_disparity).
// PATHS 0: u16 sums in the volumes' order, not path volumes; -1: u16 sums in
// the lane-split layout of sum_position (the summing path scan's output).
template <int G, int PATHS, int SPAN = 0>
__device__ __forceinline__ void select_pixels(const void *__restrict__ source, int width,
                                              int height, int disparities, size_t volume,
                                              float uniqueness, float *__restrict__ disparity,
                                              uint32_t *__restrict__ keys,
                                              uint32_t *__restrict__ right_map, size_t block,
                                              uint16_t (*values_of)[256], uint32_t one) {
    constexpr int PIXELS = 128 / G;  // per 128 threads
    const int slot = (threadIdx.x % 128) / G, member = threadIdx.x % G;
    const size_t pixel = block * PIXELS + slot;
    const bool valid = pixel < (size_t)width * height;
    const int D = disparities;
    const bool active = valid && member * 16 < D;
    // A 32-bit remainder: pixel < 2^32, as 2^32 pixels' volumes (at least
    // 16 bytes a pixel) would not fit in device memory.
    const int x = valid ? (int)((uint32_t)pixel % (uint32_t)width) : 0;
    const int d0 = member * 16;
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = 0;
    if (active) {
        const size_t at = pixel * D + d0;
        if (PATHS <= 0) {
            const uint16_t *base = static_cast<const uint16_t *>(source);
            const uint4 *sums = reinterpret_cast<const uint4 *>(
                PATHS == 0 ? base + at : base + pixel * D + 8 * member);
            const uint4 a = __ldcg(sums);
            const uint4 b = __ldcg(PATHS == 0 ? sums + 1 : sums + D / 16);
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
            v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
        } else {
            const uint8_t *volumes = static_cast<const uint8_t *>(source) + at;
            uint4 loaded[PATHS > 0 ? PATHS : 1];
#pragma unroll
            for (int p = 0; p < PATHS; ++p)  // every volume's load in flight at once
                loaded[p] = __ldcs(reinterpret_cast<const uint4 *>(volumes + p * volume));
            // The adds as multiply-adds by a run-time 1 (`one`), on the FMA pipe:
            // the byte-wise pair sums carry nowhere (127 + 127 < 256), the u16
            // sums neither (8 x 127 + 0x8000 < 0x10000).
#pragma unroll
            for (int p = 0; p < PATHS; p += 2) {
                const uint4 a = loaded[p];
                uint4 both = a;
                if (p + 1 < PATHS) {
                    const uint4 b = loaded[p + 1];
                    both = make_uint4(mad_lo(a.x, one, b.x), mad_lo(a.y, one, b.y),
                                      mad_lo(a.z, one, b.z), mad_lo(a.w, one, b.w));
                }
                uint32_t pair[8];
                unpack16(both, pair);
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = p == 0 ? pair[k] : mad_lo(pair[k], one, v[k]);
            }
        }
        if (x < d0 + 15) {  // disparities past the left edge lose
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int lo = d0 + select_disparity<PATHS, SPAN>(2 * k);
                const int hi = d0 + select_disparity<PATHS, SPAN>(2 * k + 1);
                v[k] += (lo > x ? 0x8000u : 0u) | (hi > x ? 0x80000000u : 0u);
            }
        }
        *reinterpret_cast<uint4 *>(&values_of[slot][d0]) = make_uint4(v[0], v[1], v[2], v[3]);
        *reinterpret_cast<uint4 *>(&values_of[slot][d0 + 8]) = make_uint4(v[4], v[5], v[6], v[7]);
    }
    uint32_t best = 0xFFFFFFFFu;
    if (active) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t lo = d0 + select_disparity<PATHS, SPAN>(2 * k);
            const uint32_t hi = d0 + select_disparity<PATHS, SPAN>(2 * k + 1);
            const uint32_t d = lo | (hi << 16);
            best = min(best, min(__byte_perm(v[k], d, 0x1054), __byte_perm(v[k], d, 0x3276)));
        }
    }
#pragma unroll
    for (int offset = G / 2; offset >= 1; offset /= 2)
        best = min(best, __shfl_xor_sync(kFullMask, best, offset));
    const uint32_t minimum = best >> 16;
    const int winner = (int)(best & 0xFFFFu);
    uint32_t second = 0xFFFFFFFFu;
    if (active) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int lo = d0 + select_disparity<PATHS, SPAN>(2 * k);
            const int hi = d0 + select_disparity<PATHS, SPAN>(2 * k + 1);
            // d outside [winner - 1, winner + 1]
            if ((unsigned)(lo - winner + 1) > 2u) second = min(second, v[k] & 0xFFFFu);
            if ((unsigned)(hi - winner + 1) > 2u) second = min(second, v[k] >> 16);
        }
    }
#pragma unroll
    for (int offset = G / 2; offset >= 1; offset /= 2)
        second = min(second, __shfl_xor_sync(kFullMask, second, offset));
    __syncwarp();
    if (member != 0 || !valid) return;
    const int below = max(winner - 1, 0), above = min(winner + 1, D - 1);
    const uint32_t lower = values_of[slot][select_position<PATHS, SPAN>(below)];
    const uint32_t upper = values_of[slot][select_position<PATHS, SPAN>(above)];
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
    if (keys) keys[pixel] = accepted ? ((minimum << 16) | (uint32_t)winner) : kInvalidKey;
    if (right_map && accepted && x - winner >= 0)  // a winner is at most x
        atomicMin(right_map + (pixel - winner), (minimum << 16) | (65535u - (uint32_t)winner));
}

// ---------------------------------------------------------------- check
// OpenCV's left-right check (lib/nx_stereo.ex:643-683), one block per row:
// the right map is the per-row atomicMin of (key & 0xFFFF0000) | (65535 - d)
// at x - d, so the cheapest match wins and ties go to the larger d.
// A match survives unless both floor(d) and ceil(d) disagree: the right map
// at x - d holds a match more than one disparity away. `right` is the row's
// right map (shared or global memory).
template <bool GLOBAL>  // the map in global memory, written earlier in the same launch
__device__ __forceinline__ float consistent_value(float value, int x, int width,
                                                  const uint32_t *right) {
    int low = (int)floorf(value), high = (int)ceilf(value);
    bool rejected = true;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        int d = k == 0 ? low : high;
        int rx = x - d;
        bool inside = rx >= 0 && rx < width;
        const uint32_t *at = right + min(max(rx, 0), width - 1);
        uint32_t found = GLOBAL ? __ldcg(at) : *at;
        int right_d = 65535 - (int)(found & 0xFFFFu);
        bool disagrees = inside && found != kInvalidKey && abs(right_d - d) > 1;
        rejected = rejected && disagrees;
    }
    return (value >= 0.0f && !rejected) ? value : -1.0f;
}

// `right` is the block's shared array of `width` words.
__device__ __forceinline__ void consistency_row(const float *__restrict__ disparity,
                                                const uint32_t *__restrict__ keys, int width,
                                                float *__restrict__ checked, int y,
                                                uint32_t *right) {
    const size_t row = (size_t)y * width;
    for (int x = threadIdx.x; x < width; x += blockDim.x) right[x] = kInvalidKey;
    __syncthreads();
    for (int x = threadIdx.x; x < width; x += blockDim.x) {
        uint32_t key = __ldcg(keys + row + x);
        if (key == kInvalidKey) continue;
        int winner = (int)(key & 0xFFFFu);
        if (x - winner < 0) continue;  // a winner is at most x (past-edge costs lose)
        atomicMin(&right[x - winner], (key & 0xFFFF0000u) | (65535u - (uint32_t)winner));
    }
    __syncthreads();
    for (int x = threadIdx.x; x < width; x += blockDim.x)
        checked[row + x] = consistent_value<false>(__ldcg(disparity + row + x), x, width, right);
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

// The middle of nine values by the network; then, for Stage.Disparity,
// disparity <= 0 becomes -1.
__device__ __forceinline__ float median_of_nine(float *v, int stage_mask) {
    exchange(v[1], v[2]); exchange(v[4], v[5]); exchange(v[7], v[8]);
    exchange(v[0], v[1]); exchange(v[3], v[4]); exchange(v[6], v[7]);
    exchange(v[1], v[2]); exchange(v[4], v[5]); exchange(v[7], v[8]);
    exchange(v[0], v[3]); exchange(v[5], v[8]); exchange(v[4], v[7]);
    exchange(v[3], v[6]); exchange(v[1], v[4]); exchange(v[2], v[5]);
    exchange(v[4], v[7]); exchange(v[4], v[2]); exchange(v[6], v[4]);
    exchange(v[4], v[2]);
    float out = v[4];
    if (stage_mask && !(out > 0.0f)) out = -1.0f;
    return out;
}

__device__ __forceinline__ void median_at(const float *__restrict__ image, int width,
                                          int height, int stage_mask,
                                          float *__restrict__ filtered, int x, int y) {
    if (x >= width) return;
    float v[9];
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            int sy = min(max(y + dy, 0), height - 1), sx = min(max(x + dx, 0), width - 1);
            v[(dy + 1) * 3 + dx + 1] = __ldcg(image + (size_t)sy * width + sx);
        }
    filtered[(size_t)y * width + x] = median_of_nine(v, stage_mask);
}

}  // namespace nxs
