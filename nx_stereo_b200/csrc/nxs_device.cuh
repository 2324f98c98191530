// Device helpers shared by the kernels: packed u16x2 arithmetic for the path
// recurrence and explicitly rounded f32 operations for the steps whose f32
// results must match the reference's operation order bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nxs {

constexpr unsigned kFullMask = 0xFFFFFFFFu;
constexpr uint32_t kInvalidKey = 0xFFFFFFFFu;
// A path cost no real one reaches (real ones are at most p2 + 48 <= 127); it
// stays below 0x8000 after adding p1, so packed adds never carry.
constexpr uint32_t kInf16 = 0x7FFFu;
constexpr uint32_t kInf2 = 0x7FFF7FFFu;

// Per-halfword minimum of two u16x2 words (PTX min.u16x2, sm_90+).
__device__ __forceinline__ uint32_t vmin2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

// f32 operations, each rounded to nearest even on its own: never contracted
// into a fused multiply-add, so results equal the reference's evaluation.
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

}  // namespace nxs
