// Device helpers shared by the kernels: packed u16x2 arithmetic for the path
// recurrence and explicitly rounded f32 operations for the steps whose f32
// results must match the reference's operation order bit for bit.
#pragma once

#include <cstdint>
#include <utility>

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

// Programmatic dependent launch: a kernel launched by launch_after is launched
// as the last block of the kernel before it on the stream exits, before that
// grid's completion is processed, so the launch gap between stages overlaps
// the previous stage's end. Such a kernel calls follow_previous_grid() before
// it touches global memory: it waits until the grid before it has completed
// and its writes are visible (griddepcontrol.wait, which returns at once when
// nothing precedes the kernel programmatically). Since every kernel waits at
// its top, a successor never runs ahead of any earlier kernel's writes, nor
// overwrites what an earlier kernel still reads. No kernel signals its
// successor earlier (griddepcontrol.launch_dependents): blocks launched early
// sat resident while they waited, which with many streams in flight held SMs
// other streams' kernels could use (serving saturation 2,455 -> 2,090 pairs/s).
__device__ __forceinline__ void follow_previous_grid() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... Params, typename... Args>
inline cudaError_t launch_after(void (*kernel)(Params...), dim3 grid, dim3 block, size_t shared,
                                cudaStream_t stream, Args &&...args) {
    cudaLaunchConfig_t config = {};
    config.gridDim = grid;
    config.blockDim = block;
    config.dynamicSmemBytes = shared;
    config.stream = stream;
    cudaLaunchAttribute attribute[1];
    attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attribute[0].val.programmaticStreamSerializationAllowed = 1;
    config.attrs = attribute;
    config.numAttrs = 1;
    return cudaLaunchKernelEx(&config, kernel, std::forward<Args>(args)...);
}

}  // namespace nxs
