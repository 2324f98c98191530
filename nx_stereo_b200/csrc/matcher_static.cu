// NxStereo.sgm/3 on device buffers with no device allocation at all: the
// matcher's scratch (the cost volume, the path volumes, and the selected
// disparity and winner keys of each pixel; the census codes never leave the
// census + costs kernel's shared memory) lives in one fixed array of this file
// instead of memory obtained from cudaMalloc.
//
// Who needs this: callers that must not allocate device memory once running.
// A caller whose device memory is owned by another allocator (a framework's
// caching pool, a serving runtime that reserved the whole device at start-up)
// would see a direct cudaMalloc fail or fragment that pool; a latency-bound
// caller (a BEAM scheduler thread behind a NIF, a real-time capture loop)
// cannot afford cudaMalloc/cudaFree, which may synchronise the device and
// take milliseconds. Such callers pass their inputs and outputs and get the
// scratch from here.
//
// The array holds kStaticScratchBytes on every device that loads this library,
// for as long as the process lives. All calls on a device share it: calls
// whose work overlaps on that device (two streams, or two host threads) race
// on the same bytes and must be serialised by the caller. No byte of it needs
// to start at zero: each call writes every scratch byte before reading it.
#include <cstdio>
#include <mutex>

#include "../../include/nx_stereo_b200.h"
#include "nxs_kernels.h"

namespace {

// 64 MiB: enough for the 8-path matcher on pairs up to about 7 million
// pixel-disparities, e.g. 364x272 at 64 disparities.
constexpr size_t kStaticScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char static_scratch[kStaticScratchBytes];

std::mutex setup_lock;
void *scratch_address[kMaxDevices] = {};

void write_error(char *error, size_t error_len, const char *text) {
    if (!error || error_len == 0) return;
    snprintf(error, error_len, "%s", text);
}

}  // namespace

extern "C" nxs_status nxs_sgm_device_static(const uint8_t *d_left, const uint8_t *d_right,
                                            uint32_t width, uint32_t height,
                                            const nxs_sgm_params *params, float *d_disparity,
                                            void *stream, char *error, size_t error_len) {
    if (!d_left || !d_right || !d_disparity) {
        write_error(error, error_len, "a NULL image or disparity buffer");
        return NXS_BAD_ARGUMENT;
    }
    nxs_status status = nxs_sgm_check(params, width, height, error, error_len);
    if (status != NXS_OK) return status;
    const size_t needed = nxs::matcher_scratch_bytes(width, height, params->disparities);
    if (needed > kStaticScratchBytes) {
        char text[256];
        snprintf(text, sizeof text,
                 "a %ux%u pair at %u disparities needs %zu bytes of scratch; this entry point "
                 "has %zu (64 MiB): use nxs_sgm_device",
                 width, height, params->disparities, needed, kStaticScratchBytes);
        write_error(error, error_len, text);
        return NXS_BAD_ARGUMENT;
    }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess || device < 0 || device >= kMaxDevices) {
        write_error(error, error_len, e != cudaSuccess ? cudaGetErrorString(e)
                                                       : "device ordinal beyond 63");
        return NXS_CUDA_ERROR;
    }
    // Once per device, with that device current: the array's device address.
    // In host code `static_scratch` names a host-side stand-in, not device
    // memory, so kernels get this address instead. This first call on a device
    // also loads the array onto it, so it should come before any stream capture.
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> guard(setup_lock);
        if (!scratch_address[device]) {
            void *address = nullptr;
            e = cudaGetSymbolAddress(&address, static_scratch);
            if (e != cudaSuccess) {
                write_error(error, error_len, cudaGetErrorString(e));
                return NXS_CUDA_ERROR;
            }
            scratch_address[device] = address;
        }
        base = scratch_address[device];
    }
    nxs::MatcherScratch scratch =
        nxs::carve_matcher_scratch(base, width, height, params->disparities);
    e = nxs::run_matcher(d_left, d_right, width, height, params->disparities, params->paths,
                         params->p1, params->p2, params->uniqueness, params->stage_mask ? 1 : 0,
                         scratch, d_disparity, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        write_error(error, error_len, cudaGetErrorString(e));
        return NXS_CUDA_ERROR;
    }
    return NXS_OK;
}
