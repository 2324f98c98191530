// The C ABI of include/nx_stereo_b200.h: contexts, the segment protocol
// (configure / run / release, the reference Port's three requests) and the
// direct entry points.
//
// A segment owns its CUDA streams (upload, one or two compute streams,
// download, and a notify stream for the callers' completion callbacks), a ring
// of per-request device slots and what its stages carry from pair to pair (the
// temporal filter's previous disparity and missed counts, the quality
// stage's previous disparity). A request copies its entries into pinned
// memory, enqueues the upload into its slot, every member's kernels and the
// download of the outputs, ordered by events, and returns. A segment whose
// stages carry state computes on one stream in request order, as the
// reference's Port computes them (native/stereo_match/src/main.rs:1-11); one
// whose stages carry nothing alternates its requests between two compute
// streams. Uploads and downloads of neighbouring requests overlap the compute,
// and replies complete in request order.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nx_stereo_b200.h"
#include "nxs_kernels.h"

using namespace nxs;

namespace {

void set_error(char *error, size_t error_len, const char *format, ...) {
    if (!error || error_len == 0) return;
    va_list args;
    va_start(args, format);
    vsnprintf(error, error_len, format, args);
    va_end(args);
}

nxs_status cuda_status(cudaError_t e, char *error, size_t error_len, const char *what) {
    if (e == cudaSuccess) return NXS_OK;
    set_error(error, error_len, "%s: %s", what, cudaGetErrorString(e));
    return NXS_CUDA_ERROR;
}

// A device allocation that grows on demand.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t n) {
        if (n <= bytes) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&ptr, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// Pinned host blocks recycled between requests of one segment.
struct PinnedPool {
    std::mutex lock;
    std::multimap<size_t, void *> free_blocks;
    void *take(size_t n) {
        {
            std::lock_guard<std::mutex> g(lock);
            auto it = free_blocks.lower_bound(n);
            if (it != free_blocks.end() && it->first <= 4 * n + 4096) {
                void *p = it->second;
                free_blocks.erase(it);
                return p;
            }
        }
        void *p = nullptr;
        if (cudaHostAlloc(&p, std::max<size_t>(n, 64), cudaHostAllocDefault) != cudaSuccess)
            return nullptr;
        std::lock_guard<std::mutex> g(lock);
        sizes[p] = std::max<size_t>(n, 64);
        return p;
    }
    void give(void *p) {
        if (!p) return;
        std::lock_guard<std::mutex> g(lock);
        free_blocks.emplace(sizes[p], p);
    }
    // Allocates blocks of these sizes up front, so that requests do not
    // allocate pinned memory (slow, and it can wait for the device) while
    // pairs stream through.
    cudaError_t reserve(const std::vector<size_t> &blocks) {
        std::vector<void *> taken;
        cudaError_t e = cudaSuccess;
        for (size_t n : blocks) {
            void *p = take(n);
            if (!p) {
                e = cudaErrorMemoryAllocation;
                break;
            }
            taken.push_back(p);
        }
        for (void *p : taken) give(p);
        return e;
    }
    ~PinnedPool() {
        for (auto &kv : sizes) cudaFreeHost(kv.first);
    }
    std::map<void *, size_t> sizes;
};

// The events of finished requests, kept for the next ones, so that a request
// neither creates nor destroys events (one per member boundary and one for
// done). A request gives its events back only after its done event, which
// follows every one of them, has completed.
struct EventPool {
    std::mutex lock;
    std::vector<cudaEvent_t> timed, untimed;
    cudaError_t take(bool timing, cudaEvent_t *ev) {
        {
            std::lock_guard<std::mutex> g(lock);
            std::vector<cudaEvent_t> &free_events = timing ? timed : untimed;
            if (!free_events.empty()) {
                *ev = free_events.back();
                free_events.pop_back();
                return cudaSuccess;
            }
        }
        return timing ? cudaEventCreate(ev) : cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    }
    void give(bool timing, cudaEvent_t ev) {
        if (!ev) return;
        std::lock_guard<std::mutex> g(lock);
        (timing ? timed : untimed).push_back(ev);
    }
    ~EventPool() {
        for (cudaEvent_t ev : timed) cudaEventDestroy(ev);
        for (cudaEvent_t ev : untimed) cudaEventDestroy(ev);
    }
};

uint64_t monotonic_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Maps the device's event timestamps onto CLOCK_MONOTONIC (steady_clock), the
// clock of a serving loop's arrival times, with no host function in the
// request's path: a reference event is recorded on an otherwise idle stream
// and the host spins until it completes, five times, keeping the sample seen
// in the narrowest window (its time is that window's midpoint, within a few
// microseconds). A request's completion time is then the reference's time plus
// the device's elapsed time from the reference to the request's done event. The
// reference is taken again once it is 200 ms old, which bounds the drift
// between the two clocks.
struct DeviceClock {
    std::mutex lock;
    cudaStream_t stream = nullptr;
    cudaEvent_t ref = nullptr, probe = nullptr;
    uint64_t ref_ns = 0;
    cudaError_t open() {
        cudaError_t e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        if (!e) e = cudaEventCreate(&ref);
        if (!e) e = cudaEventCreate(&probe);
        if (!e) e = calibrate();
        return e;
    }
    cudaError_t calibrate() {
        uint64_t best = UINT64_MAX;
        for (int k = 0; k < 5; ++k) {
            const uint64_t t0 = monotonic_ns();
            cudaError_t e = cudaEventRecord(probe, stream);
            if (e) return e;
            while ((e = cudaEventQuery(probe)) == cudaErrorNotReady)
                if (monotonic_ns() - t0 > 1000000000ull) return cudaErrorNotReady;
            if (e) return e;
            const uint64_t t1 = monotonic_ns();
            if (t1 - t0 < best) {
                best = t1 - t0;
                std::swap(ref, probe);
                ref_ns = t0 + (t1 - t0) / 2;
            }
        }
        return cudaSuccess;
    }
    // CLOCK_MONOTONIC nanoseconds of a completed event; 0 if it cannot be read.
    uint64_t at(cudaEvent_t event) {
        std::lock_guard<std::mutex> g(lock);
        if (monotonic_ns() - ref_ns > 200000000ull && calibrate()) return 0;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ref, event) == cudaSuccess)
            return (uint64_t)((int64_t)ref_ns + llround((double)ms * 1e6));
        if (cudaEventElapsedTime(&ms, event, ref) == cudaSuccess)  // before the reference
            return (uint64_t)((int64_t)ref_ns - llround((double)ms * 1e6));
        return 0;
    }
    ~DeviceClock() {
        if (stream) cudaStreamSynchronize(stream);
        for (cudaEvent_t ev : {ref, probe})
            if (ev) cudaEventDestroy(ev);
        if (stream) cudaStreamDestroy(stream);
    }
};

enum class Kind { Rectification, Disparity, Speckle, Temporal, Depth, Cloud, Quality };

struct Member {
    Kind kind;
    std::string kind_name;
    int disparities = 0, paths = 0, radius = 3, decimation = 1;
    // Disparity's coarse-to-fine search (coarse_to_fine non-zero) and its settings
    int coarse_to_fine = 0, band = 16, margin = 4, coarse_paths = 8, census = 0;
    float max_missed = 255.0f, min_depth_m = 0.0f, max_depth_m = INFINITY;
    // carried from pair to pair
    float *previous = nullptr, *missed = nullptr;
};

struct Spec {
    std::string name;
    uint32_t type;
    std::vector<uint32_t> dims;
    size_t bytes() const {
        size_t n = type == NXS_U8 ? 1 : (type == NXS_U16 ? 2 : 4);
        for (uint32_t d : dims) n *= d;
        return n;
    }
};

// What one request in flight uses on the device: its entries, the outputs it
// downloads, and the events that order it across the segment's streams.
struct Slot {
    uint8_t *frames[2] = {nullptr, nullptr}, *images[2] = {nullptr, nullptr};
    float *disparity[2] = {nullptr, nullptr}, *grid = nullptr, *quality_sums = nullptr;
    uint16_t *depth_mm = nullptr;
    int32_t *kept = nullptr;
    // The entries, and the outputs, each in one region (Segment::entry_at and
    // output_at): the buffers above that are entries or outputs lie inside them.
    uint8_t *entries = nullptr, *outputs = nullptr;
    cudaEvent_t entered = nullptr;   // entries on the device
    cudaEvent_t free = nullptr;      // outputs downloaded: the slot may be reused
};

// Requests cycle through kSlots slots. Entries go up on `upload`, the members
// compute on a compute stream, outputs come down on `download`: request n + 1's
// upload and compute overlap request n's download. A segment whose stages
// carry state from pair to pair (TemporalFilter, Quality) computes on one
// stream in request order, so that state advances pair by pair; one whose
// stages carry nothing computes request n on stream n mod kLanes, each with
// its own matcher scratch and depth map, so neighbouring pairs overlap on the
// device (each pair's result is the same as alone). Downloads stay in request
// order on one stream.
constexpr int kSlots = 4;
constexpr int kLanes = 2;
// Whether segments configured from now on split their matcher over two
// streams (Segment::split); set by nxs_set_split_lanes.
static std::atomic<bool> g_split_lanes{true};

struct Segment {
    uint32_t id = 0;
    int device = 0;
    nxs_geometry g{};
    std::vector<Member> members;
    std::vector<Spec> entries, outputs;
    cudaStream_t upload = nullptr, download = nullptr;
    // Runs the caller's completion callbacks (host functions), when a request
    // has one, after its download, so that a host function waiting for the
    // driver's callback thread holds up no later request's download.
    cudaStream_t notify = nullptr;
    DeviceClock clock;  // requests' completion times
    cudaStream_t lanes[kLanes] = {};  // compute streams, n_lanes of them
    int n_lanes = 1;
    std::mutex order;  // one request enqueued at a time
    uint64_t sequence = 0;
    PinnedPool pinned;
    EventPool events;
    Slot slots[kSlots];
    // A request's entries go up in one copy and its outputs come down in one:
    // each has a region per slot and a pinned block per request, laid out
    // alike (offsets 256-byte aligned, in the order of `entries` and `outputs`).
    // The outputs are one region unless one of them is also an entry (a
    // disparity passed in and out unfiltered); then each comes down on its own.
    std::vector<size_t> entry_at, output_at;
    size_t entry_bytes = 0, output_bytes = 0;
    bool outputs_packed = false;
    // shared by the requests of one compute lane, touched only on its stream
    float *depth_m[kLanes] = {}, *quality_columns = nullptr;
    DeviceBuffer scratch[kLanes];
    // Split: a segment whose Disparity member is the full search, with no
    // stage carrying state before it, runs each pair's census, costs and path
    // volumes on lanes[0] and its selection onwards on lanes[1] (the stages
    // carrying state among them, in request order), so pair n + 1's front half
    // runs beside pair n's back half. Requests alternate between the two
    // scratches; carved[k]: scratch k's path volumes written, freed[k]: read.
    bool split = false;
    cudaEvent_t carved[kLanes] = {}, freed[kLanes] = {};
    // The Rectification member's maps (the frame position each rectified pixel
    // samples, both sides), one per compute lane and rewritten on that lane's
    // stream when a request's cameras differ from those it was made for.
    float2 *rectify_maps[kLanes] = {};
    Camera rectify_cameras[kLanes][2];
    bool rectify_mapped[kLanes] = {};
    std::vector<void *> allocations;

    std::vector<cudaStream_t> streams() const {
        std::vector<cudaStream_t> all = {upload, download, notify};
        for (int k = 0; k < n_lanes; ++k) all.push_back(lanes[k]);
        return all;
    }

    template <typename T>
    cudaError_t alloc(T **p, size_t count) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) {
            allocations.push_back(q);
            *p = static_cast<T *>(q);
        }
        return e;
    }
    ~Segment() {
        cudaSetDevice(device);
        for (cudaStream_t st : streams())
            if (st) cudaStreamSynchronize(st);
        for (void *p : allocations) cudaFree(p);
        for (DeviceBuffer &b : scratch) b.release();
        for (Slot &slot : slots)
            for (cudaEvent_t ev : {slot.entered, slot.free})
                if (ev) cudaEventDestroy(ev);
        for (int k = 0; k < kLanes; ++k)
            for (cudaEvent_t ev : {carved[k], freed[k]})
                if (ev) cudaEventDestroy(ev);
        for (cudaStream_t st : streams())
            if (st) cudaStreamDestroy(st);
    }
};

}  // namespace

struct nxs_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex lock;
    std::map<uint32_t, std::shared_ptr<Segment>> segments;
    DeviceBuffer scratch, io;
};

int nxs::context_device(nxs_context *context) { return context->device; }

struct nxs_request {
    std::shared_ptr<Segment> segment;
    std::vector<void *> pinned;  // returned to the segment's pool on free
    std::vector<cudaEvent_t> marks;  // before member 0, after each member
    cudaEvent_t done = nullptr;
    std::vector<nxs_tensor> outputs;
    std::vector<std::string> names;
    std::vector<uint32_t> times_us;
    bool timed = false;
    nxs_done_fn callback = nullptr;
    void *user = nullptr;
    uint64_t tag = 0;
    std::atomic<uint64_t> done_ns{0};  // CLOCK_MONOTONIC of `done`, once read
};

// ---------------------------------------------------------------------------
// Context

extern "C" const char *nxs_version(void) { return "nx_stereo_b200 0.1 (sm_100a)"; }

extern "C" nxs_status nxs_create(int device, nxs_context **context, char *error,
                                 size_t error_len) {
    if (!context) {
        set_error(error, error_len, "context is NULL");
        return NXS_BAD_ARGUMENT;
    }
    *context = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || device < 0 || device >= count) {
        set_error(error, error_len, "no CUDA device %d (%d present%s%s)", device, count,
                  e ? ": " : "", e ? cudaGetErrorString(e) : "");
        return NXS_CUDA_ERROR;
    }
    if ((e = cudaSetDevice(device))) return cuda_status(e, error, error_len, "cudaSetDevice");
    auto *c = new nxs_context();
    c->device = device;
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking))) {
        delete c;
        return cuda_status(e, error, error_len, "cudaStreamCreate");
    }
    *context = c;
    return NXS_OK;
}

extern "C" void nxs_destroy(nxs_context *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    {
        std::lock_guard<std::mutex> g(c->lock);
        c->segments.clear();
    }
    cudaStreamSynchronize(c->stream);
    c->scratch.release();
    c->io.release();
    cudaStreamDestroy(c->stream);
    delete c;
}

// ---------------------------------------------------------------------------
// Direct entry points

static bool supported_disparities(uint32_t d) {
    return d == 64 || d == 96 || d == 128 || d == 192 || d == 256;
}

extern "C" nxs_status nxs_sgm_check(const nxs_sgm_params *p, uint32_t width, uint32_t height,
                                    char *error, size_t error_len) {
    if (!p) {
        set_error(error, error_len, "params is NULL");
        return NXS_BAD_ARGUMENT;
    }
    // native/stereo_match/src/lib.rs:41-72 and lib/nx_stereo.ex:89-134.
    if (!(width > 8 && height > 6 && width <= 4096)) {
        set_error(error, error_len,
                  "expected an image wider than 8, higher than 6 and at most 4096 wide, got %ux%u",
                  width, height);
        return NXS_BAD_ARGUMENT;
    }
    if (!supported_disparities(p->disparities)) {
        set_error(error, error_len, "disparities must be 64, 96, 128, 192 or 256, got %u",
                  p->disparities);
        return NXS_BAD_ARGUMENT;
    }
    if (p->paths != 3 && p->paths != 8) {
        set_error(error, error_len, "paths must be 3 or 8, got %u", p->paths);
        return NXS_BAD_ARGUMENT;
    }
    if (!(p->p1 < p->p2 && p->p2 + 48 <= 127)) {
        set_error(error, error_len, "expected 0 <= p1 < p2 <= 79, got %u and %u", p->p1, p->p2);
        return NXS_BAD_ARGUMENT;
    }
    if (std::isnan(p->uniqueness) || p->uniqueness < 1.0f) {
        set_error(error, error_len, "uniqueness must be at least 1.0, got %g",
                  (double)p->uniqueness);
        return NXS_BAD_ARGUMENT;
    }
    return NXS_OK;
}

extern "C" nxs_status nxs_set_path_words(uint32_t disparities, uint32_t words) {
    if (!supported_disparities(disparities) || (words != 4 && words != 8 && words != 16))
        return NXS_BAD_ARGUMENT;
    set_path_words((int)disparities, (int)words);
    return NXS_OK;
}

extern "C" uint32_t nxs_path_words(uint32_t disparities) {
    return (uint32_t)path_words((int)disparities);
}

extern "C" nxs_status nxs_set_path_sums(uint32_t mode) {
    if (mode > 1) return NXS_BAD_ARGUMENT;
    set_path_sums((int)mode);
    return NXS_OK;
}

extern "C" uint32_t nxs_path_sums(uint32_t width, uint32_t height, uint32_t disparities) {
    return path_sums_wanted((int)width, (int)height, (int)disparities) ? 1u : 0u;
}

extern "C" nxs_status nxs_set_lean_select(uint32_t blocks_per_sm) {
    if (blocks_per_sm > 16) return NXS_BAD_ARGUMENT;
    set_lean_select((int)blocks_per_sm);
    return NXS_OK;
}

extern "C" uint32_t nxs_lean_select(void) { return (uint32_t)lean_select(); }

extern "C" nxs_status nxs_set_split_lanes(uint32_t on) {
    if (on > 1) return NXS_BAD_ARGUMENT;
    g_split_lanes = on != 0;
    return NXS_OK;
}

extern "C" nxs_status nxs_set_path_tiles(uint32_t mode) {
    if (mode > 2) return NXS_BAD_ARGUMENT;
    set_path_tiles((int)mode);
    return NXS_OK;
}

extern "C" uint32_t nxs_path_tiles(void) { return (uint32_t)path_tiles(); }

extern "C" uint32_t nxs_path_wait_failures(void) { return path_wait_failures(); }

extern "C" uint64_t nxs_sgm_scratch_bytes(uint32_t width, uint32_t height, uint32_t disparities) {
    return matcher_scratch_bytes((int)width, (int)height, (int)disparities);
}

extern "C" nxs_status nxs_sgm_device(nxs_context *c, const uint8_t *d_left,
                                     const uint8_t *d_right, uint32_t width, uint32_t height,
                                     const nxs_sgm_params *p, float *d_disparity, void *stream,
                                     char *error, size_t error_len) {
    if (!c || !d_left || !d_right || !d_disparity) {
        set_error(error, error_len, "a NULL context or buffer");
        return NXS_BAD_ARGUMENT;
    }
    nxs_status s = nxs_sgm_check(p, width, height, error, error_len);
    if (s) return s;
    cudaSetDevice(c->device);
    std::lock_guard<std::mutex> g(c->lock);
    cudaError_t e = c->scratch.reserve(matcher_scratch_bytes(width, height, p->disparities));
    if (e) return cuda_status(e, error, error_len, "scratch allocation");
    MatcherScratch ms = carve_matcher_scratch(c->scratch.ptr, width, height, p->disparities);
    e = run_matcher(d_left, d_right, width, height, p->disparities, p->paths, p->p1, p->p2,
                    p->uniqueness, p->stage_mask ? 1 : 0, ms, d_disparity,
                    static_cast<cudaStream_t>(stream));
    return cuda_status(e, error, error_len, "matcher launch");
}

extern "C" nxs_status nxs_sgm(nxs_context *c, const uint8_t *left, const uint8_t *right,
                              uint32_t width, uint32_t height, const nxs_sgm_params *p,
                              float *disparity, char *error, size_t error_len) {
    if (!c || !left || !right || !disparity) {
        set_error(error, error_len, "a NULL context or buffer");
        return NXS_BAD_ARGUMENT;
    }
    nxs_status s = nxs_sgm_check(p, width, height, error, error_len);
    if (s) return s;
    cudaSetDevice(c->device);
    const size_t pixels = (size_t)width * height;
    uint8_t *d_left, *d_right;
    float *d_out;
    {
        std::lock_guard<std::mutex> g(c->lock);
        cudaError_t e = c->io.reserve(2 * ((pixels + 255) & ~(size_t)255) + 4 * pixels);
        if (e) return cuda_status(e, error, error_len, "buffer allocation");
        d_left = static_cast<uint8_t *>(c->io.ptr);
        d_right = d_left + ((pixels + 255) & ~(size_t)255);
        d_out = reinterpret_cast<float *>(d_right + ((pixels + 255) & ~(size_t)255));
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync(d_left, left, pixels, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(d_right, right, pixels, cudaMemcpyHostToDevice, c->stream)))
        return cuda_status(e, error, error_len, "copy to the device");
    s = nxs_sgm_device(c, d_left, d_right, width, height, p, d_out, c->stream, error, error_len);
    if (s) return s;
    if ((e = cudaMemcpyAsync(disparity, d_out, 4 * pixels, cudaMemcpyDeviceToHost, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
        return cuda_status(e, error, error_len, "matcher");
    return NXS_OK;
}

extern "C" nxs_status nxs_band_check(const nxs_band_params *p, uint32_t width, uint32_t height,
                                     int32_t coarse_to_fine, char *error, size_t error_len) {
    if (!p) {
        set_error(error, error_len, "params is NULL");
        return NXS_BAD_ARGUMENT;
    }
    nxs_status s = nxs_sgm_check(&p->sgm, width, height, error, error_len);
    if (s) return s;
    // sgm_band/4's band check (lib/nx_stereo.ex:300-304) and census_window!/2 (481-489)
    if (p->band != 8 && p->band != 16 && p->band != 32 && p->band != 64) {
        set_error(error, error_len, ":band must be 8, 16, 32 or 64, got %u", p->band);
        return NXS_BAD_ARGUMENT;
    }
    if (p->census > 2) {
        set_error(error, error_len,
                  "census must be 0 (sparse 9x7), 1 (dense 9x5) or 2 (dense 9x5 blend), got %u",
                  p->census);
        return NXS_BAD_ARGUMENT;
    }
    if (!coarse_to_fine) return NXS_OK;
    // sgm_coarse_to_fine/3's checks (lib/nx_stereo.ex:173-183)
    if (width % 2 || height % 2) {
        set_error(error, error_len,
                  "coarse to fine expects images of even height and width, got %ux%u", width,
                  height);
        return NXS_BAD_ARGUMENT;
    }
    if (p->sgm.disparities != 128) {
        set_error(error, error_len,
                  ":disparities must be 128: the coarse matching takes 64, got %u",
                  p->sgm.disparities);
        return NXS_BAD_ARGUMENT;
    }
    if (p->coarse_paths != 3 && p->coarse_paths != 8) {
        set_error(error, error_len, "coarse_paths must be 3 or 8, got %u", p->coarse_paths);
        return NXS_BAD_ARGUMENT;
    }
    if (p->margin > 127) {
        set_error(error, error_len, "margin must be 0..127, got %u", p->margin);
        return NXS_BAD_ARGUMENT;
    }
    nxs_sgm_params coarse = p->sgm;
    coarse.disparities = 64;
    coarse.paths = p->coarse_paths;
    return nxs_sgm_check(&coarse, width / 2, height / 2, error, error_len);
}

extern "C" uint64_t nxs_band_scratch_bytes(uint32_t width, uint32_t height, uint32_t band,
                                           int32_t coarse_to_fine) {
    return coarse_to_fine ? coarse_to_fine_scratch_bytes(width, height, band)
                          : band_scratch_bytes(width, height, band);
}

extern "C" nxs_status nxs_sgm_band_device(nxs_context *c, const uint8_t *d_left,
                                          const uint8_t *d_right, const int32_t *d_base,
                                          uint32_t width, uint32_t height,
                                          const nxs_band_params *p, float *d_disparity,
                                          void *stream, char *error, size_t error_len) {
    if (!c || !d_left || !d_right || !d_base || !d_disparity) {
        set_error(error, error_len, "a NULL context or buffer");
        return NXS_BAD_ARGUMENT;
    }
    nxs_status s = nxs_band_check(p, width, height, 0, error, error_len);
    if (s) return s;
    cudaSetDevice(c->device);
    std::lock_guard<std::mutex> g(c->lock);
    cudaError_t e = c->scratch.reserve(band_scratch_bytes(width, height, p->band));
    if (e) return cuda_status(e, error, error_len, "scratch allocation");
    BandScratch bs = carve_band_scratch(c->scratch.ptr, width, height, p->band);
    e = run_band_matcher(d_left, d_right, d_base, width, height, p->sgm.disparities, p->sgm.paths,
                         p->band, p->census, p->sgm.p1, p->sgm.p2, p->sgm.uniqueness,
                         p->sgm.stage_mask ? 1 : 0, bs, d_disparity,
                         static_cast<cudaStream_t>(stream));
    return cuda_status(e, error, error_len, "band matcher launch");
}

extern "C" nxs_status nxs_sgm_coarse_to_fine_device(nxs_context *c, const uint8_t *d_left,
                                                    const uint8_t *d_right, uint32_t width,
                                                    uint32_t height, const nxs_band_params *p,
                                                    float *d_disparity, int32_t *d_base,
                                                    void *stream, char *error,
                                                    size_t error_len) {
    if (!c || !d_left || !d_right || !d_disparity) {
        set_error(error, error_len, "a NULL context or buffer");
        return NXS_BAD_ARGUMENT;
    }
    nxs_status s = nxs_band_check(p, width, height, 1, error, error_len);
    if (s) return s;
    cudaSetDevice(c->device);
    std::lock_guard<std::mutex> g(c->lock);
    cudaError_t e = c->scratch.reserve(coarse_to_fine_scratch_bytes(width, height, p->band));
    if (e) return cuda_status(e, error, error_len, "scratch allocation");
    e = run_coarse_to_fine(d_left, d_right, width, height, p->sgm.paths, p->coarse_paths,
                           p->band, p->margin, p->census, p->sgm.p1, p->sgm.p2,
                           p->sgm.uniqueness, p->sgm.stage_mask ? 1 : 0, c->scratch.ptr,
                           d_disparity, d_base, static_cast<cudaStream_t>(stream));
    return cuda_status(e, error, error_len, "coarse-to-fine launch");
}

extern "C" nxs_status nxs_sgm_coarse_to_fine(nxs_context *c, const uint8_t *left,
                                             const uint8_t *right, uint32_t width,
                                             uint32_t height, const nxs_band_params *p,
                                             float *disparity, char *error, size_t error_len) {
    if (!c || !left || !right || !disparity) {
        set_error(error, error_len, "a NULL context or buffer");
        return NXS_BAD_ARGUMENT;
    }
    nxs_status s = nxs_band_check(p, width, height, 1, error, error_len);
    if (s) return s;
    cudaSetDevice(c->device);
    const size_t pixels = (size_t)width * height, aligned = (pixels + 255) & ~(size_t)255;
    uint8_t *d_left, *d_right;
    float *d_out;
    {
        std::lock_guard<std::mutex> g(c->lock);
        cudaError_t e = c->io.reserve(2 * aligned + 4 * pixels);
        if (e) return cuda_status(e, error, error_len, "buffer allocation");
        d_left = static_cast<uint8_t *>(c->io.ptr);
        d_right = d_left + aligned;
        d_out = reinterpret_cast<float *>(d_right + aligned);
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync(d_left, left, pixels, cudaMemcpyHostToDevice, c->stream)) ||
        (e = cudaMemcpyAsync(d_right, right, pixels, cudaMemcpyHostToDevice, c->stream)))
        return cuda_status(e, error, error_len, "copy to the device");
    s = nxs_sgm_coarse_to_fine_device(c, d_left, d_right, width, height, p, d_out, nullptr,
                                      c->stream, error, error_len);
    if (s) return s;
    if ((e = cudaMemcpyAsync(disparity, d_out, 4 * pixels, cudaMemcpyDeviceToHost, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
        return cuda_status(e, error, error_len, "coarse to fine");
    return NXS_OK;
}

#define CHECK_SIZE(cond)                   \
    do {                                   \
        if (!(cond)) return NXS_BAD_ARGUMENT; \
    } while (0)

extern "C" nxs_status nxs_census_device(const uint8_t *d_image, uint32_t width, uint32_t height,
                                        uint64_t *d_codes, void *stream) {
    CHECK_SIZE(d_image && d_codes && width > 0 && height > 0);
    return launch_census(d_image, nullptr, width, height, d_codes, nullptr,
                         static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_census_pair_device(const uint8_t *d_left, const uint8_t *d_right,
                                             uint32_t width, uint32_t height,
                                             uint64_t *d_left_codes, uint64_t *d_right_codes,
                                             void *stream) {
    CHECK_SIZE(d_left && d_right && d_left_codes && d_right_codes && width > 0 && height > 0);
    return launch_census(d_left, d_right, width, height, d_left_codes, d_right_codes,
                         static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_check_median_device(const float *d_disparity, const uint32_t *d_keys,
                                              uint32_t width, uint32_t height,
                                              uint32_t stage_mask, float *d_filtered,
                                              void *stream) {
    CHECK_SIZE(d_disparity && d_keys && d_filtered && width > 0 && width <= 4096 && height > 0);
    return launch_check_median(d_disparity, d_keys, width, height, stage_mask ? 1 : 0,
                               d_filtered, static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_costs_device(const uint64_t *d_left_codes,
                                       const uint64_t *d_right_codes, uint32_t width,
                                       uint32_t height, uint32_t disparities, uint8_t *d_costs,
                                       void *stream) {
    CHECK_SIZE(d_left_codes && d_right_codes && d_costs && width > 0 && height > 0 &&
               disparities % 16 == 0 && disparities >= 16 && disparities <= 256);
    return launch_costs(d_left_codes, d_right_codes, width, height, disparities, d_costs,
                        static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_aggregate_device(nxs_context *c, const uint8_t *d_costs,
                                           uint32_t width, uint32_t height, uint32_t disparities,
                                           uint32_t paths, uint32_t p1, uint32_t p2,
                                           uint16_t *d_sums, void *stream) {
    CHECK_SIZE(c && d_costs && d_sums && width > 0 && height > 0 && disparities % 32 == 0 &&
               disparities >= 64 && disparities <= 256 && (paths == 3 || paths == 8) &&
               p1 < p2 && p2 + 48 <= 127);
    cudaSetDevice(c->device);
    std::lock_guard<std::mutex> g(c->lock);
    const size_t volume = (size_t)width * height * disparities;
    if (c->scratch.reserve(8 * volume)) return NXS_CUDA_ERROR;
    uint8_t *volumes = static_cast<uint8_t *>(c->scratch.ptr);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (launch_paths(d_costs, width, height, disparities, paths, p1, p2, volumes, s) ||
        launch_sum_paths(volumes, width, height, disparities, paths, d_sums, s))
        return NXS_CUDA_ERROR;
    return NXS_OK;
}

extern "C" nxs_status nxs_paths_device(const uint8_t *d_costs, uint32_t width, uint32_t height,
                                       uint32_t disparities, uint32_t paths, uint32_t p1,
                                       uint32_t p2, uint8_t *d_paths, void *stream) {
    CHECK_SIZE(d_costs && d_paths && width > 0 && height > 0 && disparities % 32 == 0 &&
               disparities >= 64 && disparities <= 256 && (paths == 3 || paths == 8) &&
               p1 < p2 && p2 + 48 <= 127);
    return launch_paths(d_costs, width, height, disparities, paths, p1, p2, d_paths,
                        static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_select_paths_device(const uint8_t *d_paths, uint32_t width,
                                              uint32_t height, uint32_t disparities,
                                              uint32_t paths, float uniqueness,
                                              float *d_disparity, uint32_t *d_keys,
                                              void *stream) {
    CHECK_SIZE(d_paths && d_disparity && d_keys && width > 0 && height > 0 &&
               disparities % 16 == 0 && disparities >= 16 && disparities <= 256 &&
               (paths == 3 || paths == 8));
    return launch_select_paths(d_paths, width, height, disparities, paths, uniqueness,
                               d_disparity, d_keys, static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" uint32_t nxs_matcher_span(uint32_t disparities) {
    return (uint32_t)matcher_span((int)disparities);
}

extern "C" nxs_status nxs_costs_device_ordered(const uint64_t *d_left_codes,
                                               const uint64_t *d_right_codes, uint32_t width,
                                               uint32_t height, uint32_t disparities,
                                               uint32_t span, uint8_t *d_costs, void *stream) {
    CHECK_SIZE(d_left_codes && d_right_codes && d_costs && width > 0 && height > 0 &&
               disparities % 16 == 0 && disparities >= 16 && disparities <= 256 &&
               (span == 0 || span == 8 || span == 16));
    return launch_costs(d_left_codes, d_right_codes, width, height, disparities, d_costs,
                        static_cast<cudaStream_t>(stream), (int)span)
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_census_costs_device_ordered(const uint8_t *d_left,
                                                      const uint8_t *d_right, uint32_t width,
                                                      uint32_t height, uint32_t disparities,
                                                      uint32_t span, uint8_t *d_costs,
                                                      void *stream) {
    CHECK_SIZE(d_left && d_right && d_costs && width > 0 && height > 0 &&
               disparities % 16 == 0 && disparities >= 16 && disparities <= 256 &&
               (span == 0 || span == 8 || span == 16));
    return launch_census_costs(d_left, d_right, width, height, disparities, d_costs,
                               static_cast<cudaStream_t>(stream), (int)span)
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_paths_device_ordered(const uint8_t *d_costs, uint32_t width,
                                               uint32_t height, uint32_t disparities,
                                               uint32_t paths, uint32_t p1, uint32_t p2,
                                               uint32_t span, uint8_t *d_paths, void *stream) {
    CHECK_SIZE(d_costs && d_paths && width > 0 && height > 0 && disparities % 32 == 0 &&
               disparities >= 64 && disparities <= 256 && (paths == 3 || paths == 8) &&
               p1 < p2 && p2 + 48 <= 127 && (span == 0 || span == 8 || span == 16));
    return launch_paths(d_costs, width, height, disparities, paths, p1, p2, d_paths,
                        static_cast<cudaStream_t>(stream), (int)span)
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_select_paths_device_ordered(const uint8_t *d_paths, uint32_t width,
                                                      uint32_t height, uint32_t disparities,
                                                      uint32_t paths, float uniqueness,
                                                      uint32_t span, float *d_disparity,
                                                      uint32_t *d_keys, void *stream) {
    CHECK_SIZE(d_paths && d_disparity && d_keys && width > 0 && height > 0 &&
               disparities % 16 == 0 && disparities >= 16 && disparities <= 256 &&
               (paths == 3 || paths == 8) && (span == 0 || span == 8 || span == 16));
    return launch_select_paths(d_paths, width, height, disparities, paths, uniqueness,
                               d_disparity, d_keys, static_cast<cudaStream_t>(stream), (int)span)
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_path_sums_device(const uint8_t *d_costs, uint32_t width,
                                           uint32_t height, uint32_t disparities, uint32_t paths,
                                           uint32_t p1, uint32_t p2, uint16_t *d_sums,
                                           void *stream) {
    CHECK_SIZE(d_costs && d_sums && width > 0 && height > 0 && disparities % 16 == 0 &&
               disparities >= 64 && disparities <= 256 && (paths == 3 || paths == 8) &&
               p1 < p2 && p2 + 48 <= 127);
    return launch_paths_sums(d_costs, width, height, disparities, paths, p1, p2, d_sums,
                             static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_select_path_sums_device(const uint16_t *d_sums, uint32_t width,
                                                  uint32_t height, uint32_t disparities,
                                                  float uniqueness, float *d_disparity,
                                                  uint32_t *d_keys, void *stream) {
    CHECK_SIZE(d_sums && d_disparity && d_keys && width > 0 && height > 0 &&
               disparities % 16 == 0 && disparities >= 64 && disparities <= 256);
    return launch_select_path_sums(d_sums, width, height, disparities, uniqueness, d_disparity,
                                   d_keys, static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_select_device(const uint16_t *d_sums, uint32_t width, uint32_t height,
                                        uint32_t disparities, float uniqueness,
                                        float *d_disparity, uint32_t *d_keys, void *stream) {
    CHECK_SIZE(d_sums && d_disparity && d_keys && width > 0 && height > 0 && disparities >= 16 &&
               disparities <= 256 && disparities % 16 == 0);
    return launch_select_sums(d_sums, width, height, disparities, uniqueness, d_disparity, d_keys,
                              static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_consistency_device(const float *d_disparity, const uint32_t *d_keys,
                                             uint32_t width, uint32_t height, float *d_checked,
                                             void *stream) {
    CHECK_SIZE(d_disparity && d_keys && d_checked && width > 0 && width <= 8192 && height > 0);
    return launch_consistency(d_disparity, d_keys, width, height, d_checked,
                              static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_median3_device(const float *d_image, uint32_t width, uint32_t height,
                                         uint32_t stage_mask, float *d_filtered, void *stream) {
    CHECK_SIZE(d_image && d_filtered && width > 0 && height > 0);
    return launch_median3(d_image, width, height, stage_mask ? 1 : 0, d_filtered,
                          static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

static_assert(sizeof(Camera) == 23 * sizeof(float), "cameras compare as their bytes");

static Camera to_camera(const nxs_camera *c) {
    Camera k;
    memcpy(k.k, c->k, sizeof k.k);
    memcpy(k.d, c->d, sizeof k.d);
    memcpy(k.inverse_pr, c->inverse_pr, sizeof k.inverse_pr);
    return k;
}

extern "C" nxs_status nxs_rectify_device(const uint8_t *d_frame, uint32_t frame_width,
                                         uint32_t frame_height, const nxs_camera *camera,
                                         uint32_t width, uint32_t height, uint8_t *d_rectified,
                                         void *stream) {
    CHECK_SIZE(d_frame && camera && d_rectified && width > 0 && height > 0 &&
               frame_width >= width && frame_height >= height);
    return launch_rectify(d_frame, frame_width, frame_height, to_camera(camera), width, height,
                          d_rectified, static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_rectify_pair_device(const uint8_t *d_left_frame,
                                              const uint8_t *d_right_frame, uint32_t frame_width,
                                              uint32_t frame_height, const nxs_camera *left,
                                              const nxs_camera *right, uint32_t width,
                                              uint32_t height, uint8_t *d_left, uint8_t *d_right,
                                              void *stream) {
    CHECK_SIZE(d_left_frame && d_right_frame && left && right && d_left && d_right &&
               width > 0 && height > 0 && frame_width >= width && frame_height >= height);
    return launch_rectify_pair(d_left_frame, d_right_frame, frame_width, frame_height,
                               to_camera(left), to_camera(right), width, height, d_left, d_right,
                               static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_rectify_maps_device(const nxs_camera *left, const nxs_camera *right,
                                              uint32_t frame_width, uint32_t frame_height,
                                              uint32_t width, uint32_t height, float *d_maps,
                                              void *stream) {
    CHECK_SIZE(left && right && d_maps && (uintptr_t)d_maps % 8 == 0 && width > 0 &&
               height > 0 && frame_width >= width && frame_height >= height);
    return launch_rectify_maps(to_camera(left), to_camera(right), frame_width, frame_height,
                               width, height, reinterpret_cast<float2 *>(d_maps),
                               static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_rectify_pair_mapped_device(const uint8_t *d_left_frame,
                                                     const uint8_t *d_right_frame,
                                                     uint32_t frame_width, uint32_t frame_height,
                                                     const float *d_maps, uint32_t width,
                                                     uint32_t height, uint8_t *d_left,
                                                     uint8_t *d_right, void *stream) {
    CHECK_SIZE(d_left_frame && d_right_frame && d_maps && (uintptr_t)d_maps % 8 == 0 &&
               d_left && d_right && width > 0 && height > 0 && frame_width >= width &&
               frame_height >= height);
    return launch_rectify_mapped(d_left_frame, d_right_frame, frame_width, frame_height,
                                 reinterpret_cast<const float2 *>(d_maps), width, height, d_left,
                                 d_right, static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_despeckle_device(const float *d_disparity, uint32_t width,
                                           uint32_t height, float min_support, float max_diff,
                                           uint32_t radius, float *d_despeckled, void *stream) {
    CHECK_SIZE(d_disparity && d_despeckled && width > 0 && height > 0 && radius >= 1 &&
               radius <= 8);
    return launch_despeckle(d_disparity, width, height, min_support, max_diff, radius,
                            d_despeckled, static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_temporal_device(float *d_disparity, float *d_previous, float *d_missed,
                                          uint64_t pixels, float alpha, float delta, float hold,
                                          float max_missed, void *stream) {
    CHECK_SIZE(d_disparity && d_previous && d_missed);
    if (pixels == 0) return NXS_OK;
    return launch_temporal(d_disparity, d_previous, d_missed, pixels, alpha, delta, hold,
                           max_missed, static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_depth_device(const float *d_disparity, uint64_t pixels,
                                       float focal_length_px, float baseline_m,
                                       uint16_t *d_depth_mm, float *d_depth_m, void *stream) {
    CHECK_SIZE(d_disparity && d_depth_mm && d_depth_m);
    if (pixels == 0) return NXS_OK;
    return launch_depth(d_disparity, pixels, focal_length_px, baseline_m, d_depth_mm, d_depth_m,
                        static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_cloud_device(const float *d_depth_m, uint32_t width, uint32_t height,
                                       uint32_t decimation, float focal_length_px, float cx,
                                       float cy, float nearest_m, float farthest_m,
                                       float *d_grid, int32_t *d_kept, void *stream) {
    CHECK_SIZE(d_depth_m && d_grid && d_kept && decimation >= 1 && decimation <= width &&
               decimation <= height);
    return launch_cloud(d_depth_m, width, height, decimation, focal_length_px, cx, cy, nearest_m,
                        farthest_m, d_grid, d_kept, static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_despeckle_depth_cloud_device(
    const float *d_disparity, uint32_t width, uint32_t height, float min_support, float max_diff,
    uint32_t radius, float focal_length_px, float baseline_m, uint32_t decimation, float cx,
    float cy, float nearest_m, float farthest_m, float *d_despeckled, uint16_t *d_depth_mm,
    float *d_depth_m, float *d_grid, int32_t *d_kept, void *stream) {
    CHECK_SIZE(d_disparity && d_despeckled && d_depth_mm && d_depth_m && d_grid && d_kept &&
               width > 0 && height > 0 && radius >= 1 && radius <= 5 && decimation >= 1 &&
               decimation <= width && decimation <= height && d_despeckled != d_disparity);
    return launch_despeckle_depth_cloud(d_disparity, width, height, min_support, max_diff,
                                        radius, focal_length_px, baseline_m, decimation, cx, cy,
                                        nearest_m, farthest_m, d_despeckled, d_depth_mm,
                                        d_depth_m, d_grid, d_kept,
                                        static_cast<cudaStream_t>(stream))
               ? NXS_CUDA_ERROR
               : NXS_OK;
}

extern "C" nxs_status nxs_quality_device(const float *d_disparity, float *d_previous,
                                         uint32_t width, uint32_t height, float *d_sums,
                                         void *stream) {
    CHECK_SIZE(d_disparity && d_previous && d_sums && width > 0 && height > 0);
    // The per-column sums live in a small stream-ordered allocation.
    float *columns = nullptr;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMallocAsync(reinterpret_cast<void **>(&columns), sizeof(float) * 5 * width, s))
        return NXS_CUDA_ERROR;
    cudaError_t e = launch_quality(d_disparity, d_previous, width, height, columns, d_sums, s);
    cudaFreeAsync(columns, s);
    return e ? NXS_CUDA_ERROR : NXS_OK;
}

// ---------------------------------------------------------------------------
// The segment protocol

namespace {

const char *kind_names[] = {"rectification", "disparity", "speckle_filter", "temporal_filter",
                            "depth", "point_cloud", "quality"};

bool parse_kind(const char *name, Kind *kind) {
    for (int i = 0; i < 7; ++i)
        if (name && strcmp(name, kind_names[i]) == 0) {
            *kind = static_cast<Kind>(i);
            return true;
        }
    return false;
}

std::vector<std::string> requires_of(Kind k) {
    switch (k) {
    case Kind::Rectification: return {"left_frame", "right_frame"};
    case Kind::Disparity: return {"left", "right"};
    case Kind::Cloud: return {"depth_m"};
    default: return {"disparity"};
    }
}

std::vector<std::string> provides_of(Kind k) {
    switch (k) {
    case Kind::Rectification: return {"left", "right"};
    case Kind::Depth: return {"depth_mm", "depth_m"};
    case Kind::Cloud: return {"cloud_grid", "cloud_points"};
    case Kind::Quality: return {"quality_sums"};
    default: return {"disparity"};
    }
}

// The outputs a member returns (native/stereo_match/src/segment.rs:74-89):
// depth_m stays on the device.
std::vector<std::string> outputs_of(Kind k) {
    switch (k) {
    case Kind::Rectification: return {"left", "right"};
    case Kind::Depth: return {"depth_mm"};
    case Kind::Cloud: return {"cloud_grid", "cloud_points"};
    case Kind::Quality: return {"quality_sums"};
    default: return {"disparity"};
    }
}

const nxs_setting *find_setting(const nxs_member &m, const char *name) {
    for (uint32_t i = 0; i < m.n_settings; ++i)
        if (m.settings[i].name && strcmp(m.settings[i].name, name) == 0) return &m.settings[i];
    return nullptr;
}

// segment.rs:98-111: the settings a kind does not take, sorted.
bool takes_only(const nxs_member &m, std::initializer_list<const char *> names,
                std::string *why) {
    std::vector<std::string> unknown;
    for (uint32_t i = 0; i < m.n_settings; ++i) {
        const char *n = m.settings[i].name ? m.settings[i].name : "";
        bool known = false;
        for (const char *k : names) known = known || strcmp(n, k) == 0;
        if (!known) unknown.push_back(n);
    }
    if (unknown.empty()) return true;
    std::sort(unknown.begin(), unknown.end());
    *why = std::string(m.kind) + " has no setting ";
    for (size_t i = 0; i < unknown.size(); ++i) *why += (i ? ", " : "") + unknown[i];
    return false;
}

bool option(const nxs_member &m, const char *name, double *value, std::string *why) {
    const nxs_setting *s = find_setting(m, name);
    if (!s) {
        *why = std::string(m.kind) + " needs its " + name + " setting";
        return false;
    }
    *value = s->value;
    return true;
}

bool count_option(const nxs_member &m, const char *name, long lowest, long highest, int *out,
                  std::string *why) {
    double v;
    if (!option(m, name, &v, why)) return false;
    if (std::floor(v) == v && v >= (double)lowest && v <= (double)highest) {
        *out = (int)v;
        return true;
    }
    char buf[256];
    snprintf(buf, sizeof buf, "%s %s must be an integer from %ld to %ld, got %g", m.kind, name,
             lowest, highest, v);
    *why = buf;
    return false;
}

bool integer_option(const nxs_member &m, const char *name, std::vector<int> allowed, int *out,
                    std::string *why) {
    double v;
    if (!option(m, name, &v, why)) return false;
    for (int a : allowed)
        if ((double)a == v) {
            *out = a;
            return true;
        }
    std::string list;
    for (size_t i = 0; i < allowed.size(); ++i)
        list += (i ? ", " : "") + std::to_string(allowed[i]);
    char buf[256];
    snprintf(buf, sizeof buf, "%s %s must be one of [%s], got %g", m.kind, name, list.c_str(), v);
    *why = buf;
    return false;
}

// segment.rs:242-333: a stage of `kind` with exactly the settings it takes.
bool build_member(const nxs_geometry &g, const nxs_member &m, Member *out, std::string *why) {
    if (!parse_kind(m.kind, &out->kind)) {
        *why = std::string("no native implementation of ") + (m.kind ? m.kind : "(null)");
        return false;
    }
    out->kind_name = m.kind;
    const long w = g.width, h = g.height;
    switch (out->kind) {
    case Kind::Rectification:
        if (!takes_only(m, {}, why)) return false;
        if (g.frame_width < g.width || g.frame_height < g.height) {
            char buf[256];
            snprintf(buf, sizeof buf,
                     "rectification only shrinks: %ux%u frames are smaller than the %ux%u "
                     "working size",
                     g.frame_width, g.frame_height, g.width, g.height);
            *why = buf;
            return false;
        }
        return true;
    case Kind::Disparity: {
        if (!takes_only(m, {"num_disparities", "paths", "coarse_to_fine", "band", "margin",
                            "coarse_paths", "fine_census"},
                        why))
            return false;
        if (!integer_option(m, "num_disparities", {64, 96, 128, 192, 256}, &out->disparities,
                            why) ||
            !integer_option(m, "paths", {3, 8}, &out->paths, why))
            return false;
        nxs_sgm_params p{(uint32_t)out->disparities, (uint32_t)out->paths, 8, 64, 1.0f, 1};
        char buf[256];
        if (find_setting(m, "coarse_to_fine")) {
            // Stage.Disparity's search "coarse_to_fine" (stage/disparity.ex:72-108): the
            // band, margin, coarse paths and fine census (0 sparse 9x7, 1 dense 9x5, 2 blended)
            if (!integer_option(m, "coarse_to_fine", {0, 1}, &out->coarse_to_fine, why))
                return false;
        }
        if (out->coarse_to_fine) {
            if (!integer_option(m, "band", {8, 16, 32, 64}, &out->band, why) ||
                !count_option(m, "margin", 0, out->band - 1, &out->margin, why) ||
                !integer_option(m, "coarse_paths", {3, 8}, &out->coarse_paths, why) ||
                !count_option(m, "fine_census", 0, 2, &out->census, why))
                return false;
            nxs_band_params bp{p, (uint32_t)out->band, (uint32_t)out->margin,
                               (uint32_t)out->coarse_paths, (uint32_t)out->census};
            if (nxs_band_check(&bp, g.width, g.height, 1, buf, sizeof buf)) {
                *why = buf;
                return false;
            }
            return true;
        }
        if (nxs_sgm_check(&p, g.width, g.height, buf, sizeof buf)) {
            *why = buf;
            return false;
        }
        return true;
    }
    case Kind::Speckle:
        if (!takes_only(m, {"radius"}, why)) return false;
        return count_option(m, "radius", 1, std::min<long>(8, std::min(w, h)), &out->radius, why);
    case Kind::Temporal: {
        if (!takes_only(m, {"max_missed"}, why)) return false;
        double v;
        if (!option(m, "max_missed", &v, why)) return false;
        out->max_missed = (float)v;
        return true;
    }
    case Kind::Depth:
        return takes_only(m, {}, why);
    case Kind::Cloud: {
        if (!takes_only(m, {"decimation", "min_depth_m", "max_depth_m"}, why)) return false;
        double lo, hi;
        if (!count_option(m, "decimation", 1, std::min(w, h), &out->decimation, why) ||
            !option(m, "min_depth_m", &lo, why) || !option(m, "max_depth_m", &hi, why))
            return false;
        out->min_depth_m = (float)lo;
        out->max_depth_m = (float)hi;
        return true;
    }
    case Kind::Quality:
        return takes_only(m, {}, why);
    }
    return false;
}

Spec entry_spec(const std::string &name, const nxs_geometry &g, bool *ok) {
    *ok = true;
    if (name == "left_frame" || name == "right_frame")
        return {name, NXS_U8, {g.frame_height, g.frame_width}};
    if (name == "left" || name == "right") return {name, NXS_U8, {g.height, g.width}};
    if (name == "disparity") return {name, NXS_F32, {g.height, g.width}};
    *ok = false;
    return {};
}

Spec output_spec(const std::string &name, const nxs_geometry &g, const Member &m) {
    if (name == "left" || name == "right") return {name, NXS_U8, {g.height, g.width}};
    if (name == "disparity") return {name, NXS_F32, {g.height, g.width}};
    if (name == "depth_mm") return {name, NXS_U16, {g.height, g.width}};
    if (name == "cloud_grid")
        return {name, NXS_F32,
                {g.height / (uint32_t)m.decimation, g.width / (uint32_t)m.decimation, 3}};
    if (name == "cloud_points") return {name, NXS_S32, {}};
    return {name, NXS_F32, {5}};  // quality_sums
}

const nxs_param *find_param(const nxs_member_params &mp, const char *name) {
    for (uint32_t i = 0; i < mp.n_params; ++i)
        if (mp.params[i].name && strcmp(mp.params[i].name, name) == 0) return &mp.params[i];
    return nullptr;
}

// segment.rs:131-165: a live input of the right length.
bool input(const nxs_member_params &mp, const char *name, uint32_t length, const float **values,
           std::string *why) {
    const nxs_param *p = find_param(mp, name);
    if (!p) {
        *why = std::string("no ") + name + " among the stage's inputs";
        return false;
    }
    if (p->count != length || !p->values) {
        *why = std::string(name) + " has " + std::to_string(p->count) + " values, expected " +
               std::to_string(length);
        return false;
    }
    *values = p->values;
    return true;
}

bool scalar(const nxs_member_params &mp, const char *name, float *value, std::string *why) {
    const float *v;
    if (!input(mp, name, 1, &v, why)) return false;
    *value = v[0];
    return true;
}

bool penalty(const nxs_member_params &mp, const char *name, uint32_t *value, std::string *why) {
    float v;
    if (!scalar(mp, name, &v, why)) return false;
    if (std::floor(v) == v && v >= 0.0f && v <= 255.0f) {
        *value = (uint32_t)v;
        return true;
    }
    char buf[128];
    snprintf(buf, sizeof buf, "%s must be an integer from 0 to 255, got %g", name, (double)v);
    *why = buf;
    return false;
}

bool camera(const nxs_member_params &mp, const char *side, Camera *k, std::string *why) {
    const float *v;
    std::string s(side);
    if (!input(mp, (s + ".k").c_str(), 9, &v, why)) return false;
    memcpy(k->k, v, sizeof k->k);
    if (!input(mp, (s + ".d").c_str(), 5, &v, why)) return false;
    memcpy(k->d, v, sizeof k->d);
    if (!input(mp, (s + ".inverse_pr").c_str(), 9, &v, why)) return false;
    memcpy(k->inverse_pr, v, sizeof k->inverse_pr);
    return true;
}

// Parsed live inputs of one member for one pair.
struct Live {
    Camera cameras[2];
    nxs_sgm_params sgm{};
    float a = 0, b = 0, c = 0;  // stage scalars
};

bool parse_live(const Member &m, const nxs_geometry &g, const nxs_member_params &mp, Live *live,
                std::string *why) {
    switch (m.kind) {
    case Kind::Rectification:
        return camera(mp, "left", &live->cameras[0], why) &&
               camera(mp, "right", &live->cameras[1], why);
    case Kind::Disparity: {
        live->sgm.disparities = m.disparities;
        live->sgm.paths = m.paths;
        live->sgm.stage_mask = 1;
        if (!penalty(mp, "p1", &live->sgm.p1, why) || !penalty(mp, "p2", &live->sgm.p2, why) ||
            !scalar(mp, "uniqueness", &live->sgm.uniqueness, why))
            return false;
        char buf[256];
        if (nxs_sgm_check(&live->sgm, g.width, g.height, buf, sizeof buf)) {
            *why = buf;
            return false;
        }
        return true;
    }
    case Kind::Speckle:
        return scalar(mp, "min_support", &live->a, why) && scalar(mp, "max_diff", &live->b, why);
    case Kind::Temporal:
        return scalar(mp, "alpha", &live->a, why) && scalar(mp, "delta", &live->b, why) &&
               scalar(mp, "hold", &live->c, why);
    case Kind::Depth:
        return scalar(mp, "focal_length_px", &live->a, why) &&
               scalar(mp, "baseline_m", &live->b, why);
    case Kind::Cloud:
        return scalar(mp, "focal_length_px", &live->a, why) && scalar(mp, "cx", &live->b, why) &&
               scalar(mp, "cy", &live->c, why);
    case Kind::Quality:
        return true;
    }
    return false;
}

}  // namespace

extern "C" nxs_status nxs_configure(nxs_context *c, uint32_t id, const nxs_geometry *geometry,
                                    uint32_t n_members, const nxs_member *members, char *error,
                                    size_t error_len) {
    if (!c || !geometry || (n_members && !members)) {
        set_error(error, error_len, "a NULL context, geometry or member list");
        return NXS_BAD_ARGUMENT;
    }
    const nxs_geometry g = *geometry;
    if (g.width < 2 || g.height < 2 || g.width > 65535 || g.height > 65535) {
        set_error(error, error_len, "a segment works at 2x2 or more, got %ux%u", g.width,
                  g.height);
        return NXS_REFUSED;
    }
    auto seg = std::make_shared<Segment>();
    seg->id = id;
    seg->device = c->device;
    seg->g = g;
    std::vector<std::string> provided;
    for (uint32_t i = 0; i < n_members; ++i) {
        Member m;
        std::string why;
        if (!build_member(g, members[i], &m, &why)) {
            set_error(error, error_len, "%s", why.c_str());
            return NXS_REFUSED;
        }
        for (const std::string &r : requires_of(m.kind)) {
            bool have = std::find(provided.begin(), provided.end(), r) != provided.end();
            bool listed = false;
            for (const Spec &e : seg->entries) listed = listed || e.name == r;
            if (have || listed) continue;
            bool ok;
            Spec spec = entry_spec(r, g, &ok);
            if (!ok) {
                set_error(error, error_len,
                          "no stage before it provides %s, and a segment cannot take it as an "
                          "entry",
                          r.c_str());
                return NXS_REFUSED;
            }
            seg->entries.push_back(spec);
        }
        for (const std::string &p : provides_of(m.kind)) provided.push_back(p);
        for (const std::string &o : outputs_of(m.kind)) {
            bool listed = false;
            for (const Spec &e : seg->outputs) listed = listed || e.name == o;
            if (!listed) seg->outputs.push_back(output_spec(o, g, m));
        }
        seg->members.push_back(m);
    }
    cudaSetDevice(c->device);
    cudaError_t e = cudaSuccess;
    // Stages that carry state (TemporalFilter, Quality) keep it in request order
    // on one stream: the whole pair's, or with the split the back stream's,
    // where every stage after the Disparity member runs.
    bool carries = false, carries_before = false, full_search = false;
    for (const Member &m : seg->members) {
        const bool stateful = m.kind == Kind::Temporal || m.kind == Kind::Quality;
        carries = carries || stateful;
        carries_before = carries_before || (stateful && !full_search);
        full_search = full_search || (m.kind == Kind::Disparity && !m.coarse_to_fine);
    }
    seg->split = g_split_lanes && full_search && !carries_before;
    seg->n_lanes = carries && !seg->split ? 1 : kLanes;
    for (cudaStream_t *st : {&seg->upload, &seg->download, &seg->notify})
        if (!e) e = cudaStreamCreateWithFlags(st, cudaStreamNonBlocking);
    for (int k = 0; k < seg->n_lanes; ++k)
        if (!e) e = cudaStreamCreateWithFlags(&seg->lanes[k], cudaStreamNonBlocking);
    if (!e) e = seg->clock.open();
    const size_t pixels = (size_t)g.width * g.height;
    const size_t frame = (size_t)g.frame_width * g.frame_height;
    int max_disparities = 0, decimation = 1;
    size_t matcher_scratch = 0;  // the largest disparity member's
    for (const Member &m : seg->members) {
        if (m.kind == Kind::Disparity) {
            max_disparities = std::max(max_disparities, m.disparities);
            matcher_scratch = std::max(
                matcher_scratch, m.coarse_to_fine
                                     ? coarse_to_fine_scratch_bytes(g.width, g.height, m.band)
                                     : matcher_scratch_bytes(g.width, g.height, m.disparities));
        }
        if (m.kind == Kind::Cloud) decimation = m.decimation;
    }
    // Each speckle filter moves the disparity to the slot's other buffer.
    int final_disparity = 0;
    for (const Member &m : seg->members)
        if (m.kind == Kind::Speckle) final_disparity = 1 - final_disparity;
    // Bytes of each named buffer (the point cloud's grid with one spare point).
    const size_t grid_bytes = 4 * 3 * (pixels / (decimation * decimation) + 1);
    auto buffer_bytes = [&](const std::string &name) -> size_t {
        if (name == "left_frame" || name == "right_frame") return std::max<size_t>(frame, 1);
        if (name == "left" || name == "right") return pixels;
        if (name == "disparity") return 4 * pixels;
        if (name == "depth_mm") return 2 * pixels;
        if (name == "cloud_grid") return grid_bytes;
        if (name == "cloud_points") return 4;
        return 4 * 5;  // quality_sums
    };
    auto round256 = [](size_t n) { return (n + 255) & ~(size_t)255; };
    seg->entry_bytes = seg->output_bytes = 0;
    for (const Spec &spec : seg->entries) {
        seg->entry_at.push_back(seg->entry_bytes);
        seg->entry_bytes += round256(buffer_bytes(spec.name));
    }
    seg->outputs_packed = true;
    for (const Spec &spec : seg->outputs) {
        seg->output_at.push_back(seg->output_bytes);
        seg->output_bytes += round256(buffer_bytes(spec.name));
        for (const Spec &entry : seg->entries)  // a buffer both an entry and an output
            if (entry.name == spec.name && (spec.name != "disparity" || final_disparity == 0))
                seg->outputs_packed = false;
    }
    for (Slot &slot : seg->slots) {
        if (!e && seg->entry_bytes) e = seg->alloc(&slot.entries, seg->entry_bytes);
        if (!e && seg->outputs_packed && seg->output_bytes)
            e = seg->alloc(&slot.outputs, seg->output_bytes);
        // A named buffer lies in the entry region when it is an entry, else in the
        // output region when it is an output, else on its own.
        auto place = [&](const char *entry, const char *output, const std::string &name,
                         void **at) -> cudaError_t {
            for (size_t k = 0; entry && k < seg->entries.size(); ++k)
                if (seg->entries[k].name == entry) {
                    *at = slot.entries + seg->entry_at[k];
                    return cudaSuccess;
                }
            for (size_t k = 0; output && seg->outputs_packed && k < seg->outputs.size(); ++k)
                if (seg->outputs[k].name == output) {
                    *at = slot.outputs + seg->output_at[k];
                    return cudaSuccess;
                }
            uint8_t *own = nullptr;
            cudaError_t err = seg->alloc(&own, buffer_bytes(name));
            *at = own;
            return err;
        };
        const char *disparity_out[2] = {final_disparity == 0 ? "disparity" : nullptr,
                                        final_disparity == 1 ? "disparity" : nullptr};
        struct Named { const char *entry, *output, *name; void **at; } named[] = {
            {"left_frame", nullptr, "left_frame", (void **)&slot.frames[0]},
            {"right_frame", nullptr, "right_frame", (void **)&slot.frames[1]},
            {"left", "left", "left", (void **)&slot.images[0]},
            {"right", "right", "right", (void **)&slot.images[1]},
            {"disparity", disparity_out[0], "disparity", (void **)&slot.disparity[0]},
            {nullptr, disparity_out[1], "disparity", (void **)&slot.disparity[1]},
            {nullptr, "depth_mm", "depth_mm", (void **)&slot.depth_mm},
            {nullptr, "cloud_grid", "cloud_grid", (void **)&slot.grid},
            {nullptr, "cloud_points", "cloud_points", (void **)&slot.kept},
            {nullptr, "quality_sums", "quality_sums", (void **)&slot.quality_sums},
        };
        for (const Named &b : named)
            if (!e) e = place(b.entry, b.output, b.name, b.at);
        for (cudaEvent_t *ev : {&slot.entered, &slot.free})
            if (!e) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    }
    const bool rectifies = std::any_of(seg->members.begin(), seg->members.end(),
                                       [](const Member &m) { return m.kind == Kind::Rectification; });
    for (int k = 0; k < seg->n_lanes; ++k) {
        if (!e && rectifies) e = seg->alloc(&seg->rectify_maps[k], 2 * pixels);
        if (!e) e = seg->alloc(&seg->depth_m[k], pixels);
        if (!e && max_disparities) e = seg->scratch[k].reserve(matcher_scratch);
        for (cudaEvent_t *ev : {&seg->carved[k], &seg->freed[k]})
            if (!e && seg->split) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    }
    if (!e) e = seg->alloc(&seg->quality_columns, 5 * (size_t)g.width);
    // What the stages carry starts over: previous = -1, missed = 0
    // (stage/temporal_filter.ex:219-226, stage/quality.ex:144-145).
    for (Member &m : seg->members) {
        if (e) break;
        if (m.kind == Kind::Temporal || m.kind == Kind::Quality) {
            e = seg->alloc(&m.previous, pixels);
            if (!e) {
                std::vector<float> minus(pixels, -1.0f);
                e = cudaMemcpy(m.previous, minus.data(), 4 * pixels, cudaMemcpyHostToDevice);
            }
        }
        if (!e && m.kind == Kind::Temporal) {
            e = seg->alloc(&m.missed, pixels);
            if (!e) e = cudaMemset(m.missed, 0, 4 * pixels);
        }
    }
    if (!e) {  // pinned staging for 2 x kSlots requests: those in flight and those read out
        std::vector<size_t> blocks;
        for (int k = 0; k < 2 * kSlots; ++k) {
            blocks.push_back(std::max<size_t>(seg->entry_bytes, 4));
            if (seg->outputs_packed) blocks.push_back(std::max<size_t>(seg->output_bytes, 4));
            else
                for (const Spec &spec : seg->outputs)
                    blocks.push_back(std::max<size_t>(spec.bytes(), 4));
        }
        e = seg->pinned.reserve(blocks);
    }
    if (e) return cuda_status(e, error, error_len, "segment allocation");
    std::lock_guard<std::mutex> lock(c->lock);
    c->segments[id] = seg;  // replaces (and, once its requests finish, frees) an older one
    return NXS_OK;
}

static void CUDART_CB request_done(void *data) {
    nxs_request *r = static_cast<nxs_request *>(data);
    if (r->callback) r->callback(r->user, r->tag);
}

extern "C" nxs_status nxs_run_async(nxs_context *c, uint32_t id, uint32_t n_members,
                                    const nxs_member_params *params, uint32_t n_entries,
                                    const nxs_tensor *entries, nxs_done_fn done, void *user,
                                    uint64_t tag, nxs_request **request, char *error,
                                    size_t error_len) {
    if (!c || !request || (n_members && !params) || (n_entries && !entries)) {
        set_error(error, error_len, "a NULL context, request, params or entries");
        return NXS_BAD_ARGUMENT;
    }
    *request = nullptr;
    std::shared_ptr<Segment> seg;
    {
        std::lock_guard<std::mutex> lock(c->lock);
        auto it = c->segments.find(id);
        if (it == c->segments.end()) {
            set_error(error, error_len, "no segment %u", id);
            return NXS_NO_SEGMENT;
        }
        seg = it->second;
    }
    const nxs_geometry &g = seg->g;
    if (n_members != seg->members.size()) {
        set_error(error, error_len, "%zu stages, got the inputs of %u", seg->members.size(),
                  n_members);
        return NXS_BAD_RUN;
    }
    std::vector<Live> live(seg->members.size());
    for (size_t i = 0; i < seg->members.size(); ++i) {
        std::string why;
        if (!parse_live(seg->members[i], g, params[i], &live[i], &why)) {
            set_error(error, error_len, "%s", why.c_str());
            return NXS_BAD_RUN;
        }
    }
    // Match the entries to the segment's: name, type and shape.
    std::vector<const nxs_tensor *> matched(seg->entries.size(), nullptr);
    for (size_t k = 0; k < seg->entries.size(); ++k) {
        const Spec &spec = seg->entries[k];
        for (uint32_t i = 0; i < n_entries; ++i)
            if (entries[i].name && spec.name == entries[i].name) matched[k] = &entries[i];
        const nxs_tensor *t = matched[k];
        if (!t) {
            set_error(error, error_len, "missing entry %s", spec.name.c_str());
            return NXS_BAD_RUN;
        }
        bool shape_ok = t->type == spec.type && t->rank == spec.dims.size();
        for (size_t d = 0; shape_ok && d < spec.dims.size(); ++d)
            shape_ok = t->dims[d] == spec.dims[d];
        if (!shape_ok || !t->data || t->bytes != spec.bytes()) {
            set_error(error, error_len, "entry %s: expected type %u of shape {%u, %u}, %zu bytes",
                      spec.name.c_str(), spec.type, spec.dims[0], spec.dims[1], spec.bytes());
            return NXS_BAD_RUN;
        }
    }

    cudaSetDevice(c->device);
    auto *r = new nxs_request();
    r->segment = seg;
    r->callback = done;
    r->user = user;
    r->tag = tag;
    cudaError_t e = cudaSuccess;
    const size_t n = seg->members.size();
    r->marks.resize(n + 1, nullptr);
    for (size_t i = 0; i <= n && !e; ++i) e = seg->events.take(true, &r->marks[i]);
    if (!e) e = seg->events.take(true, &r->done);  // timed: the completion time is read from it
    // Stage the entries in pinned memory now: the caller's buffers are only
    // borrowed for the call.
    uint8_t *staged = nullptr;
    if (!e) {
        staged = static_cast<uint8_t *>(seg->pinned.take(std::max<size_t>(seg->entry_bytes, 4)));
        if (!staged) e = cudaErrorMemoryAllocation;
        else r->pinned.push_back(staged);
    }
    for (size_t k = 0; k < seg->entries.size() && !e; ++k)
        memcpy(staged + seg->entry_at[k], matched[k]->data, seg->entries[k].bytes());
    std::vector<void *> out_host(seg->outputs.size(), nullptr);
    uint8_t *out_block = nullptr;  // the outputs' one pinned block, when packed
    if (!e && seg->outputs_packed) {
        out_block =
            static_cast<uint8_t *>(seg->pinned.take(std::max<size_t>(seg->output_bytes, 4)));
        if (!out_block) e = cudaErrorMemoryAllocation;
        else {
            r->pinned.push_back(out_block);
            for (size_t k = 0; k < seg->outputs.size(); ++k)
                out_host[k] = out_block + seg->output_at[k];
        }
    }
    for (size_t k = 0; k < seg->outputs.size() && !e && !seg->outputs_packed; ++k) {
        out_host[k] = seg->pinned.take(std::max<size_t>(seg->outputs[k].bytes(), 4));
        if (!out_host[k]) e = cudaErrorMemoryAllocation;
        else r->pinned.push_back(out_host[k]);
    }
    if (e) {
        nxs_request_free(r);
        return cuda_status(e, error, error_len, "request set-up");
    }

    std::lock_guard<std::mutex> order(seg->order);
    const uint64_t sequence = seg->sequence++;
    Slot &slot = seg->slots[sequence % kSlots];
    // Split segments: `lane` picks the scratch and depth map; the pair starts
    // on lanes[0] and moves to lanes[1] after its path volumes.
    const int lane = (int)(sequence % (uint64_t)seg->n_lanes);
    cudaStream_t s = seg->lanes[seg->split ? 0 : lane];
    const size_t pixels = (size_t)g.width * g.height;
    // Upload, once the slot's last request has downloaded its outputs.
    e = cudaStreamWaitEvent(seg->upload, slot.free, 0);
    if (!e && seg->entry_bytes)
        e = cudaMemcpyAsync(slot.entries, staged, seg->entry_bytes, cudaMemcpyHostToDevice,
                            seg->upload);
    if (!e) e = cudaEventRecord(slot.entered, seg->upload);
    // Compute on the request's lane.
    if (!e) e = cudaStreamWaitEvent(s, slot.entered, 0);
    int current = 0;  // which of the slot's disparity buffers holds the disparity so far
    for (size_t i = 0; i < n && !e; ++i) {
        Member &m = seg->members[i];
        const Live &l = live[i];
        e = cudaEventRecord(r->marks[i], s);
        if (e) break;
        switch (m.kind) {
        case Kind::Rectification: {
            // The map of the lane whose stream runs this, remade only for new cameras.
            const int k = seg->n_lanes > 1 && s == seg->lanes[1] ? 1 : 0;
            if (!seg->rectify_mapped[k] ||
                memcmp(seg->rectify_cameras[k], l.cameras, sizeof l.cameras) != 0) {
                seg->rectify_mapped[k] = false;
                e = launch_rectify_maps(l.cameras[0], l.cameras[1], g.frame_width,
                                        g.frame_height, g.width, g.height, seg->rectify_maps[k],
                                        s);
                if (!e) {
                    memcpy(seg->rectify_cameras[k], l.cameras, sizeof l.cameras);
                    seg->rectify_mapped[k] = true;
                }
            }
            if (!e)
                e = launch_rectify_mapped(slot.frames[0], slot.frames[1], g.frame_width,
                                          g.frame_height, seg->rectify_maps[k], g.width, g.height,
                                          slot.images[0], slot.images[1], s);
            break;
        }
        case Kind::Disparity: {
            if (m.coarse_to_fine) {
                e = run_coarse_to_fine(slot.images[0], slot.images[1], g.width, g.height, m.paths,
                                       m.coarse_paths, m.band, m.margin, m.census, l.sgm.p1,
                                       l.sgm.p2, l.sgm.uniqueness, 1, seg->scratch[lane].ptr,
                                       slot.disparity[current], nullptr, s);
                break;
            }
            MatcherScratch ms =
                carve_matcher_scratch(seg->scratch[lane].ptr, g.width, g.height, m.disparities);
            if (!seg->split) {
                e = run_matcher(slot.images[0], slot.images[1], g.width, g.height, m.disparities,
                                m.paths, l.sgm.p1, l.sgm.p2, l.sgm.uniqueness, 1, ms,
                                slot.disparity[current], s);
                break;
            }
            // The front half once the pair two before has read this scratch (an
            // event not yet recorded is no wait); the rest on the back stream.
            cudaStream_t back = seg->lanes[1];
            e = cudaStreamWaitEvent(s, seg->freed[lane], 0);
            if (!e)
                e = run_matcher_front(slot.images[0], slot.images[1], g.width, g.height,
                                      m.disparities, m.paths, l.sgm.p1, l.sgm.p2, ms, s);
            if (!e) e = cudaEventRecord(seg->carved[lane], s);
            if (!e) e = cudaStreamWaitEvent(back, seg->carved[lane], 0);
            if (!e)
                e = run_matcher_back(g.width, g.height, m.disparities, m.paths,
                                     l.sgm.uniqueness, 1, ms, slot.disparity[current], back,
                                     true);
            if (!e) e = cudaEventRecord(seg->freed[lane], back);
            s = back;
            break;
        }
        case Kind::Speckle:
            e = launch_despeckle(slot.disparity[current], g.width, g.height, l.a, l.b, m.radius,
                                 slot.disparity[1 - current], s);
            current = 1 - current;
            break;
        case Kind::Temporal:
            e = launch_temporal(slot.disparity[current], m.previous, m.missed, pixels, l.a, l.b,
                                l.c, m.max_missed, s);
            break;
        case Kind::Depth:
            e = launch_depth(slot.disparity[current], pixels, l.a, l.b, slot.depth_mm,
                             seg->depth_m[lane], s);
            break;
        case Kind::Cloud:
            e = launch_cloud(seg->depth_m[lane], g.width, g.height, m.decimation, l.a, l.b, l.c,
                             m.min_depth_m, m.max_depth_m, slot.grid, slot.kept, s);
            break;
        case Kind::Quality:
            e = launch_quality(slot.disparity[current], m.previous, g.width, g.height,
                               seg->quality_columns, slot.quality_sums, s);
            break;
        }
    }
    if (!e) e = cudaEventRecord(r->marks[n], s);  // the last member done: outputs ready
    // Download the outputs into the request's pinned block(s).
    if (!e) e = cudaStreamWaitEvent(seg->download, r->marks[n], 0);
    if (!e && seg->outputs_packed && seg->output_bytes)
        e = cudaMemcpyAsync(out_block, slot.outputs, seg->output_bytes, cudaMemcpyDeviceToHost,
                            seg->download);
    r->outputs.resize(seg->outputs.size());
    r->names.resize(seg->outputs.size());
    for (size_t k = 0; k < seg->outputs.size() && !e; ++k) {
        const Spec &spec = seg->outputs[k];
        const void *src = spec.name == "left"           ? (const void *)slot.images[0]
                          : spec.name == "right"        ? (const void *)slot.images[1]
                          : spec.name == "disparity"    ? (const void *)slot.disparity[current]
                          : spec.name == "depth_mm"     ? (const void *)slot.depth_mm
                          : spec.name == "cloud_grid"   ? (const void *)slot.grid
                          : spec.name == "cloud_points" ? (const void *)slot.kept
                                                        : (const void *)slot.quality_sums;
        if (!seg->outputs_packed)
            e = cudaMemcpyAsync(out_host[k], src, spec.bytes(), cudaMemcpyDeviceToHost,
                                seg->download);
        r->names[k] = spec.name;
        nxs_tensor &t = r->outputs[k];
        t.name = r->names[k].c_str();
        t.type = spec.type;
        t.rank = (uint32_t)spec.dims.size();
        for (size_t d = 0; d < 4; ++d) t.dims[d] = d < spec.dims.size() ? spec.dims[d] : 0;
        t.data = out_host[k];
        t.bytes = spec.bytes();
    }
    if (!e) e = cudaEventRecord(slot.free, seg->download);
    if (!e) e = cudaEventRecord(r->done, seg->download);
    if (!e && done) e = cudaStreamWaitEvent(seg->notify, r->done, 0);
    if (!e && done) e = cudaLaunchHostFunc(seg->notify, request_done, r);
    if (e) {
        // The streams are still ordered: wait for what was enqueued before freeing.
        for (cudaStream_t st : seg->streams()) cudaStreamSynchronize(st);
        nxs_request_free(r);
        return cuda_status(e, error, error_len, "enqueueing the request");
    }
    *request = r;
    return NXS_OK;
}

extern "C" nxs_status nxs_request_poll(nxs_request *r, char *error, size_t error_len) {
    if (!r) return NXS_BAD_ARGUMENT;
    cudaSetDevice(r->segment->device);
    cudaError_t e = cudaEventQuery(r->done);
    if (e == cudaErrorNotReady) return NXS_PENDING;
    return cuda_status(e, error, error_len, "request");
}

extern "C" nxs_status nxs_request_wait(nxs_request *r, int64_t timeout_ms, char *error,
                                       size_t error_len) {
    if (!r) return NXS_BAD_ARGUMENT;
    cudaSetDevice(r->segment->device);
    if (timeout_ms < 0) return cuda_status(cudaEventSynchronize(r->done), error, error_len, "request");
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
    int spins = 0;
    for (;;) {
        cudaError_t e = cudaEventQuery(r->done);
        if (e != cudaErrorNotReady) return cuda_status(e, error, error_len, "request");
        if (std::chrono::steady_clock::now() >= deadline) {
            set_error(error, error_len, "timeout after %lld ms", (long long)timeout_ms);
            return NXS_TIMEOUT;
        }
        if (++spins < 2000) std::this_thread::yield();
        else std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

extern "C" nxs_status nxs_request_outputs(nxs_request *r, uint32_t *n_outputs,
                                          const nxs_tensor **outputs) {
    if (!r || !n_outputs || !outputs) return NXS_BAD_ARGUMENT;
    nxs_status s = nxs_request_poll(r, nullptr, 0);
    if (s) return s;
    *n_outputs = (uint32_t)r->outputs.size();
    *outputs = r->outputs.data();
    return NXS_OK;
}

extern "C" nxs_status nxs_request_times(nxs_request *r, uint32_t *n_members,
                                        const uint32_t **times_us) {
    if (!r || !n_members || !times_us) return NXS_BAD_ARGUMENT;
    nxs_status s = nxs_request_poll(r, nullptr, 0);
    if (s) return s;
    if (!r->timed) {
        r->times_us.clear();
        for (size_t i = 0; i + 1 < r->marks.size(); ++i) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, r->marks[i], r->marks[i + 1]);
            double us = std::round((double)ms * 1000.0);
            r->times_us.push_back(us > 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)us);
        }
        r->timed = true;
    }
    *n_members = (uint32_t)r->times_us.size();
    *times_us = r->times_us.data();
    return NXS_OK;
}

extern "C" uint64_t nxs_request_done_ns(nxs_request *r) {
    if (!r) return 0;
    uint64_t ns = r->done_ns.load();
    if (ns) return ns;
    cudaSetDevice(r->segment->device);
    if (cudaEventQuery(r->done) != cudaSuccess) return 0;
    ns = r->segment->clock.at(r->done);
    r->done_ns.store(ns);
    return ns;
}

extern "C" nxs_status nxs_device_memory(nxs_context *c, uint64_t *free_bytes,
                                        uint64_t *total_bytes) {
    if (!c || !free_bytes || !total_bytes) return NXS_BAD_ARGUMENT;
    cudaSetDevice(c->device);
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) return NXS_CUDA_ERROR;
    *free_bytes = f;
    *total_bytes = t;
    return NXS_OK;
}

extern "C" void nxs_request_free(nxs_request *r) {
    if (!r) return;
    cudaSetDevice(r->segment->device);
    if (r->done) cudaEventSynchronize(r->done);
    for (cudaEvent_t ev : r->marks) r->segment->events.give(true, ev);
    r->segment->events.give(true, r->done);
    for (void *p : r->pinned) r->segment->pinned.give(p);
    delete r;
}

extern "C" nxs_status nxs_release(nxs_context *c, uint32_t id) {
    if (!c) return NXS_BAD_ARGUMENT;
    std::shared_ptr<Segment> seg;
    {
        std::lock_guard<std::mutex> lock(c->lock);
        auto it = c->segments.find(id);
        if (it == c->segments.end()) return NXS_NO_SEGMENT;
        seg = it->second;
        c->segments.erase(it);
    }
    cudaSetDevice(c->device);
    for (cudaStream_t st : seg->streams()) cudaStreamSynchronize(st);
    return NXS_OK;
}
