// The stages around the matcher: Stage.Rectification, Stage.SpeckleFilter,
// Stage.TemporalFilter, Stage.Depth, Stage.PointCloud and Stage.Quality.
// Every f32 step is rounded on its own in the reference's order (the Nx
// evaluator's, which the reference's native stages reproduce), so integer
// outputs (rectified images, depth_mm) are bit-exact.
#include "nxs_device.cuh"
#include "nxs_kernels.h"

namespace nxs {

// ---------------------------------------------------------------- rectify
// lib/nx_stereo/rectify.ex:133-207: the rectified pixel (u, v) projects into
// the frame through inverse_pr, plumb_bob distortion (the radial polynomial
// summed as 1 + (k3 r2^3 + (k2 r2^2 + k1 r2)), the order of Nx's expression,
// native/stereo_match/src/rectify.rs:116-121) and the camera matrix; it is
// scaled to the frame size at pixel centres and sampled bilinearly with 0
// outside, then rounded half away from zero and clipped to u8. rectify_source
// is the frame position a pixel samples (a function of the camera alone, so a
// segment keeps it as a map), rectify_sample the sample there.
__device__ __forceinline__ float2 rectify_source(const Camera &camera, float scale_x,
                                                 float scale_y, int u, int v) {
    const float uf = (float)u, vf = (float)v;
    const float *ir = camera.inverse_pr;
    float x = fadd(fadd(fmul(ir[0], uf), fmul(ir[1], vf)), ir[2]);
    float y = fadd(fadd(fmul(ir[3], uf), fmul(ir[4], vf)), ir[5]);
    const float w = fadd(fadd(fmul(ir[6], uf), fmul(ir[7], vf)), ir[8]);
    x = fdiv(x, w);
    y = fdiv(y, w);
    const float k1 = camera.d[0], k2 = camera.d[1], t1 = camera.d[2], t2 = camera.d[3],
                k3 = camera.d[4];
    const float r2 = fadd(fmul(x, x), fmul(y, y));
    const float cubic = fmul(fmul(fmul(k3, r2), r2), r2);
    const float square = fmul(fmul(k2, r2), r2);
    const float radial = fadd(1.0f, fadd(cubic, fadd(square, fmul(k1, r2))));
    const float xd = fadd(fadd(fmul(x, radial), fmul(fmul(fmul(2.0f, t1), x), y)),
                          fmul(t2, fadd(r2, fmul(fmul(2.0f, x), x))));
    const float yd = fadd(fadd(fmul(y, radial), fmul(t1, fadd(r2, fmul(fmul(2.0f, y), y)))),
                          fmul(fmul(fmul(2.0f, t2), x), y));
    const float *k = camera.k;
    const float map_x = fadd(fadd(fmul(k[0], xd), fmul(k[1], yd)), k[2]);
    const float map_y = fadd(fmul(k[4], yd), k[5]);
    return make_float2(fsub(fmul(fadd(map_x, 0.5f), scale_x), 0.5f),
                       fsub(fmul(fadd(map_y, 0.5f), scale_y), 0.5f));
}

__device__ __forceinline__ uint8_t rectify_sample(const uint8_t *__restrict__ frame,
                                                  int frame_width, int frame_height,
                                                  float source_x, float source_y) {
    const float fx0 = floorf(source_x), fy0 = floorf(source_y);
    const float wx = fsub(source_x, fx0), wy = fsub(source_y, fy0);
    // float -> int as the reference casts: saturating, NaN to 0.
    const int x0 = __float2int_rz(fx0), y0 = __float2int_rz(fy0);
    float corner[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int sx = x0 + (i & 1), sy = y0 + (i >> 1);
        const bool inside = sx >= 0 && sx < frame_width && sy >= 0 && sy < frame_height;
        corner[i] = inside ? (float)__ldg(frame + (size_t)sy * frame_width + sx) : 0.0f;
    }
    const float top = fadd(fmul(fsub(1.0f, wx), corner[0]), fmul(wx, corner[1]));
    const float bottom = fadd(fmul(fsub(1.0f, wx), corner[2]), fmul(wx, corner[3]));
    const float value = fadd(fmul(fsub(1.0f, wy), top), fmul(wy, bottom));
    float r = roundf(value);
    r = r < 0.0f ? 0.0f : (r > 255.0f ? 255.0f : r);
    return (uint8_t)r;
}

__device__ __forceinline__ void rectify_at(const uint8_t *__restrict__ frame, int frame_width,
                                           int frame_height, const Camera &camera, float scale_x,
                                           float scale_y, int width,
                                           uint8_t *__restrict__ rectified, int u, int v) {
    if (u >= width) return;
    const float2 source = rectify_source(camera, scale_x, scale_y, u, v);
    rectified[(size_t)v * width + u] =
        rectify_sample(frame, frame_width, frame_height, source.x, source.y);
}

__global__ void rectify_kernel(const uint8_t *__restrict__ frame, int frame_width,
                               int frame_height, const Camera camera, float scale_x,
                               float scale_y, int width, uint8_t *__restrict__ rectified) {
    follow_previous_grid();
    rectify_at(frame, frame_width, frame_height, camera, scale_x, scale_y, width, rectified,
               blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y);
}

// Both sides of a pair in one launch: blockIdx.z picks the side.
struct RectifySides {
    const uint8_t *frame[2];
    uint8_t *rectified[2];
    Camera camera[2];
};

__global__ void rectify_pair_kernel(const RectifySides sides, int frame_width, int frame_height,
                                    float scale_x, float scale_y, int width) {
    follow_previous_grid();
    const int side = blockIdx.z;
    rectify_at(sides.frame[side], frame_width, frame_height, sides.camera[side], scale_x,
               scale_y, width, sides.rectified[side], blockIdx.x * blockDim.x + threadIdx.x,
               blockIdx.y);
}

cudaError_t launch_rectify_pair(const uint8_t *left_frame, const uint8_t *right_frame,
                                int frame_width, int frame_height, const Camera &left_camera,
                                const Camera &right_camera, int width, int height,
                                uint8_t *left, uint8_t *right, cudaStream_t stream) {
    RectifySides sides;
    sides.frame[0] = left_frame;
    sides.frame[1] = right_frame;
    sides.rectified[0] = left;
    sides.rectified[1] = right;
    sides.camera[0] = left_camera;
    sides.camera[1] = right_camera;
    const float scale_x = (float)((double)frame_width / (double)width);
    const float scale_y = (float)((double)frame_height / (double)height);
    dim3 grid((width + 127) / 128, height, 2);
    return launch_after(rectify_pair_kernel, grid, dim3(128), 0, stream, sides, frame_width,
                        frame_height, scale_x, scale_y, width);
}

// The maps of both sides: maps[side][v][u] = the frame position rectified
// pixel (u, v) samples, side 0 through `left`, 1 through `right`.
struct RectifyCameras {
    Camera camera[2];
};

__global__ void rectify_maps_kernel(const RectifyCameras cameras, float scale_x, float scale_y,
                                    int width, int height, float2 *__restrict__ maps) {
    follow_previous_grid();
    const int side = blockIdx.z, u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= width) return;
    maps[((size_t)side * height + v) * width + u] =
        rectify_source(cameras.camera[side], scale_x, scale_y, u, v);
}

__global__ void rectify_mapped_kernel(const RectifySides sides, const float2 *__restrict__ maps,
                                      int frame_width, int frame_height, int width, int height) {
    follow_previous_grid();
    const int side = blockIdx.z, u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= width) return;
    const float2 source = __ldg(maps + ((size_t)side * height + v) * width + u);
    sides.rectified[side][(size_t)v * width + u] =
        rectify_sample(sides.frame[side], frame_width, frame_height, source.x, source.y);
}

cudaError_t launch_rectify_maps(const Camera &left_camera, const Camera &right_camera,
                                int frame_width, int frame_height, int width, int height,
                                float2 *maps, cudaStream_t stream) {
    RectifyCameras cameras;
    cameras.camera[0] = left_camera;
    cameras.camera[1] = right_camera;
    const float scale_x = (float)((double)frame_width / (double)width);
    const float scale_y = (float)((double)frame_height / (double)height);
    dim3 grid((width + 127) / 128, height, 2);
    return launch_after(rectify_maps_kernel, grid, dim3(128), 0, stream, cameras, scale_x,
                        scale_y, width, height, maps);
}

cudaError_t launch_rectify_mapped(const uint8_t *left_frame, const uint8_t *right_frame,
                                  int frame_width, int frame_height, const float2 *maps,
                                  int width, int height, uint8_t *left, uint8_t *right,
                                  cudaStream_t stream) {
    RectifySides sides{};
    sides.frame[0] = left_frame;
    sides.frame[1] = right_frame;
    sides.rectified[0] = left;
    sides.rectified[1] = right;
    dim3 grid((width + 127) / 128, height, 2);
    return launch_after(rectify_mapped_kernel, grid, dim3(128), 0, stream, sides, maps,
                        frame_width, frame_height, width, height);
}

cudaError_t launch_rectify(const uint8_t *frame, int frame_width, int frame_height,
                           const Camera &camera, int width, int height, uint8_t *rectified,
                           cudaStream_t stream) {
    // Scale as the reference computes it: an f64 ratio rounded to f32.
    const float scale_x = (float)((double)frame_width / (double)width);
    const float scale_y = (float)((double)frame_height / (double)height);
    dim3 grid((width + 127) / 128, height);
    return launch_after(rectify_kernel, grid, dim3(128), 0, stream, frame, frame_width,
                        frame_height, camera, scale_x, scale_y, width, rectified);
}

// ---------------------------------------------------------------- despeckle
// lib/nx_stereo/filter.ex:47-80: support = the neighbours in the
// (2r+1)^2 window, centre excluded, with n > 0 and |n - c| <= max_diff
// (-1 outside the image); keep c where c > 0 and support >= min_support.
// A 32x8 block stages its window in shared memory.
constexpr int kSpeckleX = 32, kSpeckleY = 8;

__global__ void __launch_bounds__(kSpeckleX *kSpeckleY)
    despeckle_kernel(const float *__restrict__ disparity, int width, int height,
                     float min_support, float max_diff, int radius,
                     float *__restrict__ despeckled) {
    follow_previous_grid();
    extern __shared__ float window[];
    const int tw = kSpeckleX + 2 * radius, th = kSpeckleY + 2 * radius;
    const int x0 = blockIdx.x * kSpeckleX, y0 = blockIdx.y * kSpeckleY;
    const int tid = threadIdx.y * kSpeckleX + threadIdx.x;
    for (int i = tid; i < tw * th; i += kSpeckleX * kSpeckleY) {
        int sy = y0 + i / tw - radius, sx = x0 + i % tw - radius;
        window[i] = (sy >= 0 && sy < height && sx >= 0 && sx < width)
                        ? disparity[(size_t)sy * width + sx]
                        : -1.0f;
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= width || y >= height) return;
    const float centre = window[(threadIdx.y + radius) * tw + threadIdx.x + radius];
    unsigned support = 0;
    for (int dy = 0; dy <= 2 * radius; ++dy)
        for (int dx = 0; dx <= 2 * radius; ++dx) {
            if (dy == radius && dx == radius) continue;
            const float n = window[(threadIdx.y + dy) * tw + threadIdx.x + dx];
            support += (n > 0.0f) & (fabsf(fsub(n, centre)) <= max_diff);
        }
    const bool kept = centre > 0.0f && (float)support >= min_support;
    despeckled[(size_t)y * width + x] = kept ? centre : -1.0f;
}

// The same filter with the radius fixed at compile time: a thread takes
// kSpeckleRun pixels down a column, so each window row it reads from shared
// memory (2R + 1 values, into registers) serves every one of its pixels whose
// window holds it: (kSpeckleRun + 2R) x (2R + 1) shared loads for
// kSpeckleRun x ((2R + 1)^2 - 1) comparisons. The window's global loads are
// all issued before any is stored.
constexpr int kSpeckleRun = 4;

// The filtered values of this thread's kSpeckleRun pixels down column x from
// row y (a 32 x 8 block of such runs; out[k] is pixel (x, y + k)).
template <int R>
__device__ __forceinline__ void despeckle_run(const float *__restrict__ disparity, int width,
                                              int height, float min_support, float max_diff,
                                              float (&out)[kSpeckleRun], int &x, int &y) {
    constexpr int TW = kSpeckleX + 2 * R, TH = kSpeckleY * kSpeckleRun + 2 * R;
    constexpr int THREADS = kSpeckleX * kSpeckleY, PER = (TW * TH + THREADS - 1) / THREADS;
    __shared__ float window[TH][TW];
    const int x0 = blockIdx.x * kSpeckleX, y0 = blockIdx.y * kSpeckleY * kSpeckleRun;
    const int tid = threadIdx.y * kSpeckleX + threadIdx.x;
    float v[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * THREADS;
        if (i < TW * TH) {
            const int sy = y0 + i / TW - R, sx = x0 + i % TW - R;
            v[k] = (sy >= 0 && sy < height && sx >= 0 && sx < width)
                       ? disparity[(size_t)sy * width + sx]
                       : -1.0f;
        }
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * THREADS;
        if (i < TW * TH) window[i / TW][i % TW] = v[k];
    }
    __syncthreads();
    const int tx = threadIdx.x, top = threadIdx.y * kSpeckleRun;  // the run's first window row - R
    float centre[kSpeckleRun];
    unsigned support[kSpeckleRun];
#pragma unroll
    for (int k = 0; k < kSpeckleRun; ++k) {
        centre[k] = window[top + k + R][tx + R];
        support[k] = 0;
    }
#pragma unroll
    for (int r = 0; r < kSpeckleRun + 2 * R; ++r) {
        float row[2 * R + 1];
#pragma unroll
        for (int dx = 0; dx <= 2 * R; ++dx) row[dx] = window[top + r][tx + dx];
#pragma unroll
        for (int k = 0; k < kSpeckleRun; ++k) {
            const int dy = r - k;  // the row's place in pixel k's window
            if (dy < 0 || dy > 2 * R) continue;
#pragma unroll
            for (int dx = 0; dx <= 2 * R; ++dx) {
                if (dy == R && dx == R) continue;
                const float n = row[dx];
                support[k] += (n > 0.0f) & (fabsf(fsub(n, centre[k])) <= max_diff);
            }
        }
    }
    x = x0 + tx;
    y = y0 + top;
#pragma unroll
    for (int k = 0; k < kSpeckleRun; ++k)
        out[k] = centre[k] > 0.0f && (float)support[k] >= min_support ? centre[k] : -1.0f;
}

template <int R>
__global__ void __launch_bounds__(kSpeckleX *kSpeckleY)
    despeckle_run_kernel(const float *__restrict__ disparity, int width, int height,
                         float min_support, float max_diff, float *__restrict__ despeckled) {
    follow_previous_grid();
    float out[kSpeckleRun];
    int x, y;
    despeckle_run<R>(disparity, width, height, min_support, max_diff, out, x, y);
#pragma unroll
    for (int k = 0; k < kSpeckleRun; ++k)
        if (x < width && y + k < height) despeckled[(size_t)(y + k) * width + x] = out[k];
}

cudaError_t launch_despeckle(const float *disparity, int width, int height, float min_support,
                             float max_diff, int radius, float *despeckled, cudaStream_t stream) {
    dim3 block(kSpeckleX, kSpeckleY);
    dim3 runs((width + kSpeckleX - 1) / kSpeckleX,
              (height + kSpeckleY * kSpeckleRun - 1) / (kSpeckleY * kSpeckleRun));
#define NXS_DESPECKLE(R)                                                                      \
    return launch_after(despeckle_run_kernel<R>, runs, block, 0, stream, disparity, width,    \
                        height, min_support, max_diff, despeckled)
    switch (radius) {
    case 1: NXS_DESPECKLE(1);
    case 2: NXS_DESPECKLE(2);
    case 3: NXS_DESPECKLE(3);
    case 4: NXS_DESPECKLE(4);
    case 5: NXS_DESPECKLE(5);
    default: break;
    }
#undef NXS_DESPECKLE
    dim3 grid((width + kSpeckleX - 1) / kSpeckleX, (height + kSpeckleY - 1) / kSpeckleY);
    size_t shared = sizeof(float) * (kSpeckleX + 2 * radius) * (kSpeckleY + 2 * radius);
    return launch_after(despeckle_kernel, grid, block, shared, stream, disparity, width, height,
                        min_support, max_diff, radius, despeckled);
}

// ---------------------------------------------------------------- temporal
// lib/nx_stereo/filter.ex:122-130, in place over disparity, previous, missed.
__global__ void temporal_kernel(float *__restrict__ disparity, float *__restrict__ previous,
                                float *__restrict__ missed, size_t pixels, float alpha,
                                float delta, float hold, float max_missed) {
    follow_previous_grid();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels) return;
    const float current = disparity[i], before = previous[i];
    const bool matched = current > 0.0f;
    const bool agree = matched && before > 0.0f && fabsf(fsub(current, before)) <= delta;
    const float smoothed =
        agree ? fadd(fmul(alpha, current), fmul(fsub(1.0f, alpha), before)) : current;
    const float pairs_missed = matched ? 0.0f : fadd(missed[i], 1.0f);
    const bool held = !matched && before > 0.0f && pairs_missed <= hold;
    const float filtered = held ? before : smoothed;
    disparity[i] = filtered;
    previous[i] = filtered;
    missed[i] = pairs_missed < max_missed ? pairs_missed : max_missed;
}

cudaError_t launch_temporal(float *disparity, float *previous, float *missed, size_t pixels,
                            float alpha, float delta, float hold, float max_missed,
                            cudaStream_t stream) {
    return launch_after(temporal_kernel, dim3((unsigned)((pixels + 255) / 256)), dim3(256), 0,
                        stream, disparity, previous, missed, pixels, alpha, delta, hold,
                        max_missed);
}

// ---------------------------------------------------------------- depth
// lib/nx_stereo/depth.ex:26-32: depth_m = (f * B) / d where d > 0, else 0;
// depth_mm = round(depth_m * 1000), 0 beyond 65535.
__device__ __forceinline__ float depth_of(float d, float focal_baseline, uint16_t *mm) {
    const float metres = d > 0.0f ? fdiv(focal_baseline, d) : 0.0f;
    const float rounded = roundf(fmul(metres, 1000.0f));
    *mm = rounded > 65535.0f ? 0 : (uint16_t)(rounded > 0.0f ? rounded : 0.0f);
    return metres;
}

__global__ void depth_kernel(const float *__restrict__ disparity, size_t pixels,
                             float focal_length_px, float baseline_m,
                             uint16_t *__restrict__ depth_mm, float *__restrict__ depth_m) {
    follow_previous_grid();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels) return;
    uint16_t mm;
    depth_m[i] = depth_of(disparity[i], fmul(focal_length_px, baseline_m), &mm);
    depth_mm[i] = mm;
}

cudaError_t launch_depth(const float *disparity, size_t pixels, float focal_length_px,
                         float baseline_m, uint16_t *depth_mm, float *depth_m,
                         cudaStream_t stream) {
    return launch_after(depth_kernel, dim3((unsigned)((pixels + 255) / 256)), dim3(256), 0,
                        stream, disparity, pixels, focal_length_px, baseline_m, depth_mm,
                        depth_m);
}

// ---------------------------------------------------------------- cloud
// lib/nx_stereo/depth.ex:73-89: point (i, j) from pixel (i*dec, j*dec),
// x = (u - cx) * (z / f), y = (v - cy) * (z / f), NaN outside (near, far).
__device__ __forceinline__ bool cloud_point(float z, int x, int y, float focal_length_px, float cx,
                                            float cy, float nearest_m, float farthest_m,
                                            float *point) {
    const bool in_range = z > nearest_m && z < farthest_m;
    if (in_range) {
        const float z_over_f = fdiv(z, focal_length_px);
        point[0] = fmul(fsub((float)x, cx), z_over_f);
        point[1] = fmul(fsub((float)y, cy), z_over_f);
        point[2] = z;
    } else {
        point[0] = point[1] = point[2] = __int_as_float(0x7FC00000);
    }
    return in_range;
}

__global__ void cloud_kernel(const float *__restrict__ depth_m, int width, int grid_width,
                             int grid_height, int decimation, float focal_length_px, float cx,
                             float cy, float nearest_m, float farthest_m,
                             float *__restrict__ grid, int32_t *__restrict__ kept) {
    follow_previous_grid();
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y;
    if (col >= grid_width || row >= grid_height) return;
    const int x = col * decimation, y = row * decimation;
    const float z = depth_m[(size_t)y * width + x];
    float *point = grid + 3 * ((size_t)row * grid_width + col);
    const bool in_range = cloud_point(z, x, y, focal_length_px, cx, cy, nearest_m, farthest_m,
                                      point);
    const unsigned ballot = __ballot_sync(__activemask(), in_range);
    if ((threadIdx.x & 31) == __ffs(__activemask()) - 1 && ballot)
        atomicAdd(kept, (int32_t)__popc(ballot));
}

cudaError_t launch_cloud(const float *depth_m, int width, int height, int decimation,
                         float focal_length_px, float cx, float cy, float nearest_m,
                         float farthest_m, float *grid, int32_t *kept, cudaStream_t stream) {
    const int gw = width / decimation, gh = height / decimation;
    cudaError_t e = cudaMemsetAsync(kept, 0, sizeof(int32_t), stream);
    if (e) return e;
    if (gw == 0 || gh == 0) return cudaSuccess;
    dim3 grid_dim((gw + 127) / 128, gh);
    return launch_after(cloud_kernel, grid_dim, dim3(128), 0, stream, depth_m, width, gw, gh,
                        decimation, focal_length_px, cx, cy, nearest_m, farthest_m, grid, kept);
}

// ---------------------------------------------------------------- despeckle + depth + cloud
// SpeckleFilter -> Depth -> PointCloud in one launch: each thread filters its
// run of pixels as despeckle_run_kernel does, then writes their depth as
// depth_kernel does and, for those on the decimated grid, their point as
// cloud_kernel does (the same f32 steps on the same values, so the outputs are
// the three kernels' bit for bit); a warp adds its kept points to *kept at once.
template <int R>
__global__ void __launch_bounds__(kSpeckleX *kSpeckleY)
    despeckle_depth_cloud_kernel(const float *__restrict__ disparity, int width, int height,
                                 float min_support, float max_diff, float focal_length_px,
                                 float baseline_m, int decimation, int grid_width,
                                 int grid_height, float cx, float cy, float nearest_m,
                                 float farthest_m, float *__restrict__ despeckled,
                                 uint16_t *__restrict__ depth_mm, float *__restrict__ depth_m,
                                 float *__restrict__ grid, int32_t *__restrict__ kept) {
    follow_previous_grid();
    float out[kSpeckleRun];
    int x, y;
    despeckle_run<R>(disparity, width, height, min_support, max_diff, out, x, y);
    const float focal_baseline = fmul(focal_length_px, baseline_m);
    const bool on_column = x % decimation == 0 && x / decimation < grid_width;
    unsigned points = 0;
#pragma unroll
    for (int k = 0; k < kSpeckleRun; ++k) {
        const int yk = y + k;
        if (x >= width || yk >= height) continue;
        const size_t i = (size_t)yk * width + x;
        uint16_t mm;
        const float metres = depth_of(out[k], focal_baseline, &mm);
        despeckled[i] = out[k];
        depth_m[i] = metres;
        depth_mm[i] = mm;
        if (on_column && yk % decimation == 0 && yk / decimation < grid_height) {
            const int row = yk / decimation, col = x / decimation;
            points += cloud_point(metres, x, yk, focal_length_px, cx, cy, nearest_m, farthest_m,
                                  grid + 3 * ((size_t)row * grid_width + col));
        }
    }
    points = __reduce_add_sync(kFullMask, points);
    if ((threadIdx.x & 31) == 0 && points) atomicAdd(kept, (int32_t)points);
}

cudaError_t launch_despeckle_depth_cloud(const float *disparity, int width, int height,
                                         float min_support, float max_diff, int radius,
                                         float focal_length_px, float baseline_m,
                                         int decimation, float cx, float cy, float nearest_m,
                                         float farthest_m, float *despeckled, uint16_t *depth_mm,
                                         float *depth_m, float *grid, int32_t *kept,
                                         cudaStream_t stream) {
    if (radius < 1 || radius > 5 || decimation < 1) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(kept, 0, sizeof(int32_t), stream);
    if (e) return e;
    const int gw = width / decimation, gh = height / decimation;
    dim3 block(kSpeckleX, kSpeckleY);
    dim3 runs((width + kSpeckleX - 1) / kSpeckleX,
              (height + kSpeckleY * kSpeckleRun - 1) / (kSpeckleY * kSpeckleRun));
#define NXS_TAIL(R)                                                                           \
    return launch_after(despeckle_depth_cloud_kernel<R>, runs, block, 0, stream, disparity,   \
                        width, height, min_support, max_diff, focal_length_px, baseline_m,    \
                        decimation, gw, gh, cx, cy, nearest_m, farthest_m, despeckled,        \
                        depth_mm, depth_m, grid, kept)
    switch (radius) {
    case 1: NXS_TAIL(1);
    case 2: NXS_TAIL(2);
    case 3: NXS_TAIL(3);
    case 4: NXS_TAIL(4);
    default: NXS_TAIL(5);
    }
#undef NXS_TAIL
}

// ---------------------------------------------------------------- quality
// lib/nx_stereo/diagnostics.ex:264-271 with the native reduction order
// (native/stereo_match/src/measures.rs:278-309): per column, the five planes
// [matched, value, value^2, both, |change| * both] summed down the rows in
// f64 and rounded to f32; then the columns summed in order in f64 and
// rounded. One thread per column, then one per plane.
__global__ void quality_columns_kernel(const float *__restrict__ disparity,
                                       const float *__restrict__ previous, int width, int height,
                                       float *__restrict__ column_sums) {
    follow_previous_grid();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= width) return;
    double acc[5] = {0, 0, 0, 0, 0};
    for (int y = 0; y < height; ++y) {
        const float current = disparity[(size_t)y * width + x];
        const float before = previous[(size_t)y * width + x];
        const float matched = current > 0.0f ? 1.0f : 0.0f;
        const float both = fmul(before > 0.0f ? 1.0f : 0.0f, matched);
        const float value = fmul(current, matched);
        acc[0] += (double)matched;
        acc[1] += (double)value;
        acc[2] += (double)fmul(value, value);
        acc[3] += (double)both;
        acc[4] += (double)fmul(fabsf(fsub(current, before)), both);
    }
#pragma unroll
    for (int p = 0; p < 5; ++p) column_sums[(size_t)p * width + x] = (float)acc[p];
}

__global__ void quality_total_kernel(const float *__restrict__ column_sums, int width,
                                     float *__restrict__ sums) {
    follow_previous_grid();
    const int p = threadIdx.x;
    if (p >= 5) return;
    double total = 0.0;
    for (int x = 0; x < width; ++x) total += (double)column_sums[(size_t)p * width + x];
    sums[p] = (float)total;
}

cudaError_t launch_quality(const float *disparity, float *previous, int width, int height,
                           float *column_sums, float *sums, cudaStream_t stream) {
    cudaError_t e = launch_after(quality_columns_kernel, dim3((width + 127) / 128), dim3(128), 0,
                                 stream, disparity, previous, width, height, column_sums);
    if (!e) e = launch_after(quality_total_kernel, dim3(1), dim3(32), 0, stream, column_sums,
                             width, sums);
    if (e) return e;
    return cudaMemcpyAsync(previous, disparity, sizeof(float) * (size_t)width * height,
                           cudaMemcpyDeviceToDevice, stream);
}

}  // namespace nxs
