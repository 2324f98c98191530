/*
 * The reference's shader pipelines, dispatched on the CPU (TEST
 * INFRASTRUCTURE ONLY: the oracle's cross-check against the reference).
 *
 * nxs_ref_sgm follows NxStereo.Vulkan.pipeline/1 (lib/nx_stereo/vulkan.ex:
 * 262-333), the pipeline NxStereo.sgm/3 runs on a GPU (lib/nx_stereo.ex:
 * 64-74): the census of both images into 8-row feature tiles, the forward
 * and reverse horizontal scans (summed in pairs), the six line scans in the
 * order of vulkan.ex @lines (the paired ones adding their partner's
 * volume), the selection, the left-right check and the 3x3 median; with 3
 * paths the vertical scan selects as it goes, and at 128 disparities the
 * two horizontal scans are the fused one. Every stage's buffers bind in the
 * order the pipeline lists its inputs, then its outputs, and every stage
 * specialises WIDTH and HEIGHT, as vulkan.ex does.
 */
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "glsl_cpu.h"

struct nxs_module_entry {
    const char *name;
    const nxs_module *(*get)();
};
extern const nxs_module_entry nxs_modules[];

namespace {

const nxs_module *find(const std::string &name) {
    for (const nxs_module_entry *e = nxs_modules; e->name; ++e)
        if (name == e->name) return e->get();
    return nullptr;
}

struct Runner {
    int subgroup_size;
    char *error;
    int error_size;
    int status = 0;

    // Binds `buffers` to bindings 0, 1, ... and the constants by id, then
    // dispatches `groups` workgroups.
    void run(const std::string &name, uvec3 groups, const std::vector<void *> &buffers,
             const std::vector<std::pair<int, double>> &constants) {
        if (status) return;
        const nxs_module *m = find(name);
        if (!m) {
            std::snprintf(error, error_size, "no shader variant %s", name.c_str());
            status = -1;
            return;
        }
        for (int i = 0; i < m->binding_count; ++i) {
            const int b = m->binding[i];
            if (b >= (int)buffers.size()) {
                std::snprintf(error, error_size, "%s: binding %d has no buffer", name.c_str(), b);
                status = -1;
                return;
            }
            *m->buffer[i] = buffers[b];
        }
        for (int i = 0; i < m->spec_count; ++i)
            for (const auto &c : constants)
                if (c.first == m->spec_id[i]) {
                    if (m->spec_float[i]) *static_cast<float *>(m->spec[i]) = (float)c.second;
                    else *static_cast<int *>(m->spec[i]) = (int)c.second;
                }
        status = nxs_dispatch(m, groups, subgroup_size, error, error_size);
    }
};

uint ceil_div(uint a, uint b) { return (a + b - 1) / b; }

}  // namespace

namespace {

int sgm(const uint8_t *left, const uint8_t *right, int width, int height, int disparities,
        int paths, float p1, float p2, float uniqueness, float *output, float *selected,
        uint32_t *keys, int subgroup_size, char *error, int error_size) {
    if (!(width > 8 && height > 6 && width <= 4096) || (disparities != 64 && disparities != 128) ||
        (paths != 3 && paths != 8)) {
        std::snprintf(error, error_size, "sizes the reference refuses");
        return -1;
    }
    const uint W = (uint)width, H = (uint)height, D = (uint)disparities;
    const uint tile = 8;
    const size_t pixels = (size_t)W * H;
    const size_t tiled_pixels = (size_t)W * ceil_div(H, tile) * tile;
    const size_t volume_words = tiled_pixels * D / 4;
    const uint rows = ceil_div(H, tile);
    const std::string d = "_d" + std::to_string(disparities);
    std::vector<int> l(pixels), r(pixels);
    for (size_t i = 0; i < pixels; ++i) {
        l[i] = left[i];
        r[i] = right[i];
    }
    float params[3] = {p1, p2, uniqueness};
    std::vector<uint> features(tiled_pixels * 4, 0u);
    auto volume = [&]() { return std::vector<uint>(volume_words, 0u); };
    std::vector<uint> forward = volume(), costs = volume(), forward_reverse = volume();
    std::vector<float> disparity(pixels, 0.0f), consistent(pixels, 0.0f);
    std::vector<uint> winners(pixels, 0u);
    const std::vector<std::pair<int, double>> size = {{0, width}, {1, height}};
    Runner run{subgroup_size, error, error_size};

    // census_stage/3 (vulkan.ex:152-170)
    run.run("census", uvec3(ceil_div(W, 128 / 8), ceil_div(H, 4 * 8), 1),
            {l.data(), r.data(), features.data()}, size);
    // the horizontal scans (vulkan.ex:312-325)
    if (disparities == 128 && paths == 3) {
        run.run("cost_horizontal_d128", uvec3(rows, 1, 1),
                {params, features.data(), forward_reverse.data(), costs.data()}, size);
    } else {
        run.run("cost_forward" + d, uvec3(rows, 1, 1),
                {params, features.data(), forward.data(), costs.data()}, size);
        run.run("cost_reverse" + d, uvec3(rows, 1, 1),
                {params, costs.data(), forward.data(), forward_reverse.data()}, size);
    }
    if (paths == 8) {
        // @lines (vulkan.ex:92-99): {stage, output, partner}
        std::vector<uint> up = volume(), up_down_right = volume(), down_left = volume(),
                          down_left_up_right = volume(), down = volume(), down_up_left = volume();
        struct Line {
            const char *stage;
            std::vector<uint> *out, *partner;
        } lines[] = {
            {"cost_up", &up, nullptr},
            {"cost_down_right", &up_down_right, &up},
            {"cost_down_left", &down_left, nullptr},
            {"cost_up_right", &down_left_up_right, &down_left},
            {"cost_down", &down, nullptr},
            {"cost_up_left", &down_up_left, &down},
        };
        for (const Line &line : lines) {
            const std::string stage = line.stage;
            const uint count = (stage == "cost_up" || stage == "cost_down") ? W : W + H - 1;
            std::vector<void *> buffers = {params, costs.data()};
            if (line.partner) buffers.push_back(line.partner->data());
            buffers.push_back(line.out->data());
            run.run(stage + d, uvec3(ceil_div(count, tile), 1, 1), buffers, size);
        }
        run.run("select_8" + d, uvec3(W, rows, 1),
                {params, forward_reverse.data(), up_down_right.data(), down_left_up_right.data(),
                 down_up_left.data(), disparity.data(), winners.data()},
                size);
    } else {
        run.run("cost_down_select" + d, uvec3(ceil_div(W, tile), 1, 1),
                {params, costs.data(), forward_reverse.data(), disparity.data(), winners.data()},
                size);
    }
    // check_and_median_stages/2 (vulkan.ex:173-193)
    run.run("consistency", uvec3(H, 1, 1), {disparity.data(), winners.data(), consistent.data()},
            size);
    run.run("median", uvec3(ceil_div((uint)pixels, 128), 1, 1), {consistent.data(), output}, size);
    if (run.status == 0 && selected) std::memcpy(selected, disparity.data(), pixels * sizeof(float));
    if (run.status == 0 && keys) std::memcpy(keys, winners.data(), pixels * sizeof(uint32_t));
    return run.status;
}

}  // namespace

/* NxStereo.sgm/3 as the reference's shaders compute it; `selected` and `keys`
 * (either may be NULL) receive the selection's outputs before the check. */
extern "C" int nxs_ref_sgm(const uint8_t *left, const uint8_t *right, int width, int height,
                           int disparities, int paths, float p1, float p2, float uniqueness,
                           float *output, float *selected, uint32_t *keys, int subgroup_size,
                           char *error, int error_size) {
    return sgm(left, right, width, height, disparities, paths, p1, p2, uniqueness, output,
               selected, keys, subgroup_size, error, error_size);
}

/* ---- the stages around the matcher, as lib/nx_stereo/kernels.ex dispatches
 * their shaders: every buffer a stage reads or writes is bound in the order
 * its pipeline lists inputs, then outputs; params are the f32 vector
 * Kernels.scalars/1 makes. */

/* Kernels.rectify/4 for a u8 frame (kernels.ex:49-83: rectify.comp with
 * WORDS=0, four pixels a thread, the frame read as 32-bit words). `camera`
 * is k (9), d (5), inverse_pr (9). The image width must be a multiple of 4,
 * as the shader writes width / 4 words a row. */
extern "C" int nxs_ref_rectify(const uint8_t *frame, int frame_width, int frame_height,
                               const float *camera, int width, int height, uint8_t *image,
                               char *error, int error_size) {
    if (width % 4 != 0) {
        std::snprintf(error, error_size, "the shader writes whole words: width %% 4 != 0");
        return -1;
    }
    const size_t frame_bytes = (size_t)frame_width * frame_height;
    std::vector<uint> words((frame_bytes + 3) / 4, 0u);
    std::memcpy(words.data(), frame, frame_bytes);
    std::vector<float> vector(camera, camera + 23);
    std::vector<uint> packed((size_t)height * (width / 4), 0u);
    Runner run{32, error, error_size};
    run.run("rectify_bytes", uvec3(ceil_div((uint)width / 4, 64), (uint)height, 1),
            {words.data(), vector.data(), packed.data()},
            {{0, frame_width}, {1, frame_height}, {2, width}, {3, height},
             {4, (double)((float)frame_width / (float)width)},
             {5, (double)((float)frame_height / (float)height)}});
    if (run.status == 0) std::memcpy(image, packed.data(), (size_t)width * height);
    return run.status;
}

/* Kernels.despeckle/3 (kernels.ex:114-134): radius 3, params min_support, max_diff. */
extern "C" int nxs_ref_despeckle(const float *disparity, int width, int height,
                                 float min_support, float max_diff, float *output, char *error,
                                 int error_size) {
    float params[2] = {min_support, max_diff};
    std::vector<float> in(disparity, disparity + (size_t)width * height);
    Runner run{32, error, error_size};
    run.run("despeckle", uvec3(ceil_div((uint)width, 64), ceil_div((uint)height, 16), 1),
            {in.data(), params, output}, {{0, width}, {1, height}});
    return run.status;
}

/* Kernels.temporal_filter/5 (kernels.ex:168-189): params alpha, delta, hold;
 * a pixel count that is a multiple of 4. */
extern "C" int nxs_ref_temporal(const float *current, const float *previous, const float *missed,
                                int pixels, float alpha, float delta, float hold,
                                float *filtered, float *missed_out, char *error,
                                int error_size) {
    if (pixels % 4 != 0) {
        std::snprintf(error, error_size, "the shader takes whole vec4s: pixels %% 4 != 0");
        return -1;
    }
    float params[3] = {alpha, delta, hold};
    std::vector<float> c(current, current + pixels), p(previous, previous + pixels),
        m(missed, missed + pixels);
    Runner run{32, error, error_size};
    run.run("temporal_filter", uvec3(ceil_div(ceil_div((uint)pixels, 4), 64), 1, 1),
            {c.data(), p.data(), m.data(), params, filtered, missed_out}, {{0, pixels}});
    return run.status;
}

/* Kernels.depth/3 (kernels.ex:191-212): params focal_length_px, baseline_m;
 * an even pixel count; millimetres as 16-bit values two a word. */
extern "C" int nxs_ref_depth(const float *disparity, int pixels, float focal_length_px,
                             float baseline_m, uint16_t *depth_mm, float *depth_m, char *error,
                             int error_size) {
    if (pixels % 2 != 0) {
        std::snprintf(error, error_size, "the shader takes whole vec2s: pixels %% 2 != 0");
        return -1;
    }
    float params[2] = {focal_length_px, baseline_m};
    std::vector<float> d(disparity, disparity + pixels);
    std::vector<uint> mm(pixels / 2, 0u);
    Runner run{32, error, error_size};
    run.run("depth", uvec3(ceil_div(ceil_div((uint)pixels, 2), 64), 1, 1),
            {d.data(), params, mm.data(), depth_m}, {{0, pixels}});
    if (run.status == 0) std::memcpy(depth_mm, mm.data(), sizeof(uint16_t) * pixels);
    return run.status;
}

/* Kernels.point_cloud/4 (kernels.ex:214-245): the grid rows, then the sum of
 * the rows' kept counts; params focal_length_px, cx, cy, min and max depth. */
extern "C" int nxs_ref_point_cloud(const float *depth_m, int width, int height, int decimation,
                                   float focal_length_px, float cx, float cy, float nearest_m,
                                   float farthest_m, float *grid, float *kept, char *error,
                                   int error_size) {
    const int grid_height = height / decimation, grid_width = width / decimation;
    float params[5] = {focal_length_px, cx, cy, nearest_m, farthest_m};
    std::vector<float> d(depth_m, depth_m + (size_t)width * height);
    std::vector<float> rows(grid_height, 0.0f);
    Runner run{32, error, error_size};
    run.run("point_cloud_rows", uvec3((uint)grid_height, 1, 1),
            {d.data(), params, grid, rows.data()},
            {{0, width}, {1, grid_width}, {2, decimation}});
    run.run("column_sums", uvec3(1, 1, 1), {rows.data(), kept}, {{0, grid_height}, {1, 1}});
    return run.status;
}

/* Kernels.disparity_sums/3 (kernels.ex:247-268): the five sums Stage.Quality
 * reads, as per-row partial sums added by column. */
extern "C" int nxs_ref_quality(const float *current, const float *previous, int width,
                               int height, float *sums, char *error, int error_size) {
    std::vector<float> c(current, current + (size_t)width * height),
        p(previous, previous + (size_t)width * height), partials((size_t)height * 5, 0.0f);
    Runner run{32, error, error_size};
    run.run("disparity_rows", uvec3((uint)height, 1, 1), {c.data(), p.data(), partials.data()},
            {{0, width}});
    run.run("column_sums", uvec3(5, 1, 1), {partials.data(), sums}, {{0, height}, {1, 5}});
    return run.status;
}

/* ---- the coarse-to-fine search ---- */

namespace {

// A zero-filled buffer of `words` 32-bit words, with a guard of zero words
// past its end (the sizes are vulkan.ex's; the guard only keeps a read one
// past them inside this process's memory).
std::vector<uint> words_buffer(size_t words) { return std::vector<uint>(words + 256, 0u); }

uvec3 linear_workgroups(uint count) {  // vulkan.ex:257-260
    const uint rows = ceil_div(count, 65535);
    return uvec3(ceil_div(count, rows), rows, 1);
}

}  // namespace

/* NxStereo.Vulkan.band_pipeline/1 (lib/nx_stereo/vulkan.ex:196-255), the
 * pipeline NxStereo.sgm_band/4 runs on a GPU (lib/nx_stereo.ex:282-321):
 * `window` 0 sparse 9x7, 1 dense 9x5, 2 dense 9x5 with the blended centre. */
extern "C" int nxs_ref_sgm_band(const uint8_t *left, const uint8_t *right, const int32_t *base,
                                int width, int height, int disparities, int paths, int band,
                                int window, float p1, float p2, float uniqueness, float *output,
                                int subgroup_size, char *error, int error_size) {
    if (!(width > 8 && height > 6 && width <= 4096) || (disparities != 64 && disparities != 128) ||
        (paths != 3 && paths != 8) || !(band == 8 || band == 16 || band == 32 || band == 64) ||
        window < 0 || window > 2) {
        std::snprintf(error, error_size, "sizes or settings the reference refuses");
        return -1;
    }
    const uint W = (uint)width, H = (uint)height;
    const size_t pixels = (size_t)W * H;
    const size_t tiled_pixels = (size_t)W * ceil_div(H, 8) * 8;
    const uint cost_words = ceil_div((uint)band * 6, 32);
    const std::string b = "_b" + std::to_string(band);
    const uint lines_per_group = band >= 32 ? 64 / (band / 4) : 64;
    const uint diagonals = W >= H ? W : W + H - 1;
    std::vector<int> l(pixels), r(pixels), bases(base, base + pixels);
    for (size_t i = 0; i < pixels; ++i) {
        l[i] = left[i];
        r[i] = right[i];
    }
    bases.resize(pixels + 256, 0);
    float params[3] = {p1, p2, uniqueness};
    std::vector<uint> features = words_buffer(tiled_pixels * 4);
    std::vector<uint> costs = words_buffer(pixels * cost_words);
    std::vector<uint> columns = words_buffer(pixels * (cost_words + 1));
    std::vector<float> disparity(pixels, 0.0f), consistent(pixels, 0.0f);
    std::vector<uint> winners = words_buffer(pixels);
    const std::vector<std::pair<int, double>> size = {{0, width}, {1, height}};
    const std::vector<std::pair<int, double>> with_range = {
        {0, width}, {1, height}, {2, disparities}};
    Runner run{subgroup_size, error, error_size};
    auto lines_of = [&](const char *kind) {
        return std::string(kind) == "rows" ? H : std::string(kind) == "columns" ? W : diagonals;
    };

    static const char *census_stage[3] = {"census", "census_dense", "census_blend"};
    run.run(census_stage[window], uvec3(ceil_div(W, 128 / 8), ceil_div(H, 4 * 8), 1),
            {l.data(), r.data(), features.data()}, size);
    run.run("band_cost" + b, uvec3(ceil_div(W, 64), ceil_div(H, 4), 1),
            {features.data(), bases.data(), costs.data()}, with_range);
    // the horizontal scans over the column-major copy (vulkan.ex:218-223)
    std::vector<uint> horizontal = words_buffer(pixels * band / 4);
    run.run("band_transpose_costs" + b, uvec3(ceil_div(W, 8), ceil_div(H, 8), 1),
            {costs.data(), bases.data(), columns.data()}, size);
    run.run("band_scan_horizontal" + b, uvec3(ceil_div(lines_of("rows"), lines_per_group), 1, 1),
            {params, columns.data(), horizontal.data()}, size);
    std::vector<std::vector<uint>> volumes;
    std::vector<void *> select_inputs = {params, bases.data()};
    if (paths == 8 && band >= 32) {
        // opposite pairs accumulated into ten-bit sums (vulkan.ex:225-241)
        const struct {
            const char *stage, *kind;
        } wide[3] = {{"band_aggregate_vertical", "columns"},
                     {"band_aggregate_diagonal", "diagonals"},
                     {"band_aggregate_antidiagonal", "diagonals"}};
        void *previous = horizontal.data();
        for (const auto &w : wide) {
            volumes.push_back(words_buffer(pixels * band * 10 / 32));
            run.run(std::string(w.stage) + b,
                    uvec3(ceil_div(lines_of(w.kind), lines_per_group), 1, 1),
                    {params, costs.data(), bases.data(), previous, volumes.back().data()}, size);
            previous = volumes.back().data();
        }
        select_inputs.push_back(previous);
    } else {
        // @band_scans (vulkan.ex:101-108): {stage, lines, directions}
        struct Scan {
            const char *stage, *kind;
            uint directions;
        };
        std::vector<Scan> scans;
        if (paths == 3) scans = {{"band_scan_down", "columns", 1}};
        else
            scans = {{"band_scan_down_up", "columns", 2},
                     {"band_scan_down_diagonals", "diagonals", 2},
                     {"band_scan_up_diagonals", "diagonals", 2}};
        select_inputs.push_back(horizontal.data());
        volumes.reserve(scans.size());
        for (const Scan &scan : scans) {
            volumes.push_back(words_buffer(scan.directions * pixels * band / 4));
            run.run(std::string(scan.stage) + b,
                    uvec3(scan.directions * ceil_div(lines_of(scan.kind), lines_per_group), 1, 1),
                    {params, costs.data(), bases.data(), volumes.back().data()}, size);
            select_inputs.push_back(volumes.back().data());
        }
    }
    select_inputs.push_back(disparity.data());
    select_inputs.push_back(winners.data());
    run.run((paths == 8 ? "band_select_8" : "band_select") + b,
            linear_workgroups(ceil_div((uint)(pixels * (band / 4)), 64)), select_inputs,
            with_range);
    run.run("consistency", uvec3(H, 1, 1), {disparity.data(), winners.data(), consistent.data()},
            size);
    run.run("median", uvec3(ceil_div((uint)pixels, 128), 1, 1), {consistent.data(), output}, size);
    return run.status;
}

/* NxStereo.sgm_coarse_to_fine/3 (lib/nx_stereo.ex:160-225) as the reference
 * runs it on a GPU: Vulkan.shrink_pipeline/2, sgm/3's pipeline on the half
 * pair at 64 disparities, Vulkan.band_base_pipeline/4, then band_pipeline/1
 * over 128 disparities. `base_out` (may be NULL) receives the bases. */
extern "C" int nxs_ref_sgm_coarse_to_fine(const uint8_t *left, const uint8_t *right, int width,
                                          int height, int paths, int coarse_paths, int band,
                                          int margin, int window, float p1, float p2,
                                          float uniqueness, float *output, int32_t *base_out,
                                          int subgroup_size, char *error, int error_size) {
    if (width % 2 || height % 2) {
        std::snprintf(error, error_size, "an odd width or height");
        return -1;
    }
    const int hw = width / 2, hh = height / 2;
    const size_t pixels = (size_t)width * height, half = (size_t)hw * hh;
    std::vector<int> l(pixels + 256, 0), r(pixels + 256, 0);
    for (size_t i = 0; i < pixels; ++i) {
        l[i] = left[i];
        r[i] = right[i];
    }
    std::vector<int> lh(half + 256, 0), rh(half + 256, 0);
    Runner run{subgroup_size, error, error_size};
    run.run("shrink", uvec3(ceil_div((uint)half, 64), 1, 1), {l.data(), r.data(), lh.data(), rh.data()},
            {{0, hw}, {1, hh}});
    if (run.status) return run.status;
    std::vector<uint8_t> lb(half), rb(half);
    for (size_t i = 0; i < half; ++i) {
        lb[i] = (uint8_t)lh[i];
        rb[i] = (uint8_t)rh[i];
    }
    std::vector<float> coarse(half + 256, 0.0f);
    int status = sgm(lb.data(), rb.data(), hw, hh, 64, coarse_paths, p1, p2, uniqueness,
                     coarse.data(), nullptr, nullptr, subgroup_size, error, error_size);
    if (status) return status;
    std::vector<int> base(pixels + 256, 0);
    run.run("band_base", uvec3(ceil_div((uint)half, 64), 1, 1), {coarse.data(), base.data()},
            {{0, width}, {1, height}, {2, margin}, {3, 128 - band}});
    if (run.status) return run.status;
    if (base_out) std::memcpy(base_out, base.data(), sizeof(int32_t) * pixels);
    return nxs_ref_sgm_band(left, right, base.data(), width, height, 128, paths, band, window, p1,
                            p2, uniqueness, output, subgroup_size, error, error_size);
}
