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
             const std::vector<std::pair<int, int>> &constants) {
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
                if (c.first == m->spec_id[i]) *m->spec[i] = c.second;
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
    const std::vector<std::pair<int, int>> size = {{0, width}, {1, height}};
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
