// Caller-side frame setup: Camera4D (renderer.rs:45-65), FrameDynamics' derived values
// (renderer.rs:233-271), GpuUniforms::build (gpu.rs:147-211) and build_tables_data
// (gpu.rs:223-229), with the gamma LUT of renderer.rs:1102-1114 and the glyphs of hud.rs:473-532.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../../include/specrel_scene.h"
#include "sr_math.hpp"

using namespace srh;

namespace {
Tetrad<float> tetrad_of(const SrCamera* c) {
    Tetrad<float> t;
    for (int a = 0; a < 4; ++a) t.e[a] = V4<float>(c->e[a][0], c->e[a][1], c->e[a][2], c->e[a][3]);
    return t;
}
void store(SrCamera* c, const Tetrad<float>& t) {
    for (int a = 0; a < 4; ++a) {
        c->e[a][0] = t.e[a].t;
        c->e[a][1] = t.e[a].x;
        c->e[a][2] = t.e[a].y;
        c->e[a][3] = t.e[a].z;
    }
}
}  // namespace

extern "C" sr_status sr_camera_new(const float position[4], float fov_deg, SrCamera* out) {
    if (!position || !out) return SR_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    for (int k = 0; k < 4; ++k) out->position[k] = position[k];
    store(out, Tetrad<float>());
    out->proper_time = 0.0f;
    // f32::to_radians: self * (PI / 180.0) with the quotient folded in f32.
    const float rads_per_deg = 3.14159265358979323846f / 180.0f;
    out->fov_y_rad = fov_deg * rads_per_deg;
    return SR_OK;
}

extern "C" sr_status sr_camera_boost_local(SrCamera* cam, const float d[3]) {
    if (!cam || !d) return SR_ERR_INVALID_ARGUMENT;
    Tetrad<float> t = tetrad_of(cam);
    t.boost_local(V3<float>(d[0], d[1], d[2]));
    store(cam, t);
    return SR_OK;
}

extern "C" sr_status sr_camera_rotate_local(SrCamera* cam, float yaw, float pitch, float roll) {
    if (!cam) return SR_ERR_INVALID_ARGUMENT;
    Tetrad<float> t = tetrad_of(cam);
    t.rotate_local(yaw, pitch, roll);
    store(cam, t);
    return SR_OK;
}

extern "C" sr_status sr_uniforms_build(const SrCamera* cam, const SrRenderConfig* cfg, const SrFrameDynamics* dyn,
                                       uint32_t num_nodes, const float light_pos[4], uint32_t num_stars,
                                       SrGpuUniforms* u) {
    if (!cam || !cfg || !u || !light_pos || cfg->width == 0 || cfg->height == 0) return SR_ERR_INVALID_ARGUMENT;
    if (cfg->mode > 3 || cfg->shadow_mode > 2 || cfg->slice_mode > 3) return SR_ERR_INVALID_ARGUMENT;
    std::memset(u, 0, sizeof(*u));
    float aspect = (float)cfg->width / (float)cfg->height;
    float half_h = std::tan(0.5f * cam->fov_y_rad);
    float half_w = aspect * half_h;
    for (int k = 0; k < 4; ++k) {
        u->cam_pos[k] = cam->position[k];
        u->light_pos[k] = light_pos[k];
        for (int a = 0; a < 4; ++a) u->e[a][k] = cam->e[a][k];
    }
    u->half_wh[0] = half_w;
    u->half_wh[1] = half_h;
    u->size[0] = cfg->width;
    u->size[1] = cfg->height;
    u->mode = cfg->mode;
    u->shadow_mode = cfg->shadow_mode;
    u->slice_mode = cfg->slice_mode;
    u->num_nodes = num_nodes;
    u->num_stars = num_stars;
    u->prophecy_delta = cfg->prophecy_delta;
    // FrameDynamics::frontier_or_camera and frontier_view_offset (renderer.rs:235-271).
    bool has_frontier = dyn && dyn->has_frontier;
    for (int k = 0; k < 4; ++k) u->frontier_origin[k] = has_frontier ? dyn->frontier_origin[k] : cam->position[k];
    u->frontier_tau = has_frontier ? dyn->frontier_tau : cam->proper_time;
    u->frontier_view_offset = 0.14f + (dyn ? dyn->frontier_lag : 0.0f);
    // active_flashes: the first MAX_FLASHES, colour premultiplied by intensity (gpu.rs:160-167).
    uint32_t nf = dyn ? std::min<uint32_t>(dyn->n_flashes, SR_MAX_FLASHES) : 0;
    for (uint32_t i = 0; i < nf; ++i) {
        const SrFlash& f = dyn->flashes[i];
        for (int k = 0; k < 4; ++k) u->flash_at[i][k] = f.at[k];
        for (int k = 0; k < 3; ++k) u->flash_col_width[i][k] = f.color[k] * f.intensity;
        u->flash_col_width[i][3] = f.width;
    }
    u->num_flashes = nf;
    // haze_origins (renderer.rs:253-262).
    uint32_t nr = dyn ? std::min<uint32_t>(dyn->n_remote, SR_MAX_HAZE_ORIGINS - 1) : 0;
    uint32_t nh = 0;
    if (cfg->slice_mode == 3) {
        for (int k = 0; k < 4; ++k) u->haze_origin[nh][k] = u->frontier_origin[k];
        ++nh;
    }
    if (cfg->slice_mode == 1 || cfg->slice_mode == 3)
        for (uint32_t i = 0; i < nr; ++i, ++nh)
            for (int k = 0; k < 4; ++k) u->haze_origin[nh][k] = dyn->remote_origins[4 * i + k];
    u->num_haze = nh;
    return SR_OK;
}

extern "C" sr_status sr_flash_emit(SrFlash* flashes, uint32_t* n, const float at[4], int hit) {
    if (!flashes || !n || !at || *n > SR_MAX_FLASHES) return SR_ERR_INVALID_ARGUMENT;
    // push_flash (renderer.rs:293-298): evict the oldest when every slot is taken.
    if (*n >= SR_MAX_FLASHES) {
        std::memmove(flashes, flashes + 1, (SR_MAX_FLASHES - 1) * sizeof(SrFlash));
        *n = SR_MAX_FLASHES - 1;
    }
    SrFlash& f = flashes[(*n)++];
    for (int k = 0; k < 4; ++k) f.at[k] = at[k];
    if (hit) {  // emit_hit_flash (renderer.rs:283-291), HIT_FLASH_COLOR (renderer.rs:231)
        f.width = 0.5f;
        f.intensity = 3.0f;
        f.color[0] = 1.0f; f.color[1] = 0.35f; f.color[2] = 0.12f;
    } else {  // emit_flash (renderer.rs:274-281)
        f.width = 0.8f;
        f.intensity = 2.5f;
        f.color[0] = 1.0f; f.color[1] = 0.9f; f.color[2] = 0.7f;
    }
    return SR_OK;
}

extern "C" sr_status sr_flashes_retire(SrFlash* flashes, uint32_t* n, float now_t) {
    if (!n || (*n && !flashes)) return SR_ERR_INVALID_ARGUMENT;
    const float max_radius = 200.0f;  // FLASH_MAX_RADIUS (renderer.rs:228)
    uint32_t keep = 0;
    for (uint32_t i = 0; i < *n; ++i)
        if (now_t - flashes[i].at[0] < max_radius) flashes[keep++] = flashes[i];
    *n = keep;
    return SR_OK;
}

extern "C" sr_status sr_flashes_shift_time(SrFlash* flashes, uint32_t n, float dt) {
    if (n && !flashes) return SR_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < n; ++i) flashes[i].at[0] += dt;
    return SR_OK;
}

extern "C" sr_status sr_config_step_prophecy_delta(SrRenderConfig* cfg, float steps) {
    if (!cfg) return SR_ERR_INVALID_ARGUMENT;
    // PROPHECY_DELTA_MIN / MAX / STEP (renderer.rs:121-124); f32::clamp.
    float v = cfg->prophecy_delta + steps * 0.5f;
    cfg->prophecy_delta = v < 0.5f ? 0.5f : (v > 20.0f ? 20.0f : v);
    return SR_OK;
}

static const uint8_t GLYPHS[14][7] = {
    {0b01110, 0b10001, 0b10011, 0b10101, 0b11001, 0b10001, 0b01110},  // 0
    {0b00100, 0b01100, 0b00100, 0b00100, 0b00100, 0b00100, 0b01110},  // 1
    {0b01110, 0b10001, 0b00001, 0b00010, 0b00100, 0b01000, 0b11111},  // 2
    {0b11110, 0b00001, 0b00001, 0b01110, 0b00001, 0b00001, 0b11110},  // 3
    {0b00010, 0b00110, 0b01010, 0b10010, 0b11111, 0b00010, 0b00010},  // 4
    {0b11111, 0b10000, 0b11110, 0b00001, 0b00001, 0b10001, 0b01110},  // 5
    {0b01110, 0b10000, 0b10000, 0b11110, 0b10001, 0b10001, 0b01110},  // 6
    {0b11111, 0b00001, 0b00010, 0b00100, 0b01000, 0b01000, 0b01000},  // 7
    {0b01110, 0b10001, 0b10001, 0b01110, 0b10001, 0b10001, 0b01110},  // 8
    {0b01110, 0b10001, 0b10001, 0b01111, 0b00001, 0b00001, 0b01110},  // 9
    {0b00000, 0b00100, 0b00100, 0b11111, 0b00100, 0b00100, 0b00000},  // +
    {0b00000, 0b00000, 0b00000, 0b11111, 0b00000, 0b00000, 0b00000},  // -
    {0b00000, 0b00000, 0b00000, 0b00000, 0b00000, 0b01100, 0b01100},  // .
    {0b01111, 0b10000, 0b10000, 0b01110, 0b00001, 0b00001, 0b11110},  // S
};

extern "C" sr_status sr_tables_build(uint32_t* out) {
    if (!out) return SR_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < SR_GAMMA_LUT_SIZE; ++i) {
        float x = (float)i / (float)(SR_GAMMA_LUT_SIZE - 1);
        float v = std::pow(x, 1.0f / 2.2f) * 255.0f + 0.5f;
        v = v < 0.0f ? 0.0f : (v > 255.0f ? 255.0f : v);
        out[i] = (uint32_t)(uint8_t)v;
    }
    for (int g = 0; g < 14; ++g)
        for (int r = 0; r < 7; ++r) out[SR_GAMMA_LUT_SIZE + g * 7 + r] = GLYPHS[g][r];
    return SR_OK;
}
