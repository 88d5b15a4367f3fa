// TEST INFRASTRUCTURE ONLY — C ABI of the CPU oracle, loaded by the parity tests (ctypes) and by
// bench.py's CPU-baseline leg. Never linked into the shipped library.
#include <cstring>
#include <memory>

#include "oracle_arena.hpp"
#include "oracle_grad.hpp"
#include "oracle_demo.hpp"
#include "oracle_scenes.hpp"

using namespace orc;

extern "C" {

struct OrcSynthParams {
    uint32_t config;
    uint32_t n_bodies;
    uint32_t steps;
    uint32_t subdiv;
    uint32_t n_stars;
    uint32_t pad;
    uint64_t seed;
    double translate[4];
};

struct OrcSceneInfo {
    uint64_t n_prims, n_nodes, n_stars, n_star_vec4, n_materials;
    uint32_t depth;
    int32_t rindler_ok, superluminal;
    uint32_t clamped_accel;
    double cam_pos[4];
    double cam_rapidity[3];
    double bounds_min[4], bounds_max[4];
    uint32_t median_splits;  // nodes split at the centroid median (bvh4d.rs:418-424)
    uint32_t pad;
};

struct OrcCamera {
    double pos[4];
    double rapidity[3];
    double yaw, pitch, roll;
    double fov_deg;
    double proper_time;
    int32_t use_tetrad;
    int32_t pad;
    double tetrad[16];  // e0..e3, each (t, x, y, z); used when use_tetrad != 0
};

struct OrcConfig {
    uint32_t width, height, mode, shadow_mode, slice_mode;
    float prophecy_delta;
    uint32_t full_height, row_stride, row_offset;  // row sampling (0 = render the whole frame)
};

struct OrcFlash {
    double at[4];
    double width, intensity;
    double color[3];
};

struct OrcDynamics {
    int32_t has_frontier;
    uint32_t n_flashes;
    double frontier_origin[4];
    double frontier_tau;
    double frontier_lag;
    const OrcFlash* flashes;
    uint32_t n_remote;
    uint32_t pad;
    const double* remote_origins;  // n_remote x 4
};

struct OrcObserver {
    uint32_t width, height, slice_mode, pad;
    double pos[4];
    double rapidity[3];
};

struct OrcPixelOut {
    uint32_t* rgb;        // w*h packed 0x00RRGGBB (required)
    int64_t* slot;        // leaf slot of the primary hit or -1
    uint32_t* orig;       // original simplex index of the hit (0xFFFFFFFF for a miss)
    double* lambda;
    double* tau;
    double* min_bary;
    double* denom_rel;
    double* hdr;          // w*h*3 pre-bloom radiance
    uint64_t* stats;      // w*h*4: internal pops, leaf pops, tets tested, shadow rays
};
}

namespace {
struct SceneBox {
    bool fp64;
    std::unique_ptr<SynthOut<float>> f;
    std::unique_ptr<SynthOut<double>> d;
    double t_window[2] = {0.0, 0.0};  // a demo scene's valid lab-time window
};

// Bvh4D::trace of one ray (origin, direction, t_min, t_max: 10 doubles converted to T) and the
// interpolated hit: out = found, slot, original simplex index, lambda, proper time, event (4),
// tet barycentrics (4), uv (2), material.
template <class T> int trace_t(const SynthOut<T>& so, const double* r, double* out) {
    const auto& bvh = so.scene.bvh;
    V4<T> o((T)r[0], (T)r[1], (T)r[2], (T)r[3]), d((T)r[4], (T)r[5], (T)r[6], (T)r[7]);
    HitRecord<T> h{};
    int64_t slot = -1;
    bool found = bvh.trace(o, d, (T)r[8], (T)r[9], &h, &slot, nullptr);
    for (int k = 0; k < 18; ++k) out[k] = 0.0;
    out[0] = found ? 1.0 : 0.0;
    out[1] = (double)slot;
    out[2] = found ? (double)bvh.order[(size_t)slot] : -1.0;
    if (!found) return 0;
    out[3] = (double)h.lambda;
    out[4] = (double)h.proper_time;
    out[5] = (double)h.event.t; out[6] = (double)h.event.x; out[7] = (double)h.event.y; out[8] = (double)h.event.z;
    for (int k = 0; k < 4; ++k) out[9 + k] = (double)h.tet_bary[k];
    out[13] = (double)h.uv_u;
    out[14] = (double)h.uv_v;
    out[15] = (double)h.material_id;
    return 0;
}

template <class T> Tetrad<T> make_tetrad(const OrcCamera& c) {
    Tetrad<T> t = Tetrad<T>::rest();
    if (c.use_tetrad) {
        for (int a = 0; a < 4; ++a) t.e[a] = V4<T>((T)c.tetrad[4 * a], (T)c.tetrad[4 * a + 1], (T)c.tetrad[4 * a + 2], (T)c.tetrad[4 * a + 3]);
        return t;
    }
    t.boost_local(V3<T>((T)c.rapidity[0], (T)c.rapidity[1], (T)c.rapidity[2]));
    if (c.yaw != 0 || c.pitch != 0 || c.roll != 0) t.rotate_local((T)c.yaw, (T)c.pitch, (T)c.roll);
    return t;
}

template <class T>
int render_t(const Scene<T>& scene, const OrcCamera* c, const OrcConfig* cf, const OrcDynamics* dy, int threads,
             int perturb, const OrcPixelOut* out) {
    Camera4D<T> cam;
    cam.position = V4<T>((T)c->pos[0], (T)c->pos[1], (T)c->pos[2], (T)c->pos[3]);
    cam.tetrad = make_tetrad<T>(*c);
    cam.proper_time = (T)c->proper_time;
    // Camera4D::new: fov_deg.to_radians() (renderer.rs:57-64) in the scalar type.
    cam.fov_y_rad = (T)c->fov_deg * (C<T>::PI / T(180));
    RenderConfig cfg;
    cfg.width = cf->width;
    cfg.height = cf->height;
    cfg.mode = (RenderMode)cf->mode;
    cfg.shadow_mode = (ShadowMode)cf->shadow_mode;
    cfg.slice_mode = (ViewMode)cf->slice_mode;
    cfg.prophecy_delta = cf->prophecy_delta;
    if (cf->full_height) {
        cfg.full_height = cf->full_height;
        cfg.row_stride = cf->row_stride ? cf->row_stride : 1;
        cfg.row_offset = cf->row_offset;
    }
    FrameDynamics<T> dyn;
    if (dy) {
        dyn.has_frontier = dy->has_frontier != 0;
        dyn.frontier.origin = V4<T>((T)dy->frontier_origin[0], (T)dy->frontier_origin[1], (T)dy->frontier_origin[2], (T)dy->frontier_origin[3]);
        dyn.frontier.proper_time = (T)dy->frontier_tau;
        dyn.frontier_lag = (T)dy->frontier_lag;
        for (uint32_t i = 0; i < dy->n_flashes; ++i) {
            const OrcFlash& f = dy->flashes[i];
            dyn.flashes.push_back({V4<T>((T)f.at[0], (T)f.at[1], (T)f.at[2], (T)f.at[3]), (T)f.width, (T)f.intensity,
                                   V3<T>((T)f.color[0], (T)f.color[1], (T)f.color[2])});
        }
        for (uint32_t i = 0; i < dy->n_remote; ++i)
            dyn.remote_origins.push_back(V4<T>((T)dy->remote_origins[4 * i], (T)dy->remote_origins[4 * i + 1],
                                               (T)dy->remote_origins[4 * i + 2], (T)dy->remote_origins[4 * i + 3]));
    }
    perturb_ulps() = perturb;
    Renderer<T> r{scene, cam, cfg, dyn};
    bool want_aux = out->slot || out->orig || out->lambda || out->tau || out->min_bary || out->denom_rel || out->stats;
    std::vector<PixelAux<T>> aux;
    std::vector<V3<T>> hdr;
    r.render(out->rgb, want_aux ? &aux : nullptr, out->hdr ? &hdr : nullptr, threads <= 0 ? 1u : (unsigned)threads);
    perturb_ulps() = 0;
    size_t n = (size_t)cfg.width * cfg.height;
    for (size_t i = 0; i < n && want_aux; ++i) {
        const auto& a = aux[i];
        if (out->slot) out->slot[i] = a.slot;
        if (out->orig) out->orig[i] = a.slot < 0 ? 0xFFFFFFFFu : scene.bvh.order[(size_t)a.slot];
        if (out->lambda) out->lambda[i] = (double)a.lambda;
        if (out->tau) out->tau[i] = (double)a.tau;
        if (out->min_bary) out->min_bary[i] = (double)a.min_bary;
        if (out->denom_rel) out->denom_rel[i] = (double)a.denom_rel;
        if (out->stats) {
            out->stats[4 * i] = a.stats.internal_pops;
            out->stats[4 * i + 1] = a.stats.leaf_pops;
            out->stats[4 * i + 2] = a.stats.tets_tested;
            out->stats[4 * i + 3] = a.shadow_rays;
        }
    }
    if (out->hdr)
        for (size_t i = 0; i < n; ++i) {
            out->hdr[3 * i] = (double)hdr[i].x;
            out->hdr[3 * i + 1] = (double)hdr[i].y;
            out->hdr[3 * i + 2] = (double)hdr[i].z;
        }
    return 0;
}

template <class T> void info_t(const SynthOut<T>& s, OrcSceneInfo* o) {
    o->n_prims = s.scene.bvh.hot.size();
    o->n_nodes = s.scene.bvh.nodes.size();
    o->n_stars = s.scene.stars.size();
    size_t segs = 0;
    for (auto& st : s.scene.stars) segs += st.segments.size();
    o->n_star_vec4 = s.scene.stars.size() + 3 * segs;
    o->n_materials = s.scene.materials.size();
    o->depth = s.scene.bvh.depth();
    o->median_splits = s.scene.bvh.median_splits;
    o->rindler_ok = s.rindler_ok;
    o->superluminal = s.superluminal;
    o->clamped_accel = s.clamped_accel;
    for (int k = 0; k < 4; ++k) o->cam_pos[k] = s.cam_pos[k];
    for (int k = 0; k < 3; ++k) o->cam_rapidity[k] = s.cam_rapidity[k];
    if (!s.scene.bvh.nodes.empty()) {
        const auto& b = s.scene.bvh.nodes[0].aabb;
        for (int k = 0; k < 4; ++k) { o->bounds_min[k] = (double)b.min.axis(k); o->bounds_max[k] = (double)b.max.axis(k); }
    }
}
}  // namespace

extern "C" {

void* orc_scene_new(const OrcSynthParams* p, int fp64) {
    SynthParams sp;
    sp.config = p->config;
    sp.seed = p->seed;
    sp.n_bodies = p->n_bodies;
    sp.steps = p->steps;
    sp.subdiv = p->subdiv;
    sp.n_stars = p->n_stars;
    for (int k = 0; k < 4; ++k) sp.translate[k] = p->translate[k];
    auto* b = new SceneBox();
    b->fp64 = fp64 != 0;
    if (b->fp64) b->d = std::make_unique<SynthOut<double>>(synth_scene<double>(sp));
    else b->f = std::make_unique<SynthOut<float>>(synth_scene<float>(sp));
    return b;
}

void orc_scene_free(void* s) { delete (SceneBox*)s; }

// One of the reference's demo scenes (oracle_demo.hpp: 0 twin paradox, 1 barn and pole, 2
// Terrell-Penrose street, 3 Einstein's train, 4 carousel; 5 the Penrose test's own sphere, scene.rs:985-996); its initial camera event is the info's
// cam_pos, its lab-time window and light from orc_scene_demo_info.
void* orc_scene_demo(uint32_t which, int fp64) {
    if (which > 5) return nullptr;
    auto* b = new SceneBox();
    b->fp64 = fp64 != 0;
    if (b->fp64) {
        auto o = build_demo<double>(which);
        b->t_window[0] = o.t_min;
        b->t_window[1] = o.t_max;
        b->d = std::make_unique<SynthOut<double>>(std::move(o.s));
    } else {
        auto o = build_demo<float>(which);
        b->t_window[0] = o.t_min;
        b->t_window[1] = o.t_max;
        b->f = std::make_unique<SynthOut<float>>(std::move(o.s));
    }
    return b;
}

// A demo scene's lab-time window and light position: t_min, t_max, light x, y, z.
int orc_scene_demo_info(void* s, double* out5) {
    auto* b = (SceneBox*)s;
    out5[0] = b->t_window[0];
    out5[1] = b->t_window[1];
    if (b->fp64) {
        const auto& l = b->d->scene.light_pos;
        out5[2] = l.x; out5[3] = l.y; out5[4] = l.z;
    } else {
        const auto& l = b->f->scene.light_pos;
        out5[2] = l.x; out5[3] = l.y; out5[4] = l.z;
    }
    return 0;
}

// Rays through the scene's BVH (trace_t above): rays are 10 doubles each, out 18 doubles each.
int orc_trace(void* s, const double* rays, uint32_t n, double* out) {
    auto* b = (SceneBox*)s;
    for (uint32_t i = 0; i < n; ++i) {
        if (b->fp64) trace_t(*b->d, rays + 10 * (size_t)i, out + 18 * (size_t)i);
        else trace_t(*b->f, rays + 10 * (size_t)i, out + 18 * (size_t)i);
    }
    return 0;
}

// Tetrad::from_beta (minkowski.rs:437-441) in f32: e[a][k] into out16[4 * a + k].
int orc_tetrad_from_beta(const double* beta3, double* out16) {
    Tetrad<float> t = Tetrad<float>::from_beta(V3<float>((float)beta3[0], (float)beta3[1], (float)beta3[2]));
    for (int a = 0; a < 4; ++a) {
        out16[4 * a] = t.e[a].t;
        out16[4 * a + 1] = t.e[a].x;
        out16[4 * a + 2] = t.e[a].y;
        out16[4 * a + 3] = t.e[a].z;
    }
    return 0;
}

// Bvh4D::build over boxes (8 floats each: min then max, (t, x, y, z); centroids their centres),
// as the tree of simplices with those boxes: the node array (2n - 1 GpuNode slots), the leaf order
// and the number of median splits.
int orc_bvh_from_boxes(const float* boxes, uint32_t n, void* nodes_out, uint32_t* order, uint32_t* n_nodes,
                       uint32_t* median) {
    using B = Bvh<float>;
    std::vector<B::Ref> refs(n);
    for (uint32_t i = 0; i < n; ++i) {
        Aabb<float> a;
        a.min = V4<float>(boxes[8 * i], boxes[8 * i + 1], boxes[8 * i + 2], boxes[8 * i + 3]);
        a.max = V4<float>(boxes[8 * i + 4], boxes[8 * i + 5], boxes[8 * i + 6], boxes[8 * i + 7]);
        refs[i] = {a, a.center(), i};
    }
    std::vector<BvhNode<float>> nodes;
    std::atomic<uint32_t> med{0};
    if (n) B::build_recursive(nodes, refs.data(), n, 0, 6, &med);
    auto* pn = (PNode*)nodes_out;
    for (size_t i = 0; i < nodes.size(); ++i) {
        v4f(pn[i].min, nodes[i].aabb.min);
        v4f(pn[i].max, nodes[i].aabb.max);
        pn[i].right_or_first = nodes[i].right_or_first;
        pn[i].count = nodes[i].count;
        pn[i].left = nodes[i].left;
        pn[i].pad = 0;
    }
    for (uint32_t i = 0; i < n; ++i) order[i] = refs[i].index;
    *n_nodes = (uint32_t)nodes.size();
    *median = med.load();
    return 0;
}

// select_nth_unstable_by on floats (by value, `partial_cmp` order) carrying their indices: the
// oracle's restatement of Rust's selection, for the tests.
int orc_select_nth(float* keys, uint32_t* idx, uint32_t n, uint32_t k) {
    struct KI { float key; uint32_t i; };
    std::vector<KI> v(n);
    for (uint32_t j = 0; j < n; ++j) v[j] = {keys[j], idx[j]};
    select_nth_unstable(v.data(), n, k, [](const KI& a, const KI& b) { return a.key < b.key; });
    for (uint32_t j = 0; j < n; ++j) { keys[j] = v[j].key; idx[j] = v[j].i; }
    return 0;
}

// light_clock_bounce_fraction (renderer.rs:988-996) in f32.
float orc_light_clock_bounce_fraction(float proper_time, float cavity_length) {
    return light_clock_bounce_fraction<float>(proper_time, cavity_length);
}

// Material `i` of the demo scenes' table: base rgb, emission, checker rgb, grid scale, wire width,
// pattern, cavity length.
int orc_material(uint32_t i, double* out9) {
    auto m = common_materials<float>();
    if (i >= m.size()) return -1;
    const auto& x = m[i];
    double v[9] = {x.base_color.x, x.base_color.y, x.base_color.z, x.emission, x.checker_color.x, x.checker_color.y,
                   x.checker_color.z, x.grid_scale, x.cavity_length};
    for (int k = 0; k < 9; ++k) out9[k] = v[k];
    return (int)x.pattern;
}

// A float scene from the reference's packed arrays (gpu.rs:44-119 layouts): the BVH nodes and hot
// records as given, the cold attributes as leaf-ordered simplices (order = identity). Lets the
// oracle render exactly the input a caller uploads, without rebuilding it.
void* orc_scene_from_packed(const void* nodes_, uint32_t n_nodes, const void* geoms_, const void* attrs_,
                            uint32_t n_prims, const void* mats_, uint32_t n_mats, const float* stars, uint64_t n_star_vec4,
                            uint32_t n_stars, const float* light_pos) {
    const PNode* nodes = (const PNode*)nodes_;
    const PGeom* geoms = (const PGeom*)geoms_;
    const PAttr* attrs = (const PAttr*)attrs_;
    const PMat* mats = (const PMat*)mats_;
    auto* b = new SceneBox();
    b->fp64 = false;
    b->f = std::make_unique<SynthOut<float>>();
    Scene<float>& sc = b->f->scene;
    auto v4 = [](const float* p) { return V4<float>(p[0], p[1], p[2], p[3]); };
    sc.bvh.nodes.resize(n_nodes);
    for (uint32_t i = 0; i < n_nodes; ++i) {
        auto& n = sc.bvh.nodes[i];
        n.aabb.min = v4(nodes[i].min);
        n.aabb.max = v4(nodes[i].max);
        n.right_or_first = nodes[i].right_or_first;
        n.count = nodes[i].count;
        n.left = nodes[i].left;
    }
    sc.bvh.hot.resize(n_prims);
    sc.bvh.order.resize(n_prims);
    sc.bvh.simplices.resize(n_prims);
    for (uint32_t i = 0; i < n_prims; ++i) {
        Geom<float>& g = sc.bvh.hot[i];
        g.v0 = v4(geoms[i].v0); g.n = v4(geoms[i].n); g.b1 = v4(geoms[i].b1); g.b2 = v4(geoms[i].b2); g.b3 = v4(geoms[i].b3);
        sc.bvh.order[i] = i;
        Simplex<float>& s = sc.bvh.simplices[i];
        s.g = g;
        const PAttr& a = attrs[i];
        for (int k = 0; k < 4; ++k) {
            s.uv_u[k] = a.uv_u[k]; s.uv_v[k] = a.uv_v[k];
            s.tri_bary[k] = V3<float>(a.tb_x[k], a.tb_y[k], a.tb_z[k]);
            s.tau[k] = a.tau[k]; s.grad_u[k] = a.grad_u[k]; s.grad_v[k] = a.grad_v[k];
            s.decided_at[k] = a.decided_at[k];
        }
        s.normal = v4(a.normal);
        s.four_vel = v4(a.four_vel);
        s.uvs_u = a.misc[0];
        s.uvs_v = a.misc[1];
        std::memcpy(&s.material_id, &a.misc[2], 4);
    }
    for (uint32_t i = 0; i < n_mats; ++i) {
        Material<float> m;
        m.base_color = V3<float>(mats[i].base[0], mats[i].base[1], mats[i].base[2]);
        m.emission = mats[i].base[3];
        m.checker_color = V3<float>(mats[i].checker[0], mats[i].checker[1], mats[i].checker[2]);
        m.grid_scale = mats[i].checker[3];
        m.wireframe_width = mats[i].params[0];
        uint32_t pat;
        std::memcpy(&pat, &mats[i].params[1], 4);
        m.pattern = (Pattern)pat;
        m.cavity_length = mats[i].params[2];
        sc.materials.push_back(m);
    }
    sc.light_pos = V3<float>(light_pos[1], light_pos[2], light_pos[3]);
    const float* segs = stars + 4ull * n_stars;
    for (uint32_t i = 0; i < n_stars; ++i) {
        PointStar<float> st;
        st.temperature = stars[4 * i];
        uint32_t first, count;
        std::memcpy(&first, &stars[4 * i + 2], 4);
        std::memcpy(&count, &stars[4 * i + 3], 4);
        for (uint32_t k = first; k < first + count && 12ull * (k + 1) <= 4 * (n_star_vec4 - n_stars); ++k) {
            const float* p = segs + 12ull * k;
            st.segments.push_back({v4(p), v4(p + 4), p[8], p[9]});
        }
        sc.stars.push_back(st);
        sc.star_cn.push_back(stars[4 * i + 1]);
    }
    return b;
}

int orc_scene_info(void* s, OrcSceneInfo* o) {
    auto* b = (SceneBox*)s;
    std::memset(o, 0, sizeof(*o));
    if (b->fp64) info_t(*b->d, o);
    else info_t(*b->f, o);
    return 0;
}

int orc_scene_pack(void* s, void* nodes, void* geoms, void* attrs, void* mats, float* stars, uint32_t* order) {
    auto* b = (SceneBox*)s;
    if (b->fp64) return -1;
    pack_scene(b->f->scene, (PNode*)nodes, (PGeom*)geoms, (PAttr*)attrs, (PMat*)mats, stars, order);
    return 0;
}

int orc_render(void* s, const OrcCamera* c, const OrcConfig* cf, const OrcDynamics* dy, int threads, int perturb,
               const OrcPixelOut* out) {
    auto* b = (SceneBox*)s;
    if (!out || !out->rgb || cf->width == 0 || cf->height == 0) return -1;
    if (b->fp64) return render_t(b->d->scene, c, cf, dy, threads, perturb, out);
    return render_t(b->f->scene, c, cf, dy, threads, perturb, out);
}

int orc_observers(uint64_t seed, uint32_t n, OrcObserver* out) {
    auto obs = synth_observers(seed, n);
    for (uint32_t i = 0; i < n; ++i) {
        out[i].width = obs[i].width;
        out[i].height = obs[i].height;
        out[i].slice_mode = obs[i].slice_mode;
        out[i].pad = 0;
        for (int k = 0; k < 4; ++k) out[i].pos[k] = obs[i].pos[k];
        for (int k = 0; k < 3; ++k) out[i].rapidity[k] = obs[i].rapidity[k];
    }
    return 0;
}

// The camera tetrad the oracle renders with (rows e0..e3), in float or double.
int orc_tetrad(const OrcCamera* c, int fp64, double* out16) {
    if (fp64) {
        auto t = make_tetrad<double>(*c);
        for (int a = 0; a < 4; ++a) for (int k = 0; k < 4; ++k) out16[4 * a + k] = t.e[a].axis(k);
    } else {
        auto t = make_tetrad<float>(*c);
        for (int a = 0; a < 4; ++a) for (int k = 0; k < 4; ++k) out16[4 * a + k] = (double)t.e[a].axis(k);
    }
    return 0;
}

// The reference's gamma LUT (renderer.rs:1102-1114).
int orc_gamma_lut(uint8_t* out4096) {
    const auto& l = gamma_lut();
    std::memcpy(out4096, l.data(), l.size());
    return 0;
}

// Bloom + pack of a float HDR image (bloom.rs:93-125 then renderer.rs:1116-1129).
int orc_bloom_pack(const float* hdr3, uint32_t w, uint32_t h, uint32_t* rgb, float* bloomed3) {
    std::vector<V3<float>> img((size_t)w * h);
    for (size_t i = 0; i < img.size(); ++i) img[i] = V3<float>(hdr3[3 * i], hdr3[3 * i + 1], hdr3[3 * i + 2]);
    bloom_apply(img, w, h);
    for (size_t i = 0; i < img.size(); ++i) {
        if (rgb) rgb[i] = pack_rgb(img[i]);
        if (bloomed3) { bloomed3[3 * i] = img[i].x; bloomed3[3 * i + 1] = img[i].y; bloomed3[3 * i + 2] = img[i].z; }
    }
    return 0;
}

}  // extern "C"

// ---- The frozen-outcome image loss (oracle_grad.hpp), FP64 reference of the engine's gradient ----
namespace {
template <class T> Camera4D<T> camera_of(const OrcCamera* c) {
    Camera4D<T> cam;
    cam.position = V4<T>((T)c->pos[0], (T)c->pos[1], (T)c->pos[2], (T)c->pos[3]);
    cam.tetrad = make_tetrad<T>(*c);
    cam.proper_time = (T)c->proper_time;
    cam.fov_y_rad = (T)c->fov_deg * (C<T>::PI / T(180));
    return cam;
}
RenderConfig config_of(const OrcConfig* cf) {
    RenderConfig cfg;
    cfg.width = cf->width;
    cfg.height = cf->height;
    cfg.mode = (RenderMode)cf->mode;
    cfg.shadow_mode = (ShadowMode)cf->shadow_mode;
    cfg.slice_mode = (ViewMode)cf->slice_mode;
    cfg.prophecy_delta = cf->prophecy_delta;
    return cfg;
}
struct FrozenBox {
    bool fp64;
    FrozenFrame<float> f;
    FrozenFrame<double> d;
};
template <class T>
double frozen_loss_t(const Scene<T>& scene, const FrozenFrame<T>& F, const OrcCamera* c, const OrcConfig* cf,
                     const double* target, uint32_t level, unsigned threads, double* hdr_out) {
    Camera4D<T> cam = camera_of<T>(c);
    RenderConfig cfg = config_of(cf);
    FrameDynamics<T> dyn;
    Renderer<T> R{scene, cam, cfg, dyn};
    std::vector<V3<T>> img = frozen_hdr(R, F, threads);
    std::vector<V3<T>> tgt(img.size());
    for (size_t i = 0; i < img.size(); ++i) tgt[i] = V3<T>((T)target[3 * i], (T)target[3 * i + 1], (T)target[3 * i + 2]);
    if (hdr_out)
        for (size_t i = 0; i < img.size(); ++i) {
            hdr_out[3 * i] = (double)img[i].x;
            hdr_out[3 * i + 1] = (double)img[i].y;
            hdr_out[3 * i + 2] = (double)img[i].z;
        }
    return pyramid_loss(img, tgt, F.w, F.h, level);
}
}  // namespace

extern "C" {

// Records the discrete outcomes of the frame (shaded, past light cone, no flashes or haze).
// `binning`: candidate stars per pixel found by projecting each star (-1: on large star sets,
// 0: never, 1: always); the outcomes are the same either way.
void* orc_frozen_new(void* s, const OrcCamera* c, const OrcConfig* cf, int threads, int binning) {
    auto* b = (SceneBox*)s;
    if (!cf || cf->mode != 0 || cf->slice_mode != 0 || cf->width == 0 || cf->height == 0) return nullptr;
    auto* fb = new FrozenBox();
    fb->fp64 = b->fp64;
    RenderConfig cfg = config_of(cf);
    unsigned th = threads <= 0 ? 1u : (unsigned)threads;
    if (b->fp64) {
        Camera4D<double> cam = camera_of<double>(c);
        FrameDynamics<double> dyn;
        Renderer<double> R{b->d->scene, cam, cfg, dyn};
        fb->d = freeze(R, th, binning);
    } else {
        Camera4D<float> cam = camera_of<float>(c);
        FrameDynamics<float> dyn;
        Renderer<float> R{b->f->scene, cam, cfg, dyn};
        fb->f = freeze(R, th, binning);
    }
    return fb;
}

void orc_frozen_free(void* f) { delete (FrozenBox*)f; }

// sum((P(HDR) - P(target))^2) at camera `c` under the recorded outcomes; P: `level` 2x2-box
// halvings; target: width*height*3 doubles; hdr_out (optional): the HDR image, width*height*3.
double orc_frozen_loss(void* s, void* f, const OrcCamera* c, const OrcConfig* cf, const double* target, uint32_t level,
                       int threads, double* hdr_out) {
    auto* b = (SceneBox*)s;
    auto* fb = (FrozenBox*)f;
    unsigned th = threads <= 0 ? 1u : (unsigned)threads;
    if (b->fp64) return frozen_loss_t(b->d->scene, fb->d, c, cf, target, level, th, hdr_out);
    return frozen_loss_t(b->f->scene, fb->f, c, cf, target, level, th, hdr_out);
}

}  // extern "C"

// ---- The scene cache over an arena (oracle_arena.hpp) -------------------------------------------
namespace {
struct ArenaBox {
    SceneCacheOracle<float> cache;
    ArenaBvh<float> arena;
};
struct OTri { uint32_t idx[3]; float uv[3][2]; float normal[3]; };  // SrTubeTriangle
struct OSample {                                                      // SrTubeSample
    float center[4];
    float tetrad[4][4];
    float proper_time;
    float phi[3];
    float accel[3];
    float pad;
};
static_assert(sizeof(OTri) == 48 && sizeof(OSample) == 112, "tube record layouts");

std::vector<Simplex<float>> simplices_from_packed(const float* boxes, const void* geoms, const void* attrs, uint32_t n) {
    std::vector<Simplex<float>> out(n);
    for (uint32_t i = 0; i < n; ++i)
        out[i] = simplex_from_packed(((const PGeom*)geoms)[i], ((const PAttr*)attrs)[i], boxes + 8ull * i);
    return out;
}
}  // namespace

extern "C" {

void* orc_arena_new() { return new ArenaBox(); }
void orc_arena_free(void* a) { delete (ArenaBox*)a; }

int orc_arena_begin(void* a_) {
    auto* a = (ArenaBox*)a_;
    a->cache.begin(a->arena);
    return 0;
}

int orc_arena_tube(void* a_, uint32_t kind, uint32_t player, uint64_t id, const float* verts, uint32_t nv,
                   const void* tris_, uint32_t nt, const void* samples_, uint32_t ns, const float* decided,
                   uint32_t material) {
    auto* a = (ArenaBox*)a_;
    const OTri* tris = (const OTri*)tris_;
    const OSample* smp = (const OSample*)samples_;
    Mesh3D<float> mesh;
    std::vector<uint32_t> bits{nv, nt};
    auto word = [&](const void* p) {
        uint32_t u;
        std::memcpy(&u, p, 4);
        bits.push_back(u);
    };
    for (uint32_t i = 0; i < nv; ++i) {
        mesh.vertices.push_back(V3<float>(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]));
        for (int k = 0; k < 3; ++k) word(&verts[3 * i + k]);
    }
    for (uint32_t i = 0; i < nt; ++i) {
        Triangle3D<float> t;
        for (int k = 0; k < 3; ++k) {
            if (tris[i].idx[k] >= nv) return -1;
            t.indices[k] = tris[i].idx[k];
            t.uv[k] = {tris[i].uv[k][0], tris[i].uv[k][1]};
        }
        t.normal = V3<float>(tris[i].normal[0], tris[i].normal[1], tris[i].normal[2]);
        mesh.triangles.push_back(t);
        for (size_t w = 0; w < sizeof(OTri) / 4; ++w) word((const char*)&tris[i] + 4 * w);
    }
    std::vector<WorldlineSample<float>> samples(ns);
    for (uint32_t i = 0; i < ns; ++i) {
        const OSample& q = smp[i];
        WorldlineSample<float>& w = samples[i];
        w.center = V4<float>(q.center[0], q.center[1], q.center[2], q.center[3]);
        w.proper_time = q.proper_time;
        w.phi = V3<float>(q.phi[0], q.phi[1], q.phi[2]);
        w.proper_accel_local = V3<float>(q.accel[0], q.accel[1], q.accel[2]);
        for (int k = 0; k < 4; ++k) w.tetrad.e[k] = V4<float>(q.tetrad[k][0], q.tetrad[k][1], q.tetrad[k][2], q.tetrad[k][3]);
    }
    a->cache.tube(CachePart{kind, player, id}, mesh, bits, samples, decided, material);
    return 0;
}

int orc_arena_piece(void* a_, uint32_t kind, uint32_t player, uint64_t id, int64_t index, const uint32_t* key,
                    uint32_t key_len, const float* boxes, const void* geoms, const void* attrs, uint32_t n) {
    auto* a = (ArenaBox*)a_;
    std::vector<uint32_t> k(key, key + key_len);
    a->cache.piece(CachePart{kind, player, id}, index, k, simplices_from_packed(boxes, geoms, attrs, n));
    return 0;
}

// A whole tube extruded at once (build_worldtube_simplices_with_decided, mesh4d.rs:648-660), as
// boxes and packed records; returns the count (the arrays need room for 3 per triangle and step).
int64_t orc_tube_simplices(const float* verts, uint32_t nv, const void* tris_, uint32_t nt, const void* samples_,
                           uint32_t ns, const float* decided, uint32_t material, float* boxes, void* geoms,
                           void* attrs) {
    const OTri* tris = (const OTri*)tris_;
    const OSample* smp = (const OSample*)samples_;
    Mesh3D<float> mesh;
    for (uint32_t i = 0; i < nv; ++i) mesh.vertices.push_back(V3<float>(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]));
    for (uint32_t i = 0; i < nt; ++i) {
        Triangle3D<float> t;
        for (int k = 0; k < 3; ++k) {
            if (tris[i].idx[k] >= nv) return -1;
            t.indices[k] = tris[i].idx[k];
            t.uv[k] = {tris[i].uv[k][0], tris[i].uv[k][1]};
        }
        t.normal = V3<float>(tris[i].normal[0], tris[i].normal[1], tris[i].normal[2]);
        mesh.triangles.push_back(t);
    }
    std::vector<WorldlineSample<float>> samples(ns);
    for (uint32_t i = 0; i < ns; ++i) {
        const OSample& q = smp[i];
        WorldlineSample<float>& w = samples[i];
        w.center = V4<float>(q.center[0], q.center[1], q.center[2], q.center[3]);
        w.proper_time = q.proper_time;
        w.phi = V3<float>(q.phi[0], q.phi[1], q.phi[2]);
        w.proper_accel_local = V3<float>(q.accel[0], q.accel[1], q.accel[2]);
        for (int k = 0; k < 4; ++k) w.tetrad.e[k] = V4<float>(q.tetrad[k][0], q.tetrad[k][1], q.tetrad[k][2], q.tetrad[k][3]);
    }
    std::vector<Simplex<float>> out;
    extend_worldtube_simplices(out, mesh, samples, decided, material);
    Bvh<float> b;  // no tree: the records in build order
    b.hot.resize(out.size());
    b.order.resize(out.size());
    for (size_t i = 0; i < out.size(); ++i) {
        b.hot[i] = out[i].g;
        b.order[i] = (uint32_t)i;
        const Aabb<float>& bx = out[i].aabb;
        float* o = boxes + 8 * i;
        o[0] = bx.min.t; o[1] = bx.min.x; o[2] = bx.min.y; o[3] = bx.min.z;
        o[4] = bx.max.t; o[5] = bx.max.x; o[6] = bx.max.y; o[7] = bx.max.z;
    }
    b.simplices = std::move(out);
    Scene<float> sc;
    sc.bvh = std::move(b);
    pack_scene(sc, (PNode*)nullptr, (PGeom*)geoms, (PAttr*)attrs, nullptr, nullptr, nullptr);
    return (int64_t)sc.bvh.hot.size();
}

// top_tree over n items (boxes n x 8: min then max, roots, weights): the n - 1 nodes in order.
int orc_top_tree(const float* boxes, const uint32_t* roots, const float* weights, uint32_t n, uint32_t base,
                 void* nodes_out) {
    if (n < 2) return -1;
    std::vector<TopItem<float>> items(n);
    for (uint32_t i = 0; i < n; ++i) {
        const float* b = boxes + 8 * i;
        items[i].box.min = V4<float>(b[0], b[1], b[2], b[3]);
        items[i].box.max = V4<float>(b[4], b[5], b[6], b[7]);
        items[i].root = roots[i];
        items[i].weight = weights[i];
    }
    std::vector<BvhNode<float>> tree;
    top_tree_rec(items, 0, n, base, tree);
    Scene<float> sc;
    sc.bvh.nodes = tree;
    pack_scene(sc, (PNode*)nodes_out, nullptr, nullptr, nullptr, nullptr, nullptr);
    return 0;
}

// stats6: chunks built, reused, simplices built, reused, arena simplices, compacted.
int orc_arena_finish(void* a_, const float* boxes, const void* geoms, const void* attrs, uint32_t n, uint64_t* stats6) {
    auto* a = (ArenaBox*)a_;
    a->cache.finish(Bvh<float>::build(simplices_from_packed(boxes, geoms, attrs, n)), a->arena);
    const CacheStats& s = a->cache.stats;
    if (stats6) {
        stats6[0] = s.chunks_built; stats6[1] = s.chunks_reused; stats6[2] = s.simplices_built;
        stats6[3] = s.simplices_reused; stats6[4] = s.arena_simplices; stats6[5] = s.compacted;
    }
    return 0;
}

// The arena's version and the ranges its latest edit wrote (Bvh4D::version / dirty): ranges as
// (start, end) pairs, up to `cap` of each; returns via the counts how many there are.
int orc_arena_dirty(void* a_, uint64_t* layout, uint64_t* edit, uint64_t* nodes, uint32_t* n_nodes, uint64_t* prims,
                    uint32_t* n_prims, uint32_t cap) {
    auto* a = (ArenaBox*)a_;
    *layout = a->arena.layout;
    *edit = a->arena.edit;
    *n_nodes = (uint32_t)a->arena.dirty_nodes.size();
    *n_prims = (uint32_t)a->arena.dirty_prims.size();
    for (uint32_t i = 0; i < *n_nodes && i < cap; ++i) {
        nodes[2 * i] = a->arena.dirty_nodes[i].lo;
        nodes[2 * i + 1] = a->arena.dirty_nodes[i].hi;
    }
    for (uint32_t i = 0; i < *n_prims && i < cap; ++i) {
        prims[2 * i] = a->arena.dirty_prims[i].lo;
        prims[2 * i + 1] = a->arena.dirty_prims[i].hi;
    }
    return 0;
}

int orc_arena_sizes(void* a_, uint32_t* n_nodes, uint32_t* n_prims) {
    auto* a = (ArenaBox*)a_;
    *n_nodes = (uint32_t)a->arena.b.nodes.size();
    *n_prims = (uint32_t)a->arena.b.hot.size();
    return 0;
}

int orc_arena_pack(void* a_, void* nodes, void* geoms, void* attrs) {
    auto* a = (ArenaBox*)a_;
    Scene<float> sc;
    sc.bvh = a->arena.b;
    pack_scene(sc, (PNode*)nodes, (PGeom*)geoms, (PAttr*)attrs, nullptr, nullptr, nullptr);
    return 0;
}

}  // extern "C"
