// Host-side validation of a packed scene before it reaches the device (sr_upload_scene runs it).
// The reference trusts its own builder; a C ABI cannot, so every index a kernel will follow is
// checked here: child links and leaf ranges in bounds, every node reached exactly once from the
// root (a tree, so traversal terminates), material ids and leaf_to_orig in range, star segment
// ranges inside the buffer (layouts of gpu.rs:44-119).
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/specrel.h"

static std::string check(const SrSceneDesc* d, uint32_t* depth_out) {
    if (d->num_nodes && !d->nodes) return "nodes is null";
    if (d->num_prims && (!d->geoms || !d->attrs)) return "geoms/attrs is null";
    if (d->num_materials == 0 || !d->materials) return "at least one material is required";
    if (d->num_stars && (!d->stars || d->num_star_vec4 < d->num_stars)) return "stars buffer too small";
    if (d->num_stars && (d->num_star_vec4 - d->num_stars) % 3 != 0) return "star segments are not whole (3 vec4 each)";
    std::vector<uint8_t> seen(d->num_nodes, 0);
    std::vector<std::pair<uint32_t, uint32_t>> st;
    uint32_t depth = 0;
    // A root over nothing (BvhNode4D::NOTHING, bvh4d.rs:31: an empty box linking to itself, what an
    // arena holds before anything is written to it) is an empty tree; the rest is free room.
    const bool nothing = d->num_nodes && SR_NODE_IS_NOTHING(&d->nodes[0]);
    if (d->num_nodes && !nothing) st.push_back({0u, 1u});
    if (nothing) depth = 1;
    while (!st.empty()) {
        auto [i, dd] = st.back();
        st.pop_back();
        if (i >= d->num_nodes) return "child link out of range at depth " + std::to_string(dd);
        if (seen[i]) return "node " + std::to_string(i) + " is reached twice (not a tree)";
        seen[i] = 1;
        if (dd > depth) depth = dd;
        const SrGpuNode& n = d->nodes[i];
        if (n.count > 0) {
            if ((uint64_t)n.right_or_first + n.count > d->num_prims)
                return "leaf range out of bounds at node " + std::to_string(i);
        } else {
            st.push_back({n.left, dd + 1});
            st.push_back({n.right_or_first, dd + 1});
        }
    }
    for (uint32_t i = 0; i < d->num_prims; ++i) {
        uint32_t m;
        std::memcpy(&m, &d->attrs[i].misc[2], 4);
        if (m >= d->num_materials) return "material id out of range at primitive " + std::to_string(i);
    }
    if (d->leaf_to_orig)
        for (uint32_t i = 0; i < d->num_prims; ++i)
            if (d->leaf_to_orig[i] >= d->num_prims) return "leaf_to_orig out of range at slot " + std::to_string(i);
    uint64_t nseg = d->num_stars ? (d->num_star_vec4 - d->num_stars) / 3 : 0;
    for (uint32_t i = 0; i < d->num_stars; ++i) {
        uint32_t first, count;
        std::memcpy(&first, &d->stars[4 * i + 2], 4);
        std::memcpy(&count, &d->stars[4 * i + 3], 4);
        if ((uint64_t)first + count > nseg) return "star segment range out of bounds at star " + std::to_string(i);
    }
    *depth_out = depth;
    return "";
}

extern "C" sr_status sr_scene_validate(const SrSceneDesc* desc, uint32_t* depth, char* err, size_t errlen) {
    if (!desc) return SR_ERR_INVALID_ARGUMENT;
    uint32_t dd = 0;
    std::string why = check(desc, &dd);
    if (depth) *depth = dd;
    if (why.empty()) return SR_OK;
    if (err && errlen) {
        std::strncpy(err, why.c_str(), errlen - 1);
        err[errlen - 1] = 0;
    }
    return SR_ERR_BAD_SCENE;
}
