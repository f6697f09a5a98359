// Host-only entry points of the C ABI (no CUDA calls).
#include <cstring>
#include <new>
#include <vector>

#include "host_build.h"

namespace yr {
yr_status export_tree(const KdTree &t, yr_kdtree **out) {
    yr_kdtree *r = new (std::nothrow) yr_kdtree;
    if (!r) return YR_ERR_OUT_OF_MEMORY;
    std::memset(r, 0, sizeof(*r));
    r->nnodes = (uint32_t)t.nodes.size();
    r->nprims = (uint32_t)t.prims.size();
    r->nodes = new (std::nothrow) yr_kd_node[r->nnodes ? r->nnodes : 1];
    r->prims = new (std::nothrow) uint32_t[r->nprims ? r->nprims : 1];
    if (!r->nodes || !r->prims) {
        yr_kdtree_free(r);
        return YR_ERR_OUT_OF_MEMORY;
    }
    if (r->nnodes) std::memcpy(r->nodes, t.nodes.data(), sizeof(yr_kd_node) * r->nnodes);
    if (r->nprims) std::memcpy(r->prims, t.prims.data(), 4 * (size_t)r->nprims);
    std::memcpy(r->bound, t.bound.a, 12);
    std::memcpy(r->bound + 3, t.bound.g, 12);
    r->max_depth = t.max_depth;
    r->max_leaf_size = t.max_leaf_size;
    r->cost_ratio = t.cost_ratio;
    r->empty_bonus = t.empty_bonus;
    *out = r;
    return YR_OK;
}
}  // namespace yr

extern "C" {

YR_API const char *yr_status_string(yr_status s) {
    switch (s) {
    case YR_OK: return "ok";
    case YR_ERR_INVALID_ARG: return "invalid argument";
    case YR_ERR_CUDA: return "CUDA runtime error";
    case YR_ERR_OUT_OF_MEMORY: return "out of memory";
    case YR_ERR_ITERATION_CAP: return "device loop hit its iteration cap";
    case YR_ERR_STACK_OVERFLOW: return "traversal stack overflow";
    case YR_ERR_BAD_TREE: return "corrupt tree (index out of range)";
    case YR_ERR_CANCELLED: return "cancelled";
    case YR_ERR_UNSUPPORTED: return "unsupported";
    case YR_ERR_EMPTY_SCENE: return "empty scene";
    case YR_ERR_NO_DEVICE: return "no CUDA device";
    case YR_ERR_TOO_LARGE: return "size above the documented maximum";
    }
    return "unknown status";
}

YR_API const char *yr_version(void) { return "yafray_b200 0.1 (YafRay 0.0.9 hot path, sm_100a)"; }


YR_API yr_status yr_kdtree_build(const float *verts, uint32_t nverts, const uint32_t *tris, uint32_t ntris,
                                 yr_kdtree **out) {
    return yr_kdtree_build_ex(verts, nverts, tris, ntris, nullptr, 1, out);
}

YR_API yr_status yr_kdtree_build_ex(const float *verts, uint32_t nverts, const uint32_t *tris, uint32_t ntris,
                                    const yr_kdtree_params *params, int nthreads, yr_kdtree **out) {
    if (!out) return YR_ERR_INVALID_ARG;
    *out = nullptr;
    yr::KdParams kp;
    if (params) {
        kp.max_depth = params->max_depth;
        kp.max_leaf = params->max_leaf_size;
        kp.cost_ratio = params->cost_ratio;
        kp.empty_bonus = params->empty_bonus;
        kp.large_scene_penalty = params->large_scene_penalty != 0;
    }
    yr::KdTree t;
    yr_status st;
    try {
        st = yr::build_kdtree(verts, nverts, tris, ntris, t, kp, nthreads < 1 ? 1 : nthreads);
    } catch (const std::bad_alloc &) {
        return YR_ERR_OUT_OF_MEMORY;
    }
    if (st != YR_OK) return st;
    return yr::export_tree(t, out);
}

YR_API yr_status yr_object_tree_build(const float *bounds, uint32_t n, yr_object_node *out, uint32_t *nout) {
    if (!bounds || !out || !nout || n == 0) return YR_ERR_INVALID_ARG;
    std::vector<yr::Box> b(n);
    for (uint32_t i = 0; i < n; i++) {
        std::memcpy(b[i].a, bounds + 6 * (size_t)i, 12);
        std::memcpy(b[i].g, bounds + 6 * (size_t)i + 3, 12);
    }
    std::vector<yr::ObjNode> t;
    try {
        yr::build_object_tree(b, t);
    } catch (const std::bad_alloc &) {
        return YR_ERR_OUT_OF_MEMORY;
    }
    static_assert(sizeof(yr::ObjNode) == sizeof(yr_object_node), "object node layout");
    std::memcpy(out, t.data(), sizeof(yr_object_node) * t.size());
    *nout = (uint32_t)t.size();
    return YR_OK;
}

YR_API void yr_kdtree_free(yr_kdtree *tree) {
    if (!tree) return;
    delete[] tree->nodes;
    delete[] tree->prims;
    delete tree;
}

}  // extern "C"
