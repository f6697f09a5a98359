// Host-side scene preparation: SAH kd-tree per mesh and the object tree.
// Internal header (not part of the C ABI).
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/yr.h"

namespace yr {

struct Box {
    float a[3];  // min corner (bound_t::a)
    float g[3];  // max corner (bound_t::g)
};

// One mesh's kd-tree in the device format (see yr_kd_node in yr.h).
struct KdTree {
    std::vector<yr_kd_node> nodes;
    std::vector<uint32_t> prims;
    Box bound;
    int max_depth = 0;
    int max_leaf_size = 0;
    float cost_ratio = 0.f;
    float empty_bonus = 0.f;
};

// Build parameters; the defaults are meshObject_t's (mesh.cc:162: depth -1,
// leaf size -1, cost ratio 1.2, empty bonus 0.40, with kdTree_t's
// large-scene cost penalty, kdtree.cc:68-80).
struct KdParams {
    int max_depth = -1;
    int max_leaf = -1;
    float cost_ratio = 1.2f;
    float empty_bonus = 0.40f;
    bool large_scene_penalty = true;
};

// Returns YR_OK or an error status.  With nthreads > 1 the subtrees below a
// few top levels are built concurrently; the result is identical to the
// sequential build.
yr_status build_kdtree(const float *verts, uint32_t nverts, const uint32_t *tris,
                       uint32_t ntris, KdTree &out, const KdParams &params = KdParams(),
                       int nthreads = 1);

// kdTree_t's constructor defaults for n triangles (kdtree.cc:57-80): the
// depth and leaf-size limits and the cost ratio with the large-scene penalty.
void kd_limits(uint32_t n, const KdParams &kp, int &max_depth, int &max_leaf, float &cost_ratio);
// The tree bound: the triangles' bound grown by 1e-4 of its diagonal on
// every side (kdtree.cc:83-89).
Box kd_grow_bound(const Box &b);

// The same trees as build_kdtree for several meshes at once, built on the
// GPU `device` (kd_gpu.cu).  With `abi_out` (one slot per mesh) the trees
// go to yr_kdtree records allocated there instead of `out`; on failure the
// slots filled so far are left for the caller to free.
struct KdMesh {
    const float *verts;
    uint32_t nverts;
    const uint32_t *tris;
    uint32_t ntris;
};
yr_status build_kdtrees_gpu(const std::vector<KdMesh> &meshes, const KdParams &params, int device,
                            std::vector<KdTree> &out, yr_kdtree **abi_out = nullptr);

// A KdTree as a yr_kdtree allocated for the caller (freed by yr_kdtree_free).
yr_status export_tree(const KdTree &t, yr_kdtree **out);

// meshObject_t::recalcBound (mesh.cc:343-379): bound of the triangles'
// vertices grown by BOX_MIN.
Box mesh_bound(const float *verts, const uint32_t *tris, uint32_t ntris);

// referenceObject_t's matrices (reference.cc:9-46): the first three rows of
// M and of its inverse (matrix4x4_t::inverse, matrix4.cc:68-117), and M's
// rows normalised (the rotation used for normals).  Returns false when M
// is singular (the reference stops there).
struct InstanceXf {
    float m[12];
    float back[12];
    float rot[9];
};
bool instance_xf(const float *M16, InstanceXf &out);
// referenceObject_t::getBound (reference.cc:135-165) in the shipped build's
// evaluation
Box instance_bound(const Box &b, const float *M16);

// meshObject_t::autoSmooth (mesh.cc:201-279) as the shipped build
// evaluates it: the shading normal of every triangle corner (9 floats per
// triangle: a, b, c) for a smoothing angle >= 1 degree.
void smooth_normals(const float *verts, const uint32_t *tris, uint32_t nverts, uint32_t ntris, float angle,
                    std::vector<float> &corner);

// Flattened object tree node (geomeTree_t, geometree.h:8-32).
struct ObjNode {
    float bmin[3];
    int32_t left;    // child index, -1 for a leaf
    float bmax[3];
    int32_t right;   // child index for interior, object index for a leaf
};

// buildObjectTree (object3d.cc:30-53): greedy agglomerative clustering with
// the bound_distance metric (bound.cc:75-83), in the order of obj_list.
// Node 0 is the root.
void build_object_tree(const std::vector<Box> &object_bounds, std::vector<ObjNode> &out);

// A binary BVH over the boxes of the objects listed in `ids` (surface-area
// heuristic, full sweep over centroids on each axis), in the same node
// format; leaves name entries of `ids`' values.  Node 0 is the root.  Not
// a reference structure: it serves queries whose answer does not depend
// on the order in which objects are visited.
void build_sah_object_bvh(const std::vector<Box> &object_bounds, const std::vector<int> &ids,
                          std::vector<ObjNode> &out);

}  // namespace yr
