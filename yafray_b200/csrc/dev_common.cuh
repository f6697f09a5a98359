// Device data layout and exact-rounding vector helpers.
//
// All single-precision arithmetic on the parity path is written operation
// by operation in the order the reference evaluates it (x86-64 SSE, no FMA
// contraction; the library is compiled with --fmad=false).  Where the
// shipped reference build (-O3 -ffast-math) evaluates an expression in a
// different but fixed form, that form is used and marked "fast-math".
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/yr.h"

namespace yr {

constexpr float kMinRayDist = 0.00005f;     // MIN_RAYDIST (configio.py:8-11)
constexpr uint32_t kNone = 0xffffffffu;
constexpr int kMaxObjStack = 32;            // object-tree depth cap (checked at scene creation)
constexpr uint32_t kMaxLeafVisits = 1u << 22;  // iteration cap per ray

// device status word bits (first error wins; read back after each launch)
enum DevError : int {
    kDevOk = 0,
    kDevIterationCap = YR_ERR_ITERATION_CAP,
    kDevStackOverflow = YR_ERR_STACK_OVERFLOW,
    kDevBadTree = YR_ERR_BAD_TREE,
};

struct V3 {
    float x, y, z;
};

__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ float comp(const V3 &v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__host__ __device__ __forceinline__ V3 operator+(const V3 &a, const V3 &b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ V3 operator-(const V3 &a, const V3 &b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ V3 operator-(const V3 &a) { return V3{-a.x, -a.y, -a.z}; }
// vector3d_t operator*(vector, PFLOAT f) returns (f*x, f*y, f*z) (vector3d.h:121-129)
__host__ __device__ __forceinline__ V3 operator*(const V3 &a, float f) { return V3{f * a.x, f * a.y, f * a.z}; }
__host__ __device__ __forceinline__ V3 operator*(float f, const V3 &a) { return V3{f * a.x, f * a.y, f * a.z}; }
// dot product, left to right (vector3d.h:116-119)
__host__ __device__ __forceinline__ float dot(const V3 &a, const V3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// cross product (vector3d.h:156-159)
__host__ __device__ __forceinline__ V3 cross(const V3 &a, const V3 &b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// vector3d_t::length: sqrt of the float sum (sqrtf after g++ narrows it)
__device__ __forceinline__ float length(const V3 &a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
// vector3d_t::normalize (vector3d.h:207-217): 1/sqrt taken in double
__device__ __forceinline__ V3 normalize(const V3 &a) {
    float l = a.x * a.x + a.y * a.y + a.z * a.z;
    if (l != 0.f) {
        float k = (float)(1.0 / sqrt((double)l));
        return V3{a.x * k, a.y * k, a.z * k};
    }
    return a;
}
// vector3d_t::normLenSqr (vector3d.h:60-68): normalizes, returns the squared length
__device__ __forceinline__ float norm_len_sqr(V3 &a) {
    float l = a.x * a.x + a.y * a.y + a.z * a.z;
    if (l != 0.f) {
        float k = (float)(1.0 / sqrt((double)l));
        a.x *= k;
        a.y *= k;
        a.z *= k;
    }
    return l;
}

struct C3 {
    float r, g, b;
};
__host__ __device__ __forceinline__ C3 c3(float r, float g, float b) { return C3{r, g, b}; }
__host__ __device__ __forceinline__ C3 operator+(const C3 &a, const C3 &b) { return C3{a.r + b.r, a.g + b.g, a.b + b.b}; }
__host__ __device__ __forceinline__ C3 operator-(const C3 &a, const C3 &b) { return C3{a.r - b.r, a.g - b.g, a.b - b.b}; }
__host__ __device__ __forceinline__ C3 operator*(const C3 &a, const C3 &b) { return C3{a.r * b.r, a.g * b.g, a.b * b.b}; }
// color_t * CFLOAT (color.h)
__host__ __device__ __forceinline__ C3 operator*(const C3 &a, float f) { return C3{a.r * f, a.g * f, a.b * f}; }
__host__ __device__ __forceinline__ C3 operator*(float f, const C3 &a) { return C3{f * a.r, f * a.g, f * a.b}; }
__host__ __device__ __forceinline__ C3 operator/(const C3 &a, float f) { return C3{a.r / f, a.g / f, a.b / f}; }
// color_t::energy (color.h:67)
__host__ __device__ __forceinline__ float energy(const C3 &c) { return (c.r + c.g + c.b) * 0.333333f; }

// ----------------------------------------------------------------- layout
// kd node: x = word (split bits / triangle / prim offset), y = flags.
// Indices are global: right child and triangle / prim offsets already
// include the owning object's base.
struct DevObject {
    float tb[6];        // kdTree_t::treeBound (min xyz, max xyz)
    uint32_t root;      // global index of the root kd node
    uint32_t tri_base;  // first global triangle index
    uint32_t ntris;
    uint32_t flags;     // bit0: casts shadows, bit1: smoothed (corner normals in DevScene::tri_nrm),
                        // bit2: texture coordinates (DevScene::tri_uv)
    float ob[6];        // object bound (meshObject_t::getBound), the object tree's leaf box
    int inst;           // instance record (DevScene::insts) or -1; the tree
                        // and triangle fields above are then the original's
    int orco;           // orco matrix (DevScene::orco_m, 3 rows) of the mesh, or -1
    int pad[2];
};

// referenceObject_t's matrices: rows 0-2 of M and of its inverse, and the
// row-normalised rotation part of M
struct DevInst {
    float m[12];
    float back[12];
    float rot[9];
    float pad[3];
};

// matrix4x4_t * point3d_t as the shipped build groups it:
// (m0*x + m1*y) + (m2*z + m3) per row
__host__ __device__ __forceinline__ V3 xf_point(const float *m, const V3 &p) {
    return v3((m[0] * p.x + m[1] * p.y) + (m[2] * p.z + m[3]), (m[4] * p.x + m[5] * p.y) + (m[6] * p.z + m[7]),
              (m[8] * p.x + m[9] * p.y) + (m[10] * p.z + m[11]));
}
// matrix4x4_t * vector3d_t (no translation), sums left to right
__host__ __device__ __forceinline__ V3 xf_vec(const float *m, const V3 &v) {
    return v3((m[0] * v.x + m[1] * v.y) + m[2] * v.z, (m[4] * v.x + m[5] * v.y) + m[6] * v.z,
              (m[8] * v.x + m[9] * v.y) + m[10] * v.z);
}
// a 3x3 row-major rotation times a vector
__host__ __device__ __forceinline__ V3 rot_vec(const float *r, const V3 &v) {
    return v3((r[0] * v.x + r[1] * v.y) + r[2] * v.z, (r[3] * v.x + r[4] * v.y) + r[5] * v.z,
              (r[6] * v.x + r[7] * v.y) + r[8] * v.z);
}


struct DevScene {
    const float4 *tris;         // 3 per triangle: {a, N.x}, {b, N.y}, {c, N.z}
    const uint2 *nodes;
    const uint32_t *prims;
    const DevObject *objects;
    const DevInst *insts;       // instance matrices (referenceObject_t)
    const float *tri_nrm;       // corner normals, 9 per triangle, of smoothed objects
    const float *tri_uv;        // texture coordinates, 6 per triangle, of objects that have them
    const float4 *orco_m;       // orco matrices (rows 0-2 of meshObject_t::backOrco), 3 per mesh with one
    // object tree (geomeTree_t): per interior node 4 x float4 = left box
    // (min xyz, max xyz), right box, then the children's codes (>= 0:
    // interior node, < 0: ~object index) as int bits
    const float4 *onodes;
    float otb[6];               // root box
    int oroot;                  // root code (-1 = ~0: a lone object 0; no tree when notree == 0)
    // SAH BVH over the shadow-casting objects (same record format), used by
    // shadow rays, whose answer does not depend on the visiting order
    const float4 *sonodes;
    float sotb[6];
    int soroot;
    uint32_t nsotree;
    uint32_t nobjects;
    uint32_t ntris;
    uint32_t nnodes;
    uint32_t nprims;
    uint32_t notree;
    // shadow-ray tree: one kd-tree over the triangles of every object that
    // casts shadows (global triangle indices), plus each triangle's object
    const uint2 *sh_nodes;
    const uint32_t *sh_prims;
    const uint32_t *tri_obj;
    uint32_t sh_nnodes;
    uint32_t sh_nprims;
    float sh_tb[6];
    int use_sh_tree;            // 1: shadow rays use the shadow-ray tree
    int exact_order;            // 1: exact slab tests in the object tree
    float coord_max;            // max |coordinate| of the object tree's root box
    int *status;                // device status word
};

__device__ __forceinline__ void dev_fail(int *status, int code) {
    if (status) atomicCAS(status, 0, code);
}

}  // namespace yr
