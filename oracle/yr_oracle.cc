// CPU ORACLE for the YafRay 0.0.9 ray-casting hot path - TEST INFRASTRUCTURE.
//
// A plain, single-threaded C++ restatement of the reference routines on the
// path, used only by tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg to check the CUDA library.  The product never links it.
// It is pinned against the unmodified reference (oracle/_ref/yr_ref_harness,
// built from the reference sources by oracle/Makefile) through the golden
// vectors in tests/golden/.
//
// Arithmetic follows the reference's shipped build (-O3 -ffast-math): where
// g++ evaluates an expression in a rewritten form that changes the rounding
// (the slab test, Halton::getNext), the rewritten form is used ("fast-math").
// Everything else is evaluated in source order, IEEE single precision, no
// FMA contraction (built with -ffp-contract=off).
//
// Inputs are a YRS1 scene file (include/yr.h layout) plus the flattened
// kd-trees and object tree (yr_kdtree layout), so the traversal can be run
// on the reference's own trees.
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <limits>
#include <vector>

#include "../include/yr.h"
#include "../yafray_b200/csrc/noise_tables.h"

namespace {

const float kMinRay = 0.00005f;  // MIN_RAYDIST (configio.py:8-11)
const float kInf = std::numeric_limits<float>::infinity();

struct V {
    float x, y, z;
    V() : x(0), y(0), z(0) {}
    V(float a, float b, float c) : x(a), y(b), z(c) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
V operator+(const V &a, const V &b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
V operator-(const V &a, const V &b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
V operator-(const V &a) { return V(-a.x, -a.y, -a.z); }
V operator*(const V &a, float f) { return V(f * a.x, f * a.y, f * a.z); }  // vector3d.h:121-129
V operator*(float f, const V &a) { return V(f * a.x, f * a.y, f * a.z); }
V operator/(const V &a, float f) { return V(a.x / f, a.y / f, a.z / f); }
float operator*(const V &a, const V &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }  // dot (vector3d.h:116)
V operator^(const V &a, const V &b) {                                                // cross (vector3d.h:156)
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
float length(const V &a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
V normalize(V a) {  // vector3d.h:207-217, 1/sqrt in double
    float l = a.x * a.x + a.y * a.y + a.z * a.z;
    if (l != 0) {
        float k = (float)(1.0 / sqrt((double)l));
        a.x *= k;
        a.y *= k;
        a.z *= k;
    }
    return a;
}
float normLenSqr(V &a) {  // vector3d.h:60-68
    float l = a.x * a.x + a.y * a.y + a.z * a.z;
    if (l != 0) {
        float k = (float)(1.0 / sqrt((double)l));
        a.x *= k;
        a.y *= k;
        a.z *= k;
    }
    return l;
}

struct C {
    float r, g, b;
    C() : r(0), g(0), b(0) {}
    C(float a, float b_, float c) : r(a), g(b_), b(c) {}
};
C operator+(const C &a, const C &b) { return C(a.r + b.r, a.g + b.g, a.b + b.b); }
C operator-(const C &a, const C &b) { return C(a.r - b.r, a.g - b.g, a.b - b.b); }
C operator*(const C &a, const C &b) { return C(a.r * b.r, a.g * b.g, a.b * b.b); }
C operator*(const C &a, float f) { return C(a.r * f, a.g * f, a.b * f); }
C operator*(float f, const C &a) { return C(f * a.r, f * a.g, f * a.b); }
C operator/(const C &a, float f) { return C(a.r / f, a.g / f, a.b / f); }
float energy(const C &c) { return (c.r + c.g + c.b) * 0.333333f; }  // color.h:67

// The estimators' energy cut-offs: a path stops when its colour's energy
// falls below 0.05 (pathlight.cc:315), a shading point whose diffuse
// colour's energy is below 0.05 gets no path light (pathlight.cc:398), and
// a hemi light skips a point whose fromLight(N, 1) has every channel below
// 0.05 (hemilight.cc:67).  A few ulps of difference in the value decide
// these branches when it lies at the threshold.  For the tests, a render
// can record, per pixel, the smallest relative distance of any such value
// from the threshold, and can take the other branch of every decision whose
// value lies within a relative band of it (orc_render_ex).
thread_local float t_flip_band = 0.f;   // 0: every decision as computed
thread_local float t_min_margin = 1e30f;
bool below_cut(float e) {
    const float m = fabsf(e - 0.05f) / 0.05f;
    if (m < t_min_margin) t_min_margin = m;
    const bool b = e < 0.05f;
    return (t_flip_band > 0.f && m <= t_flip_band) ? !b : b;
}

struct Box {
    float a[3], g[3];
};

struct Stats {
    uint64_t primary, shadow, bounce, nodes, tests, boxes, roots;
};
// Counters of the calling thread: several threads may trace or render
// disjoint pixel sets of one loaded scene at once (the scene is read-only
// while tracing); each entry point reports its own thread's counts.
thread_local Stats t_st;
thread_local Stats *g_stats = NULL;  // the counters the slab test adds to (NULL: not counting)

// bound_t::cross(from, ray, enter, leave, dist), shipped (fast-math) form (bound.cc:389-436)
bool cross_el(const Box &b, const V &from, const V &ray, float dist, float &enter, float &leave) {
    if (g_stats) g_stats->boxes++;
    float lmin = -1, lmax = -1;
    for (int k = 0; k < 3; k++) {
        if (ray[k] == 0) continue;
        float t1 = (b.a[k] - from[k]) / ray[k], t2 = (b.g[k] - from[k]) / ray[k];
        if (t1 > t2) {
            float s = t1;
            t1 = t2;
            t2 = s;
        }
        if (k == 0) {
            lmin = t1;
            lmax = t2;
        } else {
            if (t1 > lmin) lmin = t1;
            if ((t2 < lmax) || (lmax < 0)) lmax = t2;
        }
        if (k < 2 && ((lmax < 0) || (lmin > dist))) return false;
    }
    if ((lmin <= lmax) && (lmax >= 0) && (lmin <= dist)) {
        enter = lmin;
        leave = lmax;
        return true;
    }
    return false;
}
// cross(from, ray, where, dist) (bound.cc:340-387)
bool cross_w(const Box &b, const V &from, const V &ray, float dist, float &where) {
    float e, l;
    if (!cross_el(b, from, ray, dist, e, l)) return false;
    where = (e > 0) ? e : 0;
    return true;
}

struct Obj {
    std::vector<V> tri_a, tri_b, tri_c, tri_n;
    std::vector<V> tri_na, tri_nb, tri_nc;  // corner normals when smoothed
    bool smooth = false;
    std::vector<uint32_t> tri_shader;
    std::vector<float> tri_uv;  // 6 per triangle (u, v at a, b, c), or none
    std::vector<yr_kd_node> nodes;
    std::vector<uint32_t> prims;
    Box tb, ob;
    bool cast;
    // a reference (referenceObject_t): the original object, the first three
    // rows of M and of its inverse, and M's rows normalised (reference.cc:9-46)
    int inst = -1;
    float m[12], back[12], rot[9];
    // a mesh made through meshObject_t::transform: toObjectOrco(P) =
    // backOrco * P (mesh.cc:422-515), rows 0-2 of backOrco as given
    bool has_orco = false;
    float orco[12];
};

// matrix4x4_t * point3d_t as the shipped build groups it
V xf_point(const float *m, const V &p) {
    return V((m[0] * p.x + m[1] * p.y) + (m[2] * p.z + m[3]), (m[4] * p.x + m[5] * p.y) + (m[6] * p.z + m[7]),
             (m[8] * p.x + m[9] * p.y) + (m[10] * p.z + m[11]));
}
// matrix4x4_t * vector3d_t
V xf_vec(const float *m, const V &v) {
    return V((m[0] * v.x + m[1] * v.y) + m[2] * v.z, (m[4] * v.x + m[5] * v.y) + m[6] * v.z,
             (m[8] * v.x + m[9] * v.y) + m[10] * v.z);
}
V rot_vec(const float *r, const V &v) {
    return V((r[0] * v.x + r[1] * v.y) + r[2] * v.z, (r[3] * v.x + r[4] * v.y) + r[5] * v.z,
             (r[6] * v.x + r[7] * v.y) + r[8] * v.z);
}

// referenceObject_t ctor: back = M.inverse() (matrix4x4_t::inverse,
// matrix4.cc:68-117: Gauss-Jordan, pivot on the largest |m[k][i]|, rows
// divided by the pivot then reduced), MRot = M's rows normalised
bool make_instance(Obj &o, const float *M) {
    float a[4][4], id[4][4];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            a[i][j] = M[4 * i + j];
            id[i][j] = i == j ? 1.f : 0.f;
        }
    for (int i = 0; i < 4; i++) {
        float mx = 0;
        int ci = 0;
        for (int k = i; k < 4; k++)
            if (fabsf(a[k][i]) > mx) {
                mx = fabsf(a[k][i]);
                ci = k;
            }
        if (mx == 0) return false;
        for (int j = 0; j < 4; j++) {
            float t = a[i][j];
            a[i][j] = a[ci][j];
            a[ci][j] = t;
            t = id[i][j];
            id[i][j] = id[ci][j];
            id[ci][j] = t;
        }
        float f = a[i][i];
        for (int j = 0; j < 4; j++) a[i][j] /= f;
        for (int j = 0; j < 4; j++) id[i][j] /= f;
        for (int k = 0; k < 4; k++) {
            if (k == i) continue;
            f = a[k][i];
            for (int j = 0; j < 4; j++) a[k][j] -= a[i][j] * f;
            for (int j = 0; j < 4; j++) id[k][j] -= id[i][j] * f;
        }
    }
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 4; j++) {
            o.m[4 * i + j] = M[4 * i + j];
            o.back[4 * i + j] = id[i][j];
        }
        const V r = normalize(V(M[4 * i], M[4 * i + 1], M[4 * i + 2]));
        o.rot[3 * i] = r.x;
        o.rot[3 * i + 1] = r.y;
        o.rot[3 * i + 2] = r.z;
    }
    return true;
}

struct ONode {
    Box b;
    int left, right;  // left < 0: leaf, right = object
};

struct Light {
    yr_light_desc d;
    int samples;
    C color;
    V from, direction, corner, tox, toy;
    std::vector<V> pts, jit1, jit2;
    float sampdiv;
};

struct Cam {
    V pos, vright, vup, vto;
    int resx, resy;
};


struct Scene {
    std::vector<Obj> objs;
    std::vector<ONode> otree;
    std::vector<yr_shader_desc> shaders;
    std::vector<Light> lights;
    Cam cam;
    yr_render_params rp;
    // orc_illum only: Cranley-Patterson rotation off, and the area lights'
    // random values given from outside (2 per sample) instead of Halton
    bool no_rot = false;
    const float *area_vals = nullptr;
};

// ------------------------------------------------------------- triangles
// triangle_t::hit + intersect (triangle.h:48-86)
bool tri_hit(const Obj &o, uint32_t t, const V &from, const V &ray, float &rt) {
    const V va = o.tri_a[t] - from, vb = o.tri_b[t] - from, vc = o.tri_c[t] - from;
    const V &N = o.tri_n[t];
    V r = ((ray * N) < 0) ? -ray : ray;
    if (((va ^ vb) * r) < 0) return false;
    if (((vb ^ vc) * r) < 0) return false;
    if (((vc ^ va) * r) < 0) return false;
    rt = (N * va) / (N * ray);
    return true;
}

// ---------------------------------------------------------------- kd-tree
struct KdStackE {
    uint32_t node;
    float t;
    V pb;
    int prev;
};

// kdTree_t::Intersect (kdtree.cc:591-727) if !any, IntersectS (kdtree.cc:730-866) if any
bool kd_intersect(Scene &S, const Obj &o, const V &from, const V &ray, float dist, uint32_t &tr, float &Z, bool any) {
    float a, b, t;
    t_st.roots++;
    if (!cross_el(o.tb, from, ray, dist, a, b)) return false;
    const V invDir(1.f / ray.x, 1.f / ray.y, 1.f / ray.z);
    bool hit = false;
    KdStackE stack[64];
    const uint32_t kNull = 0xffffffffu;
    uint32_t curr = 0;
    int enPt = 0;
    stack[enPt].t = a;
    stack[enPt].pb = (a >= 0.0) ? from + ray * a : from;
    int exPt = 1;
    stack[exPt].t = b;
    stack[exPt].pb = from + ray * b;
    stack[exPt].node = kNull;
    stack[exPt].prev = 0;
    while (curr != kNull) {
        if (dist < stack[enPt].t) break;
        while ((o.nodes[curr].flags & 3u) != 3u) {
            t_st.nodes++;
            const int axis = (int)(o.nodes[curr].flags & 3u);
            float split;
            memcpy(&split, &o.nodes[curr].word, 4);
            const uint32_t right = o.nodes[curr].flags >> 2;
            uint32_t far;
            if (stack[enPt].pb[axis] <= split) {
                if (stack[exPt].pb[axis] <= split) {
                    curr++;
                    continue;
                }
                if (stack[exPt].pb[axis] == split) {
                    curr = right;
                    continue;
                }
                far = right;
                curr++;
            } else {
                if (split < stack[exPt].pb[axis]) {
                    curr = right;
                    continue;
                }
                far = curr + 1;
                curr = right;
            }
            t = (split - from[axis]) * invDir[axis];
            int tmp = exPt;
            exPt++;
            if (exPt == enPt) exPt++;
            if (exPt >= 64) {
                fprintf(stderr, "oracle: kd stack overflow\n");
                abort();
            }
            const int nextAxis = (axis + 1) % 3, prevAxis = (axis + 2) % 3;
            stack[exPt].prev = tmp;
            stack[exPt].t = t;
            stack[exPt].node = far;
            stack[exPt].pb[axis] = split;
            stack[exPt].pb[nextAxis] = from[nextAxis] + t * ray[nextAxis];
            stack[exPt].pb[prevAxis] = from[prevAxis] + t * ray[prevAxis];
        }
        t_st.nodes++;
        const uint32_t np = o.nodes[curr].flags >> 2;
        for (uint32_t k = 0; k < np; k++) {
            const uint32_t ti = (np == 1) ? o.nodes[curr].word : o.prims[o.nodes[curr].word + k];
            t_st.tests++;
            float rt;
            if (tri_hit(o, ti, from, ray, rt)) {
                if (any) {
                    if (rt < dist && rt > 0.f) {
                        tr = ti;
                        return true;
                    }
                } else if (rt < Z && rt >= 0.f) {
                    Z = rt;
                    tr = ti;
                    hit = true;
                }
            }
        }
        if (!any && hit && Z <= stack[exPt].t) return true;
        enPt = exPt;
        curr = stack[exPt].node;
        exPt = stack[enPt].prev;
    }
    return hit;
}

// ------------------------------------------------------ object iterator
// geomeIterator_t (geometree.h:36-157), front-to-back mode
struct OIter {
    const Scene &S;
    const V from, ray;
    std::vector<std::pair<int, float> > stack;
    int current;
    float maximun;
    OIter(const Scene &s, float m, const V &f, const V &r) : S(s), from(f), ray(r), current(-1), maximun(m) {
        if (S.otree.empty()) return;
        float where = 0;
        if (cross_w(S.otree[0].b, from, ray, maximun, where)) down(0);
    }
    void down(int node) {
        while (S.otree[node].left >= 0) {
            float hl = kInf, hr = kInf;
            const ONode &n = S.otree[node];
            bool hitl = cross_w(S.otree[n.left].b, from, ray, maximun, hl);
            bool hitr = cross_w(S.otree[n.right].b, from, ray, maximun, hr);
            if (!hitl && !hitr) {
                if (stack.empty()) {
                    current = -1;
                    return;
                }
                node = stack.back().first;
                stack.pop_back();
                continue;
            }
            if (hl < hr) {
                if (hitr) stack.push_back(std::make_pair(n.right, hr));
                node = n.left;
            } else {
                if (hitl) stack.push_back(std::make_pair(n.left, hl));
                node = n.right;
            }
        }
        current = S.otree[node].right;
    }
    void next() {
        current = -1;
        while (!stack.empty() && stack.back().second > maximun) stack.pop_back();
        if (!stack.empty()) {
            int n = stack.back().first;
            stack.pop_back();
            down(n);
        }
    }
    void limit(float z) {
        if (z < maximun) maximun = z;
    }
};

struct Hit {
    int obj;
    uint32_t tri;
    float Z;
};

// closest hit: raytrace (limit passed to shoot) or firstHit (scene.cc:200-258, 688-721)
// object3d_t::shoot: a mesh walks its own tree; a reference walks its
// original's with origin and direction taken there by M's inverse
// (referenceObject_t::shoot, reference.cc:95-114; not renormalised)
bool shoot(Scene &S, int oi, const V &from, const V &ray, float dist, uint32_t &tr, float &Z, bool any) {
    const Obj &o = S.objs[oi];
    if (o.inst < 0) return kd_intersect(S, o, from, ray, dist, tr, Z, any);
    return kd_intersect(S, S.objs[o.inst], xf_point(o.back, from), xf_vec(o.back, ray), dist, tr, Z, any);
}

Hit closest(Scene &S, const V &f, const V &ray, bool pass_limit, bool shadow_only) {
    Hit best = {-1, 0, 0};
    float limit = kInf;
    OIter it(S, kInf, f, ray);
    while (it.current >= 0) {
        const Obj &o = S.objs[it.current];
        if (!(shadow_only && !o.cast)) {
            float dis = pass_limit ? limit : kInf;
            float Z = dis;
            uint32_t tr = 0;
            if (shoot(S, it.current, f, ray, dis, tr, Z, false) && Z > 0) {
                if (pass_limit) limit = Z;
                it.limit(Z);
                if (best.obj < 0 || Z < best.Z) {
                    best.obj = it.current;
                    best.tri = tr;
                    best.Z = Z;
                }
            }
        }
        it.next();
    }
    return best;
}

// scene_t::isShadowed (scene.cc:107-185)
bool shadowed(Scene &S, const V &p, int own, const V &ray, float dist) {
    const V self = p + ray * S.rp.self_bias;
    const V p2 = p + ray * kMinRay;
    OIter it(S, dist, p2, ray);
    while (it.current >= 0) {
        const Obj &o = S.objs[it.current];
        if (o.cast) {
            float Z = dist;
            uint32_t tr;
            if (shoot(S, it.current, it.current == own ? self : p2, ray, dist, tr, Z, true)) return true;
        }
        it.next();
    }
    return false;
}

bool shadowed_point(Scene &S, const V &p, int own, const V &l) {
    t_st.shadow++;
    V ray = l - p;
    float dist = length(ray);
    ray = normalize(ray);
    return shadowed(S, p, own, ray, dist);
}

bool shadowed_dir(Scene &S, const V &p, int own, const V &dir) {
    t_st.shadow++;
    return shadowed(S, p, own, normalize(dir), kInf);
}

// ------------------------------------------------------------------- QMC
// Halton setStart(n) + getNext() (mcqmc.h:24-49), shipped (fast-math) form
float halton(unsigned base, unsigned n) {
    const double inv = 1.0 / double(base);
    double value = 0.0, factor = inv;
    unsigned i = n;
    while (i > 0) {
        value += double(i % base) * factor;
        i /= base;
        factor *= inv;
    }
    const double r = (1.0 - 0.0000000001) - value;
    if (inv < r) {
        value = value + inv;
    } else {
        double hh, h = inv;
        do {
            hh = h;
            h *= inv;
        } while (h >= r);
        value = (hh + h) + (value - 1.0);
    }
    return (float)value;
}

uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}
// per-pixel Cranley-Patterson rotation (the library's documented hash)
float cp_rot(uint32_t seed, uint32_t pixel, uint32_t dim) {
    uint32_t h = fmix32(seed * 0x9e3779b9u + 0x632be5abu);
    h = fmix32(h ^ (pixel * 0x85ebca77u));
    h = fmix32(h ^ (dim * 0xc2b2ae3du + 0x27d4eb2fu));
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}
float cp_add(float v, float r) {
    float u = v + r;
    if (u >= 1.0f) u -= 1.0f;
    return u;
}
float rot(const Scene &S, uint32_t pixel, uint32_t dim) { return S.no_rot ? 0.f : cp_rot(S.rp.seed, pixel, dim); }
const unsigned kPrimes[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
uint32_t light_dim(int k, int v) { return 64u + 16u * (uint32_t)k + 2u * (uint32_t)v; }

// RI_LP (mcqmc.h:73-78)
float ri_lp(unsigned i) {
    unsigned r = 0;
    for (unsigned v = 1u << 31; i; i >>= 1, v |= v >> 1)
        if (i & 1) r ^= v;
    return (float)(double(r) / 4294967296.0);
}

// ----------------------------------------------------------------- noise
// Blender permutation (noise.cc:118-127, first half)
const unsigned char kPerm[256] = {
    162, 160, 25,  59,  248, 235, 170, 238, 243, 28,  103, 40,  29,  237, 0,   222, 149, 46,  220, 63,  58,  130,
    53,  77,  108, 186, 54,  208, 246, 12,  121, 50,  209, 89,  244, 8,   139, 99,  137, 47,  184, 180, 151, 131,
    242, 143, 24,  199, 81,  20,  101, 135, 72,  32,  66,  168, 128, 181, 64,  19,  178, 34,  126, 87,  188, 127,
    107, 157, 134, 76,  200, 219, 124, 213, 37,  78,  90,  85,  116, 80,  205, 179, 122, 187, 195, 203, 182, 226,
    228, 236, 253, 152, 11,  150, 211, 158, 92,  161, 100, 241, 129, 97,  225, 196, 36,  114, 73,  140, 144, 75,
    132, 52,  56,  171, 120, 202, 31,  1,   215, 147, 17,  193, 88,  169, 49,  249, 68,  109, 191, 51,  156, 95,
    9,   148, 163, 133, 6,   198, 154, 30,  123, 70,  21,  48,  39,  43,  27,  113, 60,  91,  214, 111, 98,  172,
    79,  194, 192, 14,  177, 35,  167, 223, 71,  176, 119, 105, 5,   233, 230, 231, 118, 115, 15,  254, 110, 155,
    86,  239, 18,  165, 55,  252, 174, 217, 3,   142, 221, 16,  185, 206, 201, 141, 218, 42,  189, 104, 23,  159,
    190, 212, 10,  204, 210, 232, 67,  61,  112, 183, 2,   125, 153, 216, 13,  96,  138, 4,   44,  62,  146, 229,
    175, 83,  7,   224, 41,  166, 197, 227, 245, 247, 74,  65,  38,  106, 22,  94,  82,  45,  33,  173, 240, 145,
    255, 234, 84,  250, 102, 26,  69,  57,  207, 117, 164, 136, 251, 93};
int hsh(int i) { return kPerm[i & 255]; }
// the two signed terms of newPerlin_t::grad (noise.h:33-39)
void grad_parts(int hash, float x, float y, float z, float &U, float &Vv) {
    int h = hash & 15;
    float u = h < 8 ? x : y, v = h < 4 ? y : h == 12 || h == 14 ? x : z;
    U = (h & 1) == 0 ? u : -u;
    Vv = (h & 2) == 0 ? v : -v;
}
// newPerlin_t::operator() (noise.cc:161-183) as the shipped build
// (-O3 -ffast-math) evaluates it: g++ splits every grad() into its two
// signed terms (U = +-u, V = +-v of each cube corner) and regroups the
// three lerps into the sum below; this is its order of operations, read
// from the compiler's optimized tree of noise.cc, term for term.
float perlin(const V &pt) {
    const float px = pt.x, py = pt.y, pz = pt.z;
    const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
    const int X = ((int)fx) & 255, Y = ((int)fy) & 255, Z = ((int)fz) & 255;
    const float x = px - fx, y = py - fy, z = pz - fz;
    const float x1 = x - 1.f, y1 = y - 1.f, z1 = z - 1.f;
    const int A = hsh(X) + Y, AA = hsh(A) + Z, AB = hsh(A + 1) + Z, B = hsh(X + 1) + Y, BA = hsh(B) + Z,
              BB = hsh(B + 1) + Z;
    float U_aa, V_aa, U_ba, V_ba, U_ab, V_ab, U_bb, V_bb, U_aa1, V_aa1, U_ba1, V_ba1, U_ab1, V_ab1, U_bb1, V_bb1;
    grad_parts(hsh(AA), x, y, z, U_aa, V_aa);
    grad_parts(hsh(BA), x1, y, z, U_ba, V_ba);
    grad_parts(hsh(AB), x, y1, z, U_ab, V_ab);
    grad_parts(hsh(BB), x1, y1, z, U_bb, V_bb);
    grad_parts(hsh(AA + 1), x, y, z1, U_aa1, V_aa1);
    grad_parts(hsh(BA + 1), x1, y, z1, U_ba1, V_ba1);
    grad_parts(hsh(AB + 1), x, y1, z1, U_ab1, V_ab1);
    grad_parts(hsh(BB + 1), x1, y1, z1, U_bb1, V_bb1);
    const float t283 = x * x;
    const float t293 = y * y;
    const float t348 = x * 6.f;
    const float t349 = t348 - 15.f;
    const float t350 = x * t349;
    const float t351 = t350 + 10.f;
    const float t282 = x * t351;
    const float t352 = t282 * t283;
    const float t341 = y * 6.f;
    const float t342 = t341 - 15.f;
    const float t343 = y * t342;
    const float t344 = t343 + 10.f;
    const float t292 = y * t344;
    const float t345 = t292 * t293;
    const float t334 = z * 6.f;
    const float t335 = t334 - 15.f;
    const float t336 = z * t335;
    const float t337 = t336 + 10.f;
    const float t485 = U_aa + V_aa;
    const float t528 = U_ba - U_aa;
    const float t527 = V_ba + t528;
    const float t25 = t527 - V_aa;
    const float t26 = t25 * t352;
    const float t390 = U_ab + t528;
    const float t310 = U_bb + V_bb;
    const float t304 = V_aa - V_ab;
    const float t512 = U_aa - U_ba;
    const float t311 = t512 - U_ab;
    const float t303 = t310 + t311;
    const float t294 = t304 - V_ba;
    const float t504 = t294 + t303;
    const float t505 = t352 * t504;
    const float t321 = V_ab + t505;
    const float t322 = U_ab - U_aa;
    const float t312 = t321 + t322;
    const float t40 = t312 - V_aa;
    const float t41 = t40 * t345;
    const float t483 = t26 + t41;
    const float t477 = t483 + t485;
    const float t452 = U_ba1 + V_ba1;
    const float t458 = t512 - U_aa1;
    const float t440 = t452 + t458;
    const float t386 = U_bb1 + V_bb1;
    const float t381 = V_aa1 - V_ab1;
    const float t281 = U_ab1 + U_ba1;
    const float t383 = t386 - t281;
    const float t411 = U_ab1 - U_aa1;
    const float t410 = V_ab1 - V_aa1;
    const float t407 = V_aa + t410;
    const float t380 = V_ba - V_ba1;
    const float t346 = t380 + t381;
    const float t340 = V_ab - V_aa;
    const float t389 = U_aa1 - U_bb;
    const float t384 = t389 + t390;
    const float t347 = t383 + t384;
    const float t339 = t346 + t347;
    const float t323 = t340 - V_bb;
    const float t416 = t323 + t339;
    const float t414 = t352 * t416;
    const float t413 = U_aa - U_ab;
    const float t408 = t411 + t413;
    const float t404 = t407 + t408;
    const float t405 = t414 - V_ab;
    const float t425 = t404 + t405;
    const float t426 = t345 * t425;
    const float t466 = V_aa1 + t426;
    const float t442 = V_aa - V_aa1;
    const float t434 = t442 - V_ba;
    const float t427 = t434 + t440;
    const float t428 = t352 * t427;
    const float t468 = U_aa1 - U_aa;
    const float t464 = t466 + t468;
    const float t460 = t428 - V_aa;
    const float t83 = t460 + t464;
    const float tpowmult276 = z * z;
    const float tpowmult284 = z * tpowmult276;
    const float t489 = tpowmult284 * t337;
    const float t84 = t83 * t489;
    const float tnv123 = t84 + t477;
    return (float)(((double)tnv123 + 1.0) * 0.5);
}
// fBm_t::operator() (noise.cc:638-650)
float fbm(V tp, float H, float lac, float oct) {
    float value = 0, pwr = 1, pwHL = (float)pow((double)lac, (double)-H);
    for (int i = 0; i < (int)oct; i++) {
        value += ((float)2.0 * perlin(tp) - (float)1.0) * pwr;
        pwr *= pwHL;
        tp = V(tp.x * lac, tp.y * lac, tp.z * lac);
    }
    float rmd = oct - floorf(oct);
    if (rmd != 0.f) value += rmd * ((float)2.0 * perlin(tp) - (float)1.0) * pwr;
    return value;
}
// turbulence (noise.cc:808-819)
float turbulence(const V &pt, int oct, float size, bool hard) {
    float amp = 1, sum = 0;
    V tp(pt.x * size, pt.y * size, pt.z * size);
    for (int i = 0; i <= oct; i++, amp *= 0.5f, tp = V(tp.x * 2.0f, tp.y * 2.0f, tp.z * 2.0f)) {
        float val = perlin(tp);
        if (hard) val = (float)fabs(2.0 * (double)val - 1.0);
        sum += amp * val;
    }
    return sum * ((float)(1 << oct) / (float)((1 << (oct + 1)) - 1));
}

// ---------------------------------------------------------- noise bases
// Blender's feature-point and gradient tables (noise.cc:7-116, 129-187)
const float kHashPnt[768] = YR_HASHPNT_INIT;
const float kHashVect[768] = YR_HASHVECT_INIT;

// stdPerlin_t::operator() (noise.cc:374-434) in the shipped build's
// (-O3 -ffast-math) evaluation: t = x + 1e4 in float, each corner value
// u = (q0*rx + q1*ry) + q2*rz and each lerp toward v formed as
// ((v0 + v1) + (v2 - u)) * s + u; stdp_p / stdp_g repeat the permutation
// and hashvectf with period 256
float std_perlin(const V &pt) {
    const float vec[3] = {pt.x, pt.y, pt.z};
    int b0[3], b1[3];
    float r0[3], r1[3], sv[3];
    for (int k = 0; k < 3; k++) {
        const float t = vec[k] + 10000.0f;
        const int ti = (int)t;
        b0[k] = ti & 255;
        b1[k] = (b0[k] + 1) & 255;
        r0[k] = t - (float)ti;
        r1[k] = r0[k] - 1.0f;
        sv[k] = (float)((double)(r0[k] * r0[k]) * (3.0 - (double)r0[k] * 2.0));
    }
    const int i = hsh(b0[0]), j = hsh(b1[0]);
    const int b00 = hsh(i + b0[1]), b10 = hsh(j + b0[1]), b01 = hsh(i + b1[1]), b11 = hsh(j + b1[1]);
    auto at = [](int g, float rx, float ry, float rz) {
        const float *q = kHashVect + 3 * (g & 255);
        return (q[0] * rx + q[1] * ry) + q[2] * rz;
    };
    auto lerp_to = [](int g, float rx, float ry, float rz, float u, float s) {
        const float *q = kHashVect + 3 * (g & 255);
        return ((q[0] * rx + q[1] * ry) + (q[2] * rz - u)) * s + u;
    };
    const float sx = sv[0], sy = sv[1], sz = sv[2];
    float u = at(b00 + b0[2], r0[0], r0[1], r0[2]);
    const float a0 = lerp_to(b10 + b0[2], r1[0], r0[1], r0[2], u, sx);
    u = at(b01 + b0[2], r0[0], r1[1], r0[2]);
    const float bb0 = lerp_to(b11 + b0[2], r1[0], r1[1], r0[2], u, sx);
    const float c = (bb0 - a0) * sy + a0;
    u = at(b00 + b1[2], r0[0], r0[1], r1[2]);
    const float a1 = lerp_to(b10 + b1[2], r1[0], r0[1], r1[2], u, sx);
    u = at(b01 + b1[2], r0[0], r1[1], r1[2]);
    const float bb1 = lerp_to(b11 + b1[2], r1[0], r1[1], r1[2], u, sx);
    const float d = (bb1 - a1) * sy + a1;
    return (float)((double)((d - c) * sz + c) * 0.75 + 0.5);
}

// blenderNoise_t::operator() (noise.cc:439-510) in the shipped build's
// evaluation: the corner weights cn in double as x*x*(2x - 3) + 1 and
// 1 - x*x*(2x + 3), the four corners of each z layer summed as a vector
// reduction ((v0 + v2) + (v1 + v3)) and scaled once by that layer's z
// weight: n = cn6*R1 + (cn3*R0 + 0.5)
float blender_noise(const V &pt) {
    const float x = pt.x, y = pt.y, z = pt.z;
    const int ix = (int)floorf(x), iy = (int)floorf(y), iz = (int)floorf(z);
    const float ox = x - (float)ix, oy = y - (float)iy, oz = z - (float)iz;
    const float jx = ox - 1.0f, jy = oy - 1.0f, jz = oz - 1.0f;
    auto cn_o = [](float o) { return (float)((double)(o * o) * ((double)o * 2.0 - 3.0) + 1.0); };
    auto cn_j = [](float j) { return (float)(1.0 - (double)(j * j) * ((double)j * 2.0 + 3.0)); };
    const float cn1 = cn_o(ox), cn2 = cn_o(oy), cn3 = cn_o(oz), cn4 = cn_j(jx), cn5 = cn_j(jy), cn6 = cn_j(jz);
    const int b00 = hsh(hsh(ix & 255) + (iy & 255)), b10 = hsh(hsh((ix + 1) & 255) + (iy & 255)),
              b01 = hsh(hsh(ix & 255) + ((iy + 1) & 255)), b11 = hsh(hsh((ix + 1) & 255) + ((iy + 1) & 255));
    const int b20 = iz & 255, b21 = (iz + 1) & 255;
    auto g = [](int k, float a, float b, float c) {
        const float *h = kHashVect + 3 * hsh(k);
        return (h[0] * a + h[1] * b) + h[2] * c;
    };
    const float w0 = cn4 * cn5, w1 = cn2 * cn4, w2 = cn1 * cn5, w3 = cn1 * cn2;
    const float R0 = (w0 * g(b20 + b11, jx, jy, oz) + w2 * g(b20 + b01, ox, jy, oz)) +
                     (w1 * g(b20 + b10, jx, oy, oz) + w3 * g(b20 + b00, ox, oy, oz));
    const float R1 = (w0 * g(b21 + b11, jx, jy, jz) + w2 * g(b21 + b01, ox, jy, jz)) +
                     (w1 * g(b21 + b10, jx, oy, jz) + w3 * g(b21 + b00, ox, oy, jz));
    float n = cn6 * R1 + (cn3 * R0 + 0.5f);
    if (n > 1.0f) n = 1.0f;
    if (n < 0.0f) n = 0.0f;
    return n;
}

// the distance metrics of voronoi_t (noise.h:69-129), e = mk_exponent, as
// the shipped build evaluates them (sums grouped x + (y + z); manhattan,
// minkovsky 1/2, 4 and general in double)
float vor_dist(int metric, float x, float y, float z, float e) {
    switch (metric) {
    case YR_DIST_SQUARED: return x * x + (y * y + z * z);
    case YR_DIST_MANHATTAN: return (float)((double)fabsf(x) + ((double)fabsf(y) + (double)fabsf(z)));
    case YR_DIST_CHEBYCHEV: {
        x = fabsf(x);
        y = fabsf(y);
        z = fabsf(z);
        const float t = (y > z) ? y : z;
        return (x > t) ? x : t;
    }
    case YR_DIST_MINKOVSKY_HALF: {
        const float d = (float)((sqrt((double)fabsf(x)) + sqrt((double)fabsf(y))) + sqrt((double)fabsf(z)));
        return d * d;
    }
    case YR_DIST_MINKOVSKY_FOUR: {
        const float x2 = x * x, y2 = y * y, z2 = z * z;
        return (float)sqrt(sqrt((double)(x2 * x2 + (y2 * y2 + z2 * z2))));
    }
    case YR_DIST_MINKOVSKY: {
        const double ed = (double)e;
        return (float)pow((pow((double)fabsf(x), ed) + pow((double)fabsf(y), ed)) + pow((double)fabsf(z), ed),
                          (double)(1.0f / e));
    }
    default: return sqrtf(x * x + (y * y + z * z));
    }
}

const float *hashpnt(int x, int y, int z) {  // HASHPNT (noise.cc:6)
    return kHashPnt + 3 * kPerm[(kPerm[(kPerm[z & 255] + y) & 255] + x) & 255];
}

// voronoi_t::getFeatures (noise.cc:550-589): the 4 nearest feature points
struct Features {
    float da[4];
    V pa[4];
};
void vor_features(const V &pt, int metric, float mex, Features &F) {
    const float x = pt.x, y = pt.y, z = pt.z;
    const int xi = (int)floorf(x), yi = (int)floorf(y), zi = (int)floorf(z);
    F.da[0] = F.da[1] = F.da[2] = F.da[3] = 1e10f;
    for (int xx = xi - 1; xx <= xi + 1; xx++)
        for (int yy = yi - 1; yy <= yi + 1; yy++)
            for (int zz = zi - 1; zz <= zi + 1; zz++) {
                const float *p = hashpnt(xx, yy, zz);
                // (x - xx) - p[0]: the shipped build's grouping of x - (p[0] + xx)
                const float xd = (x - (float)xx) - p[0], yd = (y - (float)yy) - p[1], zd = (z - (float)zz) - p[2];
                const float d = vor_dist(metric, xd, yd, zd, mex);
                const V fp(p[0] + (float)xx, p[1] + (float)yy, p[2] + (float)zz);
                int k = 4;
                while (k > 0 && d < F.da[k - 1]) k--;
                if (k < 4) {
                    for (int m = 3; m > k; m--) {
                        F.da[m] = F.da[m - 1];
                        F.pa[m] = F.pa[m - 1];
                    }
                    F.da[k] = d;
                    F.pa[k] = fp;
                }
            }
}

// cellNoise_t::operator() (noise.cc:614-622)
float cell_noise(const V &pt) {
    const int xi = (int)floorf(pt.x), yi = (int)floorf(pt.y), zi = (int)floorf(pt.z);
    unsigned int n = (unsigned)xi + (unsigned)yi * 1301u + (unsigned)zi * 314159u;
    n ^= (n << 13);
    return (float)((double)(float)(n * (n * n * 15731u + 789221u) + 1376312589u) / 4294967296.0);
}

// the basis of newNoise (basictex.cc:34-60)
float noise_gen(uint32_t type, const V &p) {
    switch (type) {
    case YR_NOISE_STDPERLIN: return std_perlin(p);
    case YR_NOISE_BLENDER: return blender_noise(p);
    case YR_NOISE_VORONOI_F1:
    case YR_NOISE_VORONOI_F2:
    case YR_NOISE_VORONOI_F3:
    case YR_NOISE_VORONOI_F4:
    case YR_NOISE_VORONOI_F2F1:
    case YR_NOISE_VORONOI_CRACKLE: {  // voronoi_t::operator() (noise.cc:591-611), real distance
        Features F;
        vor_features(p, YR_DIST_REAL, 2.5f, F);
        switch (type) {
        case YR_NOISE_VORONOI_F2: return F.da[1];
        case YR_NOISE_VORONOI_F3: return F.da[2];
        case YR_NOISE_VORONOI_F4: return F.da[3];
        case YR_NOISE_VORONOI_F2F1: return F.da[1] - F.da[0];
        case YR_NOISE_VORONOI_CRACKLE: {
            const float t = (F.da[1] - F.da[0]) * 10.0f;
            return (t > 1.0f) ? 1.0f : t;
        }
        default: return F.da[0];
        }
    }
    case YR_NOISE_CELLNOISE: return cell_noise(p);
    default: return perlin(p);
    }
}
float signed_noise(uint32_t type, const V &p) { return (float)2.0 * noise_gen(type, p) - (float)1.0; }

// turbulence (noise.cc:808-819) over any basis; only the blender basis
// offsets the point (noiseGenerator_t::offset, noise.h:16-17, 55-63)
float turbulence_gen(uint32_t type, const V &pt, int oct, float size, bool hard) {
    float amp = 1, sum = 0;
    const V q = type == YR_NOISE_BLENDER ? V(pt.x + 1.0f, pt.y + 1.0f, pt.z + 1.0f) : pt;
    V tp(q.x * size, q.y * size, q.z * size);
    for (int i = 0; i <= oct; i++, amp *= 0.5f, tp = V(tp.x * 2.0f, tp.y * 2.0f, tp.z * 2.0f)) {
        float val = noise_gen(type, tp);
        if (hard) val = (float)fabs(2.0 * (double)val - 1.0);
        sum += amp * val;
    }
    return sum * ((float)(1 << oct) / (float)((1 << (oct + 1)) - 1));
}

// the musgrave generators (noise.cc:638-800) over basis `nt`, in the
// shipped build's groupings: sn + offset as (offset - 1) + 2n, heteroterrain
// value *= (sn + offset)*pwr + 1, hybrid weight = (gain*w)*signal, the
// fractional octaves' products reordered as noted per case
float musgrave(uint32_t kind, uint32_t nt, V tp, float H, float lac, float oct, float offset, float gain) {
    const float pwHL = (float)pow((double)lac, (double)-H);
    auto scale = [&](V &p) { p = V(p.x * lac, p.y * lac, p.z * lac); };
    const float rmd = oct - floorf(oct);
    switch (kind) {
    case YR_TEX_MUSGRAVE_MULTIFRACTAL: {
        float value = 1, pwr = 1;
        for (int i = 0; i < (int)oct; i++) {
            value *= (pwr * signed_noise(nt, tp) + (float)1.0);
            pwr *= pwHL;
            scale(tp);
        }
        if (rmd != (float)0.0) value *= ((rmd * pwr) * signed_noise(nt, tp) + (float)1.0);
        return value;
    }
    case YR_TEX_MUSGRAVE_HETEROTERRAIN: {
        auto sno = [&](const V &q) { return (offset - 1.0f) + noise_gen(nt, q) * 2.0f; };
        float pwr = pwHL;
        float value = noise_gen(nt, tp) * 2.0f + (offset - 1.0f);
        scale(tp);
        for (int i = 1; i < (int)oct; i++) {
            value = (sno(tp) * pwr + 1.0f) * value;
            pwr *= pwHL;
            scale(tp);
        }
        if (rmd != (float)0.0) value = (pwr * value) * (sno(tp) * rmd) + value;
        return value;
    }
    case YR_TEX_MUSGRAVE_HYBRIDMF: {
        auto sno = [&](const V &q) { return (offset - 1.0f) + noise_gen(nt, q) * 2.0f; };
        float pwr = pwHL;
        float result = sno(tp);
        float weight = gain * result;
        scale(tp);
        for (int i = 1; (weight > (float)0.001) && (i < (int)oct); i++) {
            const float w = weight > 1.0f ? 1.0f : weight;
            const float signal = sno(tp) * pwr;
            pwr *= pwHL;
            result = signal * w + result;
            weight = (gain * w) * signal;
            scale(tp);
        }
        if (rmd != (float)0.0) result = sno(tp) * (rmd * pwr) + result;
        return result;
    }
    case YR_TEX_MUSGRAVE_RIDGEDMF: {
        float pwr = pwHL;
        float signal = offset - fabsf(signed_noise(nt, tp));
        signal *= signal;
        float result = signal;
        for (int i = 1; i < (int)oct; i++) {
            scale(tp);
            float weight = gain * signal;
            weight = weight > 0.0f ? weight : 0.0f;
            weight = weight < 1.0f ? weight : 1.0f;
            const float q = offset - fabsf(signed_noise(nt, tp));
            signal = weight * (q * q);
            result = signal * pwr + result;
            pwr = pwHL * pwr;
        }
        return result;
    }
    default: {  // fBm
        float value = 0, pwr = 1;
        for (int i = 0; i < (int)oct; i++) {
            value += signed_noise(nt, tp) * pwr;
            pwr *= pwHL;
            scale(tp);
        }
        if (rmd != 0.f) value += rmd * signed_noise(nt, tp) * pwr;
        return value;
    }
    }
}

C col3(const float *p) { return C(p[0], p[1], p[2]); }

// marble / wood wave shapes (basictex.cc:124-140, 199-214)
float wave(uint32_t shape, float w) {
    if (shape == YR_WAVE_SAW) {
        w *= (float)(0.5 * M_1_PI);
        w -= floorf(w);
    } else if (shape == YR_WAVE_TRI) {
        w *= (float)(0.5 * M_1_PI);
        w = fabsf((float)2.0 * (w - floorf(w)) - (float)1.0);
    } else {
        w = (sinf(w) + 1.0f) * 0.5f;  // the shipped build's form of 0.5 + 0.5*sin(w)
    }
    return w;
}

// A texture's value: getFloat, and getColor (rgb) at texture point p.
struct TexVal {
    float f;
    C col;
};
TexVal texture_eval(const yr_shader_desc &d, const V &p) {
    TexVal r;
    const C c1 = col3(d.tex_color1), c2 = col3(d.tex_color2);
    const V ps(p.x * d.tex_size, p.y * d.tex_size, p.z * d.tex_size);
    switch (d.tex_type) {
    case YR_TEX_CLOUDS: {  // textureClouds_t::getFloat (basictex.cc:76-85)
        float v = turbulence_gen(d.tex_noise, p, d.tex_depth, d.tex_size, d.tex_hard != 0);
        if (d.tex_variant == 1 || d.tex_variant == 2) {
            v *= v;
            if (d.tex_variant == 1) v = -v;
        }
        r.f = v;
        break;
    }
    case YR_TEX_MARBLE: {  // textureMarble_t::getFloat (basictex.cc:122-146)
        const float sharp = d.tex_sharpness > 1 ? (float)(1.0 / (double)d.tex_sharpness) : 1.0f;
        const double tu = d.tex_turbulence == 0.0f
                              ? 0.0
                              : (double)(d.tex_turbulence *
                                         turbulence_gen(d.tex_noise, p, d.tex_depth, d.tex_size, d.tex_hard != 0));
        const float w = (float)((double)(p.x + p.y + p.z) * 5.0 + tu);
        r.f = powf(wave(d.tex_shape, w), sharp);
        break;
    }
    case YR_TEX_WOOD: {  // textureWood_t::getFloat (basictex.cc:192-216)
        float w = d.tex_variant ? sqrtf(p.x * p.x + p.y * p.y + p.z * p.z) * 20.0f : (p.x + p.y + p.z) * 10.0f;
        const double tu = d.tex_turbulence == 0.0f
                              ? 0.0
                              : (double)(d.tex_turbulence *
                                         turbulence_gen(d.tex_noise, p, d.tex_depth, d.tex_size, d.tex_hard != 0));
        w = (float)((double)w + tu);
        r.f = wave(d.tex_shape, w);
        break;
    }
    case YR_TEX_VORONOI: {  // textureVoronoi_t (basictex.cc:560-617)
        const float aw[4] = {fabsf(d.tex_weights[0]), fabsf(d.tex_weights[1]), fabsf(d.tex_weights[2]),
                             fabsf(d.tex_weights[3])};
        float iscale = aw[0] + aw[1] + aw[2] + aw[3];
        if (iscale != 0) iscale = d.tex_intensity / iscale;
        Features F;
        vor_features(ps, (int)d.tex_metric, d.tex_mk_exponent, F);
        // the weighted sum as the shipped build's vector reduction
        const float inte = iscale * fabsf((d.tex_weights[0] * F.da[0] + d.tex_weights[2] * F.da[2]) +
                                          (d.tex_weights[1] * F.da[1] + d.tex_weights[3] * F.da[3]));
        r.f = inte;
        if (d.tex_shape == 0) {
            r.col = C(inte, inte, inte);
        } else {
            C col;
            for (int k = 0; k < 4; k++) {  // cellNoiseColor (noise.cc:795-803)
                const float *cl = hashpnt((int)floorf(F.pa[k].x), (int)floorf(F.pa[k].y), (int)floorf(F.pa[k].z));
                col = col + C(aw[k] * cl[0], aw[k] * cl[1], aw[k] * cl[2]);
            }
            if (d.tex_shape >= 2) {
                const float dd = F.da[1] - F.da[0];
                float t1 = dd > 0.1f ? 1.0f : dd * 10.0f;  // the shipped build's form
                if (d.tex_shape == 3) t1 *= inte;
                else t1 *= iscale;
                col = col * t1;
            } else {
                col = col * iscale;
            }
            r.col = col;
        }
        return r;
    }
    case YR_TEX_DISTORTED_NOISE: {  // textureDistortedNoise_t::getFloat (basictex.cc:721-727)
        const V rv(signed_noise(d.tex_noise, V(ps.x + 13.5f, ps.y + 13.5f, ps.z + 13.5f)),
                   signed_noise(d.tex_noise, ps), signed_noise(d.tex_noise, V(ps.x - 13.5f, ps.y - 13.5f, ps.z - 13.5f)));
        r.f = signed_noise(d.tex_noise2, V(ps.x + rv.x * d.tex_distort, ps.y + rv.y * d.tex_distort,
                                           ps.z + rv.z * d.tex_distort));
        break;
    }
    case YR_TEX_GRADIENT: {  // textureGradient_t::getFloat (basictex.cc:772-800)
        const float x = d.tex_variant ? p.y : p.x, y = d.tex_variant ? p.x : p.y;
        float gr;
        switch (d.tex_shape) {
        case YR_GRAD_QUADRATIC:
            gr = (float)((1.0 + (double)x) * 0.5);
            r.f = gr < 0 ? 0.f : gr * gr;
            break;
        case YR_GRAD_CUBIC:
            gr = (float)((1.0 + (double)x) * 0.5);
            if (gr > 1) {  // getColor folds color1 + 1*(color2 - color1) to color2 in the shipped build
                r.f = 1.f;
                r.col = c2;
                return r;
            }
            r.f = gr < 0 ? 0.f : (float)((double)(gr * gr) * (3.0 - 2.0 * (double)gr));
            break;
        case YR_GRAD_DIAGONAL: r.f = (float)(((double)x + (double)y + 2.0) * 0.25); break;
        case YR_GRAD_SPHERE:
        case YR_GRAD_HALO:
            gr = (float)(1.0 - (double)sqrtf(x * x + y * y + p.z * p.z));
            r.f = gr < 0 ? 0.f : (d.tex_shape == YR_GRAD_HALO ? gr * gr : gr);
            break;
        default: r.f = (float)((1.0 + (double)x) * 0.5);
        }
        break;
    }
    default:  // musgrave: iscale * generator(p * size) (basictex.cc:677-680)
        r.f = d.tex_intensity *
              musgrave(d.tex_type, d.tex_noise, ps, d.tex_H, d.tex_lacunarity, d.tex_octaves, d.tex_offset, d.tex_gain);
    }
    r.col = c1 + r.f * (c2 - c1);
    return r;
}

// --------------------------------------------------------------- shading
struct SP {
    V P, N, Ng, NU, NV;
    V orco;  // toObjectOrco(P): P, or M^-1 P on a reference
    int obj;
    int shader;
    float sx = 0.f, sy = 0.f;  // screen position (camera hits only; 0 elsewhere)
    float u = -1.f, v = -1.f;  // texture coordinates (triangle_t::getSurface)
};

void createCS(const V &N, V &u, V &v) {  // vector3d.h:240-258
    if ((N.x == 0) && (N.y == 0)) {
        u = (N.z < 0) ? V(-1, 0, 0) : V(1, 0, 0);
        v = V(0, 1, 0);
    } else {
        const float d = (float)(1.0 / sqrt((double)(N.y * N.y + N.x * N.x)));
        u = V(N.y * d, -N.x * d, 0);
        v = N ^ u;
    }
}
V faceForward(const V &Ng, const V &N, const V &I) { return ((Ng * I) < 0) ? -N : N; }
V reflectv(const V &n, const V &v) {
    const float vn = v * n;
    if (vn < 0) return -v;
    return (2 * vn) * n - v;
}

SP surface(const Scene &S, int obj, uint32_t tri, float Z, const V &from_w, const V &ray_w) {
    SP s;
    // a reference's hit is formed in its original's space (the ray taken
    // there by M's inverse), then N, Ng, NU, NV go back by MRot and P by M
    // (referenceObject_t::shoot, reference.cc:95-114)
    const Obj &ow = S.objs[obj];
    const bool ref = ow.inst >= 0;
    const V from = ref ? xf_point(ow.back, from_w) : from_w, ray = ref ? xf_vec(ow.back, ray_w) : ray_w;
    s.P = from + Z * ray;
    const Obj &o = ref ? S.objs[ow.inst] : ow;
    s.N = s.Ng = o.tri_n[tri];
    const bool has_uv = !o.tri_uv.empty();
    // without uv, corner normals or orco, getSurface returns u = v = -1 at
    // once; otherwise u, v are the barycentric blend of the triangle's
    // coordinates, or 0 without any (triangle.cc:138-160)
    if (o.smooth || has_uv) s.u = s.v = 0.f;
    if (o.smooth || has_uv) {
        // triangle_t::getSurface + getInterpolation (triangle.cc:74-155), in
        // the shipped build's evaluation order (fast-math): the reciprocal
        // of the denominator, fa from the sum of the numerators, and
        // na*fa + (nb*fb + nc*fc)
        const V &a = o.tri_a[tri], &b = o.tri_b[tri], &c = o.tri_c[tri], &h = s.P, &N = s.Ng;
        float uu0, vv0, uu1, vv1, uu2, vv2;
        const float nx = fabsf(N.x), ny = fabsf(N.y), nz = fabsf(N.z);
        if (nx >= ny && nx >= nz) {
            uu0 = h.y - a.y; vv0 = h.z - a.z; uu1 = b.y - a.y; vv1 = b.z - a.z; uu2 = c.y - a.y; vv2 = c.z - a.z;
        } else if (ny >= nx && ny >= nz) {
            uu0 = h.x - a.x; vv0 = h.z - a.z; uu1 = b.x - a.x; vv1 = b.z - a.z; uu2 = c.x - a.x; vv2 = c.z - a.z;
        } else {
            uu0 = h.x - a.x; vv0 = h.y - a.y; uu1 = b.x - a.x; vv1 = b.y - a.y; uu2 = c.x - a.x; vv2 = c.y - a.y;
        }
        const float an = uu0 * vv2 - vv0 * uu2, bn = uu1 * vv0 - vv1 * uu0, den = uu1 * vv2 - vv1 * uu2;
        const float rc = 1.f / den, fb = an * rc, fc = bn * rc, fa = 1.f - (an + bn) * rc;
        if (o.smooth) {
            const V &na = o.tri_na[tri], &nb = o.tri_nb[tri], &nc = o.tri_nc[tri];
            s.N = normalize(V(na.x * fa + (nb.x * fb + nc.x * fc), na.y * fa + (nb.y * fb + nc.y * fc),
                              na.z * fa + (nb.z * fb + nc.z * fc)));
        }
        if (has_uv) {
            const float *uv = &o.tri_uv[6 * (size_t)tri];
            s.u = uv[0] * fa + (uv[2] * fb + uv[4] * fc);
            s.v = uv[1] * fa + (uv[3] * fb + uv[5] * fc);
        }
    }
    createCS(s.N, s.NU, s.NV);
    s.orco = s.P;
    if (ref) {
        s.N = rot_vec(ow.rot, s.N);
        s.Ng = rot_vec(ow.rot, s.Ng);
        s.P = xf_point(ow.m, s.P);
        s.NU = rot_vec(ow.rot, s.NU);
        s.NV = rot_vec(ow.rot, s.NV);
        s.orco = xf_point(ow.back, s.P);  // referenceObject_t::toObjectOrco
    }
    if (o.has_orco) s.orco = xf_point(o.orco, s.orco);  // meshObject_t::toObjectOrco of a transformed mesh
    s.obj = obj;
    s.shader = (int)o.tri_shader[tri];
    return s;
}


// the modulator's texture point (modulator_t::doMapping, texture.cc:122-320,
// procedural path): texco "global" / "orco" (an untransformed mesh without
// orco data: P) or "normal", then projections size*(src[axis] + ofs) /
// size*ofs
V tex_point(const yr_shader_desc &d, const SP &sp, const V &eye) {
    const uint32_t tc = d.tex_map & 0xffu;
    V src = tc == YR_TEXCO_NORMAL ? sp.N : (tc == YR_TEXCO_ORCO ? sp.orco : sp.P);
    if (tc == YR_TEXCO_WINDOW) src = V(sp.sx, sp.sy, 0.f);
    if (tc == YR_TEXCO_UV) src = V((float)((double)sp.u * 2.0 - 1.0), (float)(1.0 - (double)sp.v * 2.0), 0.f);
    if (tc == YR_TEXCO_REFLECT) {  // texture.cc:158-165
        const V neye = normalize(eye);
        src = reflectv(faceForward(sp.Ng, sp.N, neye), neye);
    }
    float t[3];
    for (int k = 0; k < 3; k++) {
        const uint32_t pc = (d.tex_map >> (8 * (k + 1))) & 0xffu;
        const int a = pc == YR_PROJ_DEFAULT ? k : (pc >= YR_PROJ_X && pc <= YR_PROJ_Z ? (int)pc - 1 : -1);
        t[k] = a < 0 ? d.mod_size[k] * d.mod_ofs[k] : d.mod_size[k] * (src[a] + d.mod_ofs[k]);
    }
    return V(t[0], t[1], t[2]);
}

// mix(a, b, point) (color.cc:103-109)
C mixc(const C &a, const C &b, float w) {
    if (w < 0.0) return b;
    if (w > 1.0) return a;
    return a * w + (1 - w) * b;
}

// modulator_t::modulate (texture.cc:499-534): the diffuse colour C, the
// specular colour S and the Phong exponent H after the modulator, each
// channel by its own weight ("color", "specular", "hard"; a channel whose
// weight is not above 0 is left as it is), modes mix / mul / add / sub
struct Mod {
    C c, s;
    float h;
};
Mod modulated(const Scene &S, const SP &sp, const V &eye) {
    const yr_shader_desc &d = S.shaders[sp.shader];
    Mod m;
    m.c = col3(d.color);
    m.s = col3(d.specular);
    m.h = d.hard;
    if (d.tex_type == YR_TEX_NONE || !(d.mod_color > 0 || d.mod_specular > 0 || d.mod_hard > 0)) return m;
    const TexVal tv = texture_eval(d, tex_point(d, sp, eye));
    const C &tex = tv.col;
    const float tf = tv.f, wc = d.mod_color, ws = d.mod_specular, wh = d.mod_hard;
    switch (d.mod_mode) {
    case YR_MOD_MUL:
        if (wc > 0) m.c = mixc(tex, C(1, 1, 1), wc) * m.c;
        if (ws > 0) m.s = mixc(tex, C(1, 1, 1), ws) * m.s;
        if (wh > 0) m.h = (tf * wh + (1 - wh)) * m.h;
        break;
    case YR_MOD_ADD:
        if (wc > 0) m.c = (tex * wc) + m.c;
        if (ws > 0) m.s = (tex * ws) + m.s;
        if (wh > 0) m.h = tf * wh + m.h;
        break;
    case YR_MOD_SUB:
        if (wc > 0) m.c = (tex * -wc) + m.c;
        if (ws > 0) m.s = (tex * -ws) + m.s;
        if (wh > 0) m.h = (tf * -wh) + m.h;
        break;
    default:
        if (wc > 0) m.c = mixc(tex, m.c, wc);
        if (ws > 0) m.s = mixc(tex, m.s, ws);
        if (wh > 0) m.h = tf * wh + m.h * (1 - wh);
        break;
    }
    return m;
}

// the diffuse colour after the modulator (genericShader_t::getDiffuse,
// basicshaders.cc:191-204)
C diffuse(const Scene &S, const SP &sp, const V &eye) { return modulated(S, sp, eye).c; }

// genericShader_t::fromLight (basicshaders.cc:46-70)
C fromLight(const Scene &S, const SP &sp, const V &ldir, const C &lcol, const V &eye) {
    V edir = normalize(eye);
    V N = faceForward(sp.Ng, sp.N, edir);
    float inte = N * ldir;
    if (inte < 0) return C();
    const Mod m = modulated(S, sp, eye);
    edir = reflectv(N, edir);
    float refle = edir * ldir;
    if (refle < 0) refle = 0;
    else refle = (float)pow((double)refle, (double)m.h);
    return ((C(1.f * inte, 1.f * inte, 1.f * inte) * lcol) * m.c) + (m.s * refle) * lcol;
}

// --------------------------------------------------------------- lights
struct Ctx {
    uint32_t pixel, s, pi;  // pixel, camera sample, path index
    int npath;
    uint32_t stride = 1;    // camera samples per pixel: round r of the path light uses index (r*stride + s)*P + i
};

C illum_point(Scene &S, const Light &L, const SP &sp, const V &eye) {
    V Lv = L.from - sp.P;
    V dir = normalize(Lv);
    float id2 = Lv * Lv;
    if (id2 != 0.f) id2 = 1.f / id2;
    C col;
    if (L.d.cast_shadows ? !shadowed_point(S, sp.P, sp.obj, L.from) : true)
        col = fromLight(S, sp, dir, L.color * id2, eye);
    return col;
}

// areaLight_t::guessLight (arealight.cc:176-198): `psamples` probes of
// unjittered grid points, in order; a probe sees shadow when the point is
// behind the surface or occluded, light otherwise; the guess stops at the
// first probe once both were seen.  Probe j of QMC sample index m0 looks at
// grid point floor(samples * u), u = halton(5, m0*psamples + j) rotated by
// the light's first dimension (the reference draws rand() % samples); in
// the pinning queries the grid points come from the reference's draws.
enum { kGuessShadow = 0, kGuessPenumbra = 1, kGuessLight = 2 };
int guess_light(Scene &S, const Light &L, const SP &sp, const V &N, uint32_t m0, float r0) {
    const int F = L.d.psamples;
    if (F <= 0) return kGuessPenumbra;
    bool luz = false, sombra = false;
    for (int j = 0; j < F; j++) {
        if (luz && sombra) return kGuessPenumbra;
        int rs;
        if (S.area_vals) {
            rs = (int)S.area_vals[2 * L.samples + j];
        } else {
            const float u = cp_add(halton(5, m0 * (uint32_t)F + (uint32_t)j), r0);
            rs = (int)(u * (float)L.samples);
            if (rs >= L.samples) rs = L.samples - 1;
        }
        const V Lv = L.pts[rs] - sp.P;
        if ((Lv * N) < 0) sombra = true;
        else if (shadowed_point(S, sp.P, sp.obj, L.pts[rs])) sombra = true;
        else luz = true;
    }
    if (luz && sombra) return kGuessPenumbra;
    return luz ? kGuessLight : kGuessShadow;
}

C illum_area(Scene &S, int k, const Light &L, const SP &sp, const V &eye, int v, uint32_t m0, const Ctx &cx) {
    V edir = normalize(eye);
    V N = faceForward(sp.Ng, sp.N, edir);
    float plane_at = (sp.P - L.from) * L.direction;
    if (plane_at <= 0) return C();
    const uint32_t d = light_dim(k, v);
    const float r0 = rot(S, cx.pixel, d), r1 = rot(S, cx.pixel, d + 1);
    C resul;
    if (L.samples > 1) {
        const int g = guess_light(S, L, sp, N, m0, r0);
        if (g == kGuessShadow) return C();  // fromLight of zero energy
        if (g == kGuessLight) {
            // every grid point, unjittered, without a shadow test (arealight.cc:156-166)
            for (int i = 0; i < L.samples; i++) {
                V dir = L.pts[i] - sp.P;
                float ld2 = normLenSqr(dir);
                ld2 = (ld2 != 0) ? (1.f / ld2) : 1.f;
                resul = resul + fromLight(S, sp, dir, (L.d.power * L.color) * ld2, eye);
            }
            return (plane_at * resul) / (float)L.samples;
        }
    }
    for (int i = 0; i < L.samples; i++) {
        const uint32_t m = m0 * (uint32_t)L.samples + (uint32_t)i;
        float h2, h3;
        if (S.area_vals) {
            // the shipped build draws toY's value first in the one-sample
            // expression corner + toX*ourRandom() + toY*ourRandom()
            h2 = S.area_vals[L.samples == 1 ? 1 : 2 * i];
            h3 = S.area_vals[L.samples == 1 ? 0 : 2 * i + 1];
        } else {
            h2 = cp_add(halton(2, m), r0);
            h3 = cp_add(halton(3, m), r1);
        }
        V sampleP;
        if (L.samples == 1) sampleP = (L.corner + L.tox * h2) + L.toy * h3;
        else sampleP = (L.pts[i] + L.jit1[i] * (h2 - 0.5f)) + L.jit2[i] * (h3 - 0.5f);
        V Lv = sampleP - sp.P;
        if ((Lv * N) < 0) continue;
        if (!shadowed_point(S, sp.P, sp.obj, sampleP)) {
            V dir = Lv;
            float ld2 = normLenSqr(dir);
            ld2 = (ld2 != 0) ? (1.f / ld2) : 1.f;
            resul = resul + fromLight(S, sp, dir, (L.d.power * L.color) * ld2, eye);
        }
    }
    return (plane_at * resul) / (float)L.samples;
}

V uniHemi(const V &N, const V &Ru, const V &Rv, float z1, float z2) {  // hemilight.cc:103-114
    z2 = (float)((double)z2 * 6.283185307179586);
    const float c = (float)cos((double)z2), s = (float)sin((double)z2);
    return (Ru * c + Rv * s) * (float)sqrt(1.0 - (double)(z1 * z1)) + N * z1;
}

C illum_hemi(Scene &S, int k, const Light &L, const SP &sp, const V &eye, int v, uint32_t m0, const Ctx &cx) {
    V N = faceForward(sp.Ng, sp.N, eye);
    C fl = fromLight(S, sp, N, C(1, 1, 1), eye);
    float mad = fabsf(fl.r);
    if (fabsf(fl.g) > mad) mad = fabsf(fl.g);
    if (fabsf(fl.b) > mad) mad = fabsf(fl.b);
    if (below_cut(mad)) return C();
    const uint32_t d = light_dim(k, v);
    const float r0 = rot(S, cx.pixel, d), r1 = rot(S, cx.pixel, d + 1);
    C total;
    for (int sm = 0; sm < L.samples; sm++) {
        const uint32_t m = m0 * (uint32_t)L.samples + (uint32_t)sm;
        V dir = uniHemi(N, sp.NU, sp.NV, cp_add(halton(2, m), r0), cp_add(halton(3, m), r1));
        float occ = dir * N;
        if (occ > 0) {
            bool sh = (L.d.maxdist > 0) ? shadowed_point(S, sp.P, sp.obj, sp.P + L.d.maxdist * dir)
                                        : shadowed_dir(S, sp.P, sp.obj, dir);
            if (!sh) total = total + L.color * occ;
        }
    }
    return (L.sampdiv * total) * fl;
}

V cosHemi(const V &N, const V &Ru, const V &Rv, float z1, float z2) {  // pathtools.cc:32-43
    if (z1 > 1.0f) z1 = 1.0f;
    z2 = (float)((double)z2 * 6.283185307179586);
    const float c = (float)cos((double)z2), s = (float)sin((double)z2);
    return (Ru * c + Rv * s) * (float)sqrt(1.0 - (double)z1) + N * sqrtf(z1);
}

// scene_t::light (scene.cc:260-277) without the path light (indirect) or
// with it (camera vertex); v = QMC vertex level, m0 = QMC sample index.
C light_sum(Scene &S, const SP &sp, const V &eye, bool indirect, int v, uint32_t m0, const Ctx &cx);

void expgam_adjust(float *c, float e, float g, bool clamp_rgb);

// the scene's color_t::expgam_Adjust (scene_t::adjustColor, scene.h:164):
// applied whether or not the render tone-maps its samples
C adjust_color(const Scene &S, const C &c) {
    float v[3] = {c.r, c.g, c.b};
    const float e = -S.rp.exposure, g = S.rp.gamma != 0.f ? (float)(1.0 / (double)S.rp.gamma) : 0.f;
    expgam_adjust(v, e, g, (S.rp.flags & YR_RENDER_CLAMP_RGB) != 0);
    return C(v[0], v[1], v[2]);
}

// The adaptive extra rounds of pathLight_t::takeSample (pathlight.cc:349-374):
// from the first round's four partial sums (path i adds to sum i % 4),
// each times multiplier() = 1/P, the per-channel minimum and maximum after
// the scene's tone adjustment; extra = int(diff^2) - 1 in [0, 3] with
// diff = maxAbsDiff(max, min) / (max(ene, 1) * 4) / threshold and
// ene = maxAbsDiff(min, 0).
int extra_rounds(const Scene &S, const C *sub, int P, float threshold) {
    float mn[3] = {1000, 1000, 1000}, mx[3] = {0, 0, 0};
    const float mult = (float)(1.0 / (double)(float)P);
    for (int k = 0; k < 4; k++) {
        const C c = sub[k] * mult;
        const float v[3] = {c.r, c.g, c.b};
        for (int ch = 0; ch < 3; ch++) {
            if (v[ch] > mx[ch]) mx[ch] = v[ch];
            if (v[ch] < mn[ch]) mn[ch] = v[ch];
        }
    }
    const C lo = adjust_color(S, C(mn[0], mn[1], mn[2])), hi = adjust_color(S, C(mx[0], mx[1], mx[2]));
    const float ene = fmaxf(fabsf(lo.r), fmaxf(fabsf(lo.g), fabsf(lo.b)));
    const float mad = fmaxf(fabsf(hi.r - lo.r), fmaxf(fabsf(hi.g - lo.g), fabsf(hi.b - lo.b)));
    float diff = (float)((double)mad / (((ene < 1.0) ? 1.0 : (double)ene) * 2.0 * 2.0));
    diff /= threshold;
    int extra = (int)(diff * diff) - 1;
    if (extra > 3) extra = 3;
    if (extra < 0) extra = 0;
    return extra;
}

// pathLight_t::normalSample + takeSample (pathlight.cc:223-403), explicit indices
C illum_path(Scene &S, const Light &L, const SP &sp, const V &eye, const Ctx &cx) {
    V N = faceForward(sp.Ng, sp.N, eye);
    C dif = diffuse(S, sp, eye);
    if (below_cut(energy(dif))) return C();
    const int P = L.d.samples, depth = L.d.depth;
    C total, sub[4];
    int rounds = 1;
    for (int r = 0; r < rounds; r++) {
    for (int i = 0; i < P; i++) {
        const uint32_t n = ((uint32_t)r * cx.stride + cx.s) * (uint32_t)P + (uint32_t)i;
        V ray = cosHemi(N, sp.NU, sp.NV, cp_add(halton(kPrimes[0], n), rot(S, cx.pixel, 0)),
                        cp_add(halton(kPrimes[1], n), rot(S, cx.pixel, 1)));
        const V startray = ray;
        V where = sp.P;
        C raycolor(1, 1, 1);
        const float startN = startray * N;
        for (int j = 0; j < depth; ++j) {
            if (below_cut(energy(raycolor))) break;
            t_st.bounce++;
            const V f = where + ray * kMinRay;
            Hit h = closest(S, f, ray, false, true);
            if (h.obj < 0) {
                const C contri = (startN * raycolor) * col3(S.rp.background);
                total = total + contri;
                if (r == 0) sub[i % 4] = sub[i % 4] + contri;
                break;
            }
            SP t = surface(S, h.obj, h.tri, h.Z, f, ray);
            Ctx c2 = cx;
            c2.pi = (uint32_t)i;
            const V eye2 = (t.P + (-ray)) - t.P;
            C light = light_sum(S, t, eye2, true, j + 1, n, c2);
            const C contri = (startN * raycolor) * light;
            total = total + contri;
            if (r == 0) sub[i % 4] = sub[i % 4] + contri;
            const V HN = faceForward(t.Ng, t.N, -ray);
            raycolor = raycolor * diffuse(S, t, -ray);
            if (j + 1 < depth) {
                const int lev = j + 1;
                ray = cosHemi(HN, t.NU, t.NV,
                              cp_add(halton(kPrimes[2 * lev], n), rot(S, cx.pixel, 2 * lev)),
                              cp_add(halton(kPrimes[2 * lev + 1], n), rot(S, cx.pixel, 2 * lev + 1)));
            }
            where = t.P;
        }
    }
        if (r == 0 && L.d.threshold > 0.f) rounds += extra_rounds(S, sub, P, L.d.threshold);
    }
    total = total * ((float)(1.0 / (double)(float)P) / (float)rounds);
    return (dif * total) * L.d.power;
}

C light_sum(Scene &S, const SP &sp, const V &eye, bool indirect, int v, uint32_t m0, const Ctx &cx) {
    C fl;
    for (size_t k = 0; k < S.lights.size(); k++) {
        const Light &L = S.lights[k];
        switch (L.d.type) {
        case YR_LIGHT_POINT: fl = fl + illum_point(S, L, sp, eye); break;
        case YR_LIGHT_AREA: fl = fl + illum_area(S, (int)k, L, sp, eye, v, m0, cx); break;
        case YR_LIGHT_HEMI: fl = fl + illum_hemi(S, (int)k, L, sp, eye, v, m0, cx); break;
        case YR_LIGHT_PATH:
            if (!indirect) fl = fl + illum_path(S, L, sp, eye, cx);
            break;
        }
    }
    return fl;
}

// camera_t ctor + shootRay (camera.cc:27-87, 146-210)
void make_camera(const yr_camera_desc &c, Cam &o) {
    const V pos(c.pos[0], c.pos[1], c.pos[2]);
    V vup = V(c.up[0], c.up[1], c.up[2]) - pos;
    V vto = V(c.look[0], c.look[1], c.look[2]) - pos;
    V vright = vup ^ vto;
    vup = vright ^ vto;
    vup = normalize(vup);
    vright = normalize(vright);
    vright = vright * -1.0f;
    float vl = vto * vto;
    if (vl != 0) {
        vl = sqrtf(vl);
        const float d = 1.0f / vl;  // the shipped build divides in float
        vto = V(vto.x * d, vto.y * d, vto.z * d);
    }
    // the shipped build (-ffast-math) multiplies by the reciprocals of
    // resx and resy: vup *= (resy*aspect) * (1/resx), vup *= 1/resy, vright *= 1/resx
    const float rx = 1.0f / (float)c.resx, ry = 1.0f / (float)c.resy;
    vup = vup * (((float)c.resy * c.aspect) * rx);
    vto = (vto * c.focal) - 0.5f * (vup + vright);
    vup = vup * ry;
    vright = vright * rx;
    o.pos = pos;
    o.vright = vright;
    o.vup = vup;
    o.vto = vto;
    o.resx = c.resx;
    o.resy = c.resy;
}
V shoot(const Cam &c, float px, float py) { return normalize(c.vto + (c.vright * px + c.vup * py)); }

// color_t::expgam_Adjust (color.h:175-195) as the shipped build evaluates
// it: x = 1 - exp(e*max(x,0)) with the product in float and exp in double;
// x = pow(max(x,0), gamma_R) in double; clamp to [0,1] only when neither
void expgam_adjust(float *c, float e, float g, bool clamp_rgb) {
    if (e == 0.f && g == 1.f) {
        if (clamp_rgb)
            for (int k = 0; k < 3; k++) c[k] = fmaxf(fminf(c[k], 1.f), 0.f);
        return;
    }
    if (e != 0.f)
        for (int k = 0; k < 3; k++) c[k] = (float)(1.0 - exp((double)(e * fmaxf(c[k], 0.f))));
    if (g != 1.f)
        for (int k = 0; k < 3; k++) c[k] = (float)pow((double)fmaxf(c[k], 0.f), (double)g);
}

// the scene's per-sample tone mapping (scene.cc:763, 807), when on
void tonemap_sample(const Scene &S, float *rgba) {
    if (!(S.rp.flags & YR_RENDER_TONEMAP)) return;
    // scene_t::setExposure / setGamma (scene.h:162-163)
    const float e = -S.rp.exposure, g = S.rp.gamma != 0.f ? (float)(1.0 / (double)S.rp.gamma) : 0.f;
    expgam_adjust(rgba, e, g, (S.rp.flags & YR_RENDER_CLAMP_RGB) != 0);
}

// one camera sample: scene_t::raytrace (scene.cc:200-258)
void camera_sample(Scene &S, uint32_t pixel, uint32_t s, float *rgba) {
    const uint32_t spp = S.rp.spp ? S.rp.spp : 1;
    const int x = (int)(pixel % (uint32_t)S.cam.resx), y = (int)(pixel / (uint32_t)S.cam.resx);
    float fx = 0.5f, fy = 0.5f;
    if (s > 0) {
        const uint32_t c = s - 1;
        const float tsd = (float)(1.0 / (float)(spp - 1));
        fx = (float)(0.5 + (double)S.rp.aa_pixelwidth * ((double)ri_lp(c + pixel) - 0.5));
        fy = (float)(0.5 + (double)S.rp.aa_pixelwidth * ((double)((float)c * tsd) - 0.5));
    }
    const V ray = shoot(S.cam, (float)x + fx, (float)y + fy);
    t_st.primary++;
    if (S.rp.raydepth <= 0) {
        rgba[0] = rgba[1] = rgba[2] = rgba[3] = 0.f;
        tonemap_sample(S, rgba);
        return;
    }
    const V f = S.cam.pos + ray * kMinRay;
    Hit h = closest(S, f, ray, true, false);
    if (h.obj < 0) {
        rgba[0] = S.rp.background[0];
        rgba[1] = S.rp.background[1];
        rgba[2] = S.rp.background[2];
        rgba[3] = 0.f;
        tonemap_sample(S, rgba);
        return;
    }
    SP sp = surface(S, h.obj, h.tri, h.Z, f, ray);
    // state.screenpos, given to the camera hit (scene.cc:234, 749-750, 798-799)
    sp.sx = (float)(2.0 * (double)(((float)x + fx) / (float)S.cam.resx) - 1.0);
    sp.sy = (float)(1.0 - 2.0 * (double)(((float)y + fy) / (float)S.cam.resy));
    Ctx cx;
    cx.pixel = pixel;
    cx.s = s;
    cx.pi = 0;
    cx.stride = spp;
    C c = light_sum(S, sp, S.cam.pos - sp.P, false, 0, s, cx);
    rgba[0] = c.r;
    rgba[1] = c.g;
    rgba[2] = c.b;
    rgba[3] = 1.f;
    tonemap_sample(S, rgba);
}

// ----------------------------------------------------------- scene load
template <class T>
bool rdv(FILE *f, T *p, size_t n) {
    return n == 0 || fread(p, sizeof(T), n, f) == n;
}

V vtx(const std::vector<float> &v, uint32_t i) { return V(v[3 * i], v[3 * i + 1], v[3 * i + 2]); }

}  // namespace

extern "C" {

typedef struct orc_scene orc_scene;
struct orc_scene {
    Scene s;
};

// meshObject_t::autoSmooth (mesh.cc:201-279) in the shipped build's order:
// vertex normals (angle >= 180) are normalized with the length summed as
// y*y + (x*x + z*z); the per-corner test uses the dot y*y' + (z*z' + x*x').
void auto_smooth(Obj &ob, const std::vector<uint32_t> &t, uint32_t nv, float angle) {
    const size_t nt = ob.tri_n.size();
    ob.smooth = true;
    ob.tri_na.resize(nt);
    ob.tri_nb.resize(nt);
    ob.tri_nc.resize(nt);
    std::vector<V> *corner[3] = {&ob.tri_na, &ob.tri_nb, &ob.tri_nc};
    if (angle >= 180.f) {
        std::vector<V> vn(nv);
        for (size_t k = 0; k < nt; k++)
            for (int j = 0; j < 3; j++) vn[t[3 * k + j]] = vn[t[3 * k + j]] + ob.tri_n[k];
        for (size_t i = 0; i < vn.size(); i++) {
            V &a = vn[i];
            const float l = a.y * a.y + (a.x * a.x + a.z * a.z);
            if (l != 0) {
                const float q = (float)(1.0 / sqrt((double)l));
                a.x *= q;
                a.y *= q;
                a.z *= q;
            }
        }
        for (size_t k = 0; k < nt; k++)
            for (int j = 0; j < 3; j++) (*corner[j])[k] = vn[t[3 * k + j]];
        return;
    }
    const float cosa = (float)cos((double)angle * M_PI / 180.0);
    std::vector<std::vector<size_t> > cnx(nv);
    for (size_t k = 0; k < nt; k++)
        for (int j = 0; j < 3; j++) cnx[t[3 * k + j]].push_back(k);
    for (size_t k = 0; k < nt; k++) {
        const V &N = ob.tri_n[k];
        for (int j = 0; j < 3; j++) {
            V sn(0, 0, 0);
            const std::vector<size_t> &around = cnx[t[3 * k + j]];
            for (size_t m = 0; m < around.size(); m++) {
                const V &M = ob.tri_n[around[m]];
                if (cosa < M.y * N.y + (M.z * N.z + M.x * N.x)) sn = sn + M;
            }
            (*corner[j])[k] = normalize(sn);
        }
    }
}

// Load a YRS1 file.  Trees are added with orc_set_tree / orc_set_object_tree.
orc_scene *orc_load(const char *path) {
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    char magic[4];
    uint32_t hdr[4];
    orc_scene *o = new orc_scene;
    Scene &S = o->s;
    yr_camera_desc cam;
    bool ok = rdv(f, magic, 4) && memcmp(magic, "YRS1", 4) == 0 && rdv(f, hdr, 4) && rdv(f, &cam, 1);
    // render parameters before record version 3 end at exposure (gamma then 1)
    memset(&S.rp, 0, sizeof(S.rp));
    S.rp.gamma = 1.f;
    const size_t rpsize = hdr[3] >= 3 ? sizeof(yr_render_params) : offsetof(yr_render_params, exposure);
    ok = ok && fread(&S.rp, 1, rpsize, f) == rpsize;
    S.shaders.assign(hdr[1], yr_shader_desc());
    std::vector<yr_light_desc> ld(hdr[2]);
    // shader records before version 2 end at mod_mode, before version 5 at mod_specular
    const size_t shsize = hdr[3] >= 5   ? sizeof(yr_shader_desc)
                          : hdr[3] >= 2 ? offsetof(yr_shader_desc, mod_specular)
                                        : offsetof(yr_shader_desc, mod_mode);
    for (uint32_t i = 0; ok && i < hdr[1]; i++) ok = fread(&S.shaders[i], 1, shsize, f) == shsize;
    ok = ok && rdv(f, ld.data(), hdr[2]);
    S.objs.resize(hdr[0]);
    for (uint32_t i = 0; ok && i < hdr[0]; i++) {
        uint32_t oh[4];
        float smooth_angle = 0.f;
        int32_t inst = -1;
        ok = rdv(f, oh, 4) && (hdr[3] < 1 || rdv(f, &smooth_angle, 1)) && (hdr[3] < 4 || rdv(f, &inst, 1));
        if (!ok) break;
        if (inst >= 0) {  // record version 4: a reference, its matrix, and M^-1 when given
            float M[16], inv[16];
            int32_t has_inv = 0;
            ok = rdv(f, M, 16) && rdv(f, &has_inv, 1) && (!has_inv || rdv(f, inv, 16)) && (uint32_t)inst < hdr[0] &&
                 make_instance(S.objs[i], M);
            if (ok && has_inv)
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 4; b++) S.objs[i].back[4 * a + b] = inv[4 * a + b];
            S.objs[i].inst = inst;
            int32_t has_uv = 0, has_orco = 0;  // record versions 6, 7: uv and orco flags (none on a reference)
            if (ok && hdr[3] >= 6) ok = rdv(f, &has_uv, 1);
            if (ok && hdr[3] >= 7) ok = rdv(f, &has_orco, 1) && has_orco == 0;
            continue;
        }
        std::vector<float> v(3 * (size_t)oh[0]);
        std::vector<uint32_t> t(3 * (size_t)oh[1]), ts;
        ok = rdv(f, v.data(), v.size()) && rdv(f, t.data(), t.size());
        if (ok && oh[2] == YR_PER_TRIANGLE) {
            ts.resize(oh[1]);
            ok = rdv(f, ts.data(), ts.size());
        }
        Obj &ob = S.objs[i];
        if (ok && hdr[3] >= 6) {  // record version 6: texture coordinates, 6 per triangle
            int32_t has_uv = 0;
            ok = rdv(f, &has_uv, 1);
            if (ok && has_uv) {
                ob.tri_uv.resize(6 * (size_t)oh[1]);
                ok = rdv(f, ob.tri_uv.data(), ob.tri_uv.size());
            }
        }
        if (ok && hdr[3] >= 7) {  // record version 7: the orco matrix (4x4, rows 0-2 used)
            int32_t has_orco = 0;
            float om[16];
            ok = rdv(f, &has_orco, 1) && (!has_orco || rdv(f, om, 16));
            if (ok && has_orco) {
                ob.has_orco = true;
                for (int k = 0; k < 12; k++) ob.orco[k] = om[k];
            }
        }
        ob.cast = oh[3] != 0;
        for (uint32_t k = 0; ok && k < oh[1]; k++) {
            V a = vtx(v, t[3 * k]), b = vtx(v, t[3 * k + 1]), c = vtx(v, t[3 * k + 2]);
            ob.tri_a.push_back(a);
            ob.tri_b.push_back(b);
            ob.tri_c.push_back(c);
            ob.tri_n.push_back(normalize((b - a) ^ (c - a)));  // triangle.cc:30-43
            ob.tri_shader.push_back(oh[2] == YR_PER_TRIANGLE ? ts[k] : oh[2]);
        }
        if (ok && smooth_angle >= 1.f) auto_smooth(ob, t, oh[0], smooth_angle);
    }
    fclose(f);
    // references take the shadow flag of their original (reference.cc:41)
    for (size_t i = 0; ok && i < S.objs.size(); i++)
        if (S.objs[i].inst >= 0) {
            if (S.objs[S.objs[i].inst].inst >= 0) ok = false;  // no reference to a reference
            else S.objs[i].cast = S.objs[S.objs[i].inst].cast;
        }
    if (!ok) {
        delete o;
        return NULL;
    }
    make_camera(cam, S.cam);
    for (size_t k = 0; k < ld.size(); k++) {
        Light L;
        L.d = ld[k];
        L.samples = ld[k].samples;
        L.color = col3(ld[k].color);
        L.sampdiv = 0;
        const V a(ld[k].p[0][0], ld[k].p[0][1], ld[k].p[0][2]), b(ld[k].p[1][0], ld[k].p[1][1], ld[k].p[1][2]),
            c(ld[k].p[2][0], ld[k].p[2][1], ld[k].p[2][2]), d(ld[k].p[3][0], ld[k].p[3][1], ld[k].p[3][2]);
        if (L.d.type == YR_LIGHT_POINT) {
            L.from = a;
            L.color = L.color * ld[k].power;
        } else if (L.d.type == YR_LIGHT_AREA) {
            // areaLight_t ctor + fillQuad (arealight.cc:31-91)
            const int nsam = ld[k].samples;
            float ab = length(b - a), bc = length(c - b), cd = length(d - c), da = length(a - d);
            float max_v = (bc > da) ? bc : da, max_h = (ab > cd) ? ab : cd;
            int v_samp = (int)((max_v / (max_v + max_h)) * 2.0 * (double)sqrtf((float)nsam));
            int h_samp = (int)((max_h / (max_v + max_h)) * 2.0 * (double)sqrtf((float)nsam));
            if (nsam == 1) {
                L.samples = 1;
            } else {
                V inc_v_a = (d - a) / (float)v_samp, inc_v_b = (c - b) / (float)v_samp;
                V line_a = a + 0.5f * inc_v_a, line_b = b + 0.5f * inc_v_b;
                for (int i = 0; i < v_samp; ++i) {
                    V inc_h = (line_b - line_a) / (float)h_samp;
                    V point = line_a + 0.5f * inc_h;
                    for (int j = 0; j < h_samp; ++j) {
                        float vf = ((float)j) / ((float)h_samp);
                        V inc_v = inc_v_a * (float)(1.0 - vf) + inc_v_b * vf;
                        L.pts.push_back(point);
                        L.jit1.push_back(inc_h);
                        L.jit2.push_back(inc_v);
                        point = point + inc_h;
                    }
                    line_a = line_a + inc_v_a;
                    line_b = line_b + inc_v_b;
                }
                L.samples = (int)L.pts.size();
            }
            L.direction = normalize((b - a) ^ (d - a));
            L.from = (((a + b) + c) + d) * 0.25f;
            L.corner = a;
            L.tox = b - a;
            L.toy = d - a;
        } else if (L.d.type == YR_LIGHT_HEMI) {
            L.sampdiv = ld[k].power / (float)ld[k].samples;
        }
        S.lights.push_back(L);
    }
    memset(&t_st, 0, sizeof(t_st));
    return o;
}

void orc_free(orc_scene *o) { delete o; }

int orc_set_tree(orc_scene *o, uint32_t obj, const yr_kd_node *nodes, uint32_t nnodes, const uint32_t *prims,
                 uint32_t nprims, const float *tree_bound, const float *obj_bound) {
    if (!o || obj >= o->s.objs.size()) return 1;
    Obj &ob = o->s.objs[obj];
    ob.nodes.assign(nodes, nodes + nnodes);
    ob.prims.assign(prims, prims + nprims);
    memcpy(ob.tb.a, tree_bound, 12);
    memcpy(ob.tb.g, tree_bound + 3, 12);
    memcpy(ob.ob.a, obj_bound, 12);
    memcpy(ob.ob.g, obj_bound + 3, 12);
    return 0;
}

// node records: bmin[3], left, bmax[3], right (left < 0: leaf, right = object)
int orc_set_object_tree(orc_scene *o, const float *recs, uint32_t n) {
    o->s.otree.resize(n);
    for (uint32_t i = 0; i < n; i++) {
        const float *r = recs + 8 * (size_t)i;
        ONode &nd = o->s.otree[i];
        memcpy(nd.b.a, r, 12);
        memcpy(&nd.left, r + 3, 4);
        memcpy(nd.b.g, r + 4, 12);
        memcpy(&nd.right, r + 7, 4);
    }
    return 0;
}

// rays: org[3], tmax, dir[3], flags (yr_ray); hits: t, object, triangle, nodes
void orc_trace_closest(orc_scene *o, const float *rays, uint32_t n, uint32_t *hits, int shadow_only) {
    for (uint32_t i = 0; i < n; i++) {
        const float *r = rays + 8 * (size_t)i;
        const V org(r[0], r[1], r[2]), dir(r[4], r[5], r[6]);
        const uint64_t n0 = t_st.nodes;
        Hit h = closest(o->s, org + dir * kMinRay, dir, false, shadow_only != 0);
        float t = h.obj >= 0 ? h.Z : 0.f;
        memcpy(&hits[4 * i], &t, 4);
        hits[4 * i + 1] = h.obj >= 0 ? (uint32_t)h.obj : 0xffffffffu;
        hits[4 * i + 2] = h.obj >= 0 ? h.tri : 0xffffffffu;
        hits[4 * i + 3] = (uint32_t)(t_st.nodes - n0);
    }
}

// shadow rays: p[3], object, l[3], flags (yr_shadow_ray)
void orc_trace_shadow(orc_scene *o, const float *rays, uint32_t n, uint8_t *occ) {
    for (uint32_t i = 0; i < n; i++) {
        const float *r = rays + 8 * (size_t)i;
        int own;
        uint32_t flags;
        memcpy(&own, r + 3, 4);
        memcpy(&flags, r + 7, 4);
        const V p(r[0], r[1], r[2]), l(r[4], r[5], r[6]);
        occ[i] = (flags & 1u) ? shadowed_dir(o->s, p, own, l) : shadowed_point(o->s, p, own, l);
    }
}

// Kd traversal of one object only (kdTree_t::Intersect / IntersectS):
// out: hit, tri, Z bits, nodes visited
void orc_kd(orc_scene *o, uint32_t obj, const float *from, const float *dir, float dist, int any, uint32_t *out) {
    const uint64_t n0 = t_st.nodes;
    uint32_t tr = 0;
    float Z = dist < 0 ? kInf : dist;
    bool h = kd_intersect(o->s, o->s.objs[obj], V(from[0], from[1], from[2]), V(dir[0], dir[1], dir[2]),
                          dist < 0 ? kInf : dist, tr, Z, any != 0);
    out[0] = h;
    out[1] = h ? tr : 0xffffffffu;
    float z = (h && !any) ? Z : 0.f;
    memcpy(&out[2], &z, 4);
    out[3] = (uint32_t)(t_st.nodes - n0);
}

// Render pixels [x0,x1) x [y0,y1) into rgba (full image layout, resx*resy*4).
// stats: primary, shadow, bounce, nodes, tests, slab tests, kd roots tried
// orc_render_ex: the same, taking the other branch of every energy cut-off
// whose value lies within `flip_band` (relative) of the threshold (0: none),
// and writing per pixel the smallest relative distance of any cut-off value
// from the threshold into margin (full image layout, resx*resy; may be NULL).
// Threads may render disjoint regions of one scene at once.
void orc_render_ex(orc_scene *o, float *rgba, int x0, int x1, int y0, int y1, uint64_t *stats, float flip_band,
                   float *margin);

void orc_render(orc_scene *o, float *rgba, int x0, int x1, int y0, int y1, uint64_t *stats) {
    orc_render_ex(o, rgba, x0, x1, y0, y1, stats, 0.f, NULL);
}

void orc_render_ex(orc_scene *o, float *rgba, int x0, int x1, int y0, int y1, uint64_t *stats, float flip_band,
                   float *margin) {
    Scene &S = o->s;
    const uint32_t spp = S.rp.spp ? S.rp.spp : 1;
    memset(&t_st, 0, sizeof(t_st));
    g_stats = &t_st;
    t_flip_band = flip_band;
    for (int y = y0; y < y1; y++)
        for (int x = x0; x < x1; x++) {
            const uint32_t pixel = (uint32_t)(y * S.cam.resx + x);
            t_min_margin = 1e30f;
            float first[4], tot[4] = {0, 0, 0, 0}, c[4];
            for (uint32_t s = 0; s < spp; s++) {
                camera_sample(S, pixel, s, c);
                if (s == 0) memcpy(first, c, 16);
                else
                    for (int k = 0; k < 4; k++) tot[k] += c[k];
            }
            float *px = rgba + 4 * (size_t)pixel;
            if (spp > 1) {
                const float d = (float)(1 + (spp - 1));
                for (int k = 0; k < 4; k++) px[k] = (first[k] + tot[k]) / d;
            } else {
                memcpy(px, first, 16);
            }
            if (S.rp.flags & YR_RENDER_ALPHA_PREMULTIPLY)  // colorA_t::alphaPremultiply
                for (int k = 0; k < 3; k++) px[k] *= px[3];
            if (margin) margin[pixel] = t_min_margin;
        }
    t_flip_band = 0.f;
    if (stats) {
        stats[0] = t_st.primary;
        stats[1] = t_st.shadow;
        stats[2] = t_st.bounce;
        stats[3] = t_st.nodes;
        stats[4] = t_st.tests;
        stats[5] = t_st.boxes;
        stats[6] = t_st.roots;
    }
    g_stats = NULL;
}

// One light's illuminate at the first hit of (from, dir) (scene_t::firstHit,
// scene.cc:688-720), eye point `eye`, QMC sample index m0 at vertex level 0,
// rotation off; an area light takes its 2 values per sample from `vals`.
// Returns whether the ray hit; rgb = the light's contribution.
int orc_illum(orc_scene *o, uint32_t light, const float *eye, const float *from, const float *dir, uint32_t m0,
              const float *vals, float *rgb) {
    Scene &S = o->s;
    rgb[0] = rgb[1] = rgb[2] = 0.f;
    if (light >= S.lights.size()) return -1;
    const V d(dir[0], dir[1], dir[2]);
    const V f = V(from[0], from[1], from[2]) + d * kMinRay;
    Hit h = closest(S, f, d, false, false);
    if (h.obj < 0) return 0;
    SP sp = surface(S, h.obj, h.tri, h.Z, f, d);
    Ctx cx;
    cx.pixel = 0;
    cx.s = m0;
    cx.pi = 0;
    cx.npath = 0;
    const V eyev = V(eye[0], eye[1], eye[2]) - sp.P;
    const Light &L = S.lights[light];
    S.no_rot = true;
    S.area_vals = L.d.type == YR_LIGHT_AREA ? vals : nullptr;
    C c;
    switch (L.d.type) {
    case YR_LIGHT_POINT: c = illum_point(S, L, sp, eyev); break;
    case YR_LIGHT_AREA: c = illum_area(S, (int)light, L, sp, eyev, 0, m0, cx); break;
    case YR_LIGHT_HEMI: c = illum_hemi(S, (int)light, L, sp, eyev, 0, m0, cx); break;
    case YR_LIGHT_PATH: c = illum_path(S, L, sp, eyev, cx); break;
    }
    S.no_rot = false;
    S.area_vals = nullptr;
    rgb[0] = c.r;
    rgb[1] = c.g;
    rgb[2] = c.b;
    return 1;
}

// primary ray directions of pixel centres (camera_t::shootRay)
void orc_camera_rays(orc_scene *o, float *dirs) {
    const Cam &c = o->s.cam;
    for (int y = 0; y < c.resy; y++)
        for (int x = 0; x < c.resx; x++) {
            V d = shoot(c, (float)x + 0.5f, (float)y + 0.5f);
            float *p = dirs + 3 * ((size_t)y * c.resx + x);
            p[0] = d.x;
            p[1] = d.y;
            p[2] = d.z;
        }
}

float orc_halton(uint32_t base, uint32_t n) { return halton(base, n); }
float orc_ri_lp(uint32_t i) { return ri_lp(i); }
float orc_cp_rot(uint32_t seed, uint32_t pixel, uint32_t dim) { return cp_rot(seed, pixel, dim); }
float orc_perlin(float x, float y, float z) { return perlin(V(x, y, z)); }
float orc_noise_gen(uint32_t type, float x, float y, float z) { return noise_gen(type, V(x, y, z)); }
float orc_turbulence_gen(uint32_t type, float x, float y, float z, int oct, float size, int hard) {
    return turbulence_gen(type, V(x, y, z), oct, size, hard != 0);
}
// voronoi_t::getFeatures distances da[0..3] under `metric`
void orc_vor_features(int metric, float mex, float x, float y, float z, float *da) {
    Features F;
    vor_features(V(x, y, z), metric, mex, F);
    for (int k = 0; k < 4; k++) da[k] = F.da[k];
}
// a shader record's texture at texture point (x, y, z): getColor rgb, getFloat
void orc_texture(const yr_shader_desc *d, float x, float y, float z, float *out) {
    const TexVal t = texture_eval(*d, V(x, y, z));
    out[0] = t.col.r;
    out[1] = t.col.g;
    out[2] = t.col.b;
    out[3] = t.f;
}
float orc_fbm(float x, float y, float z, float H, float lac, float oct) { return fbm(V(x, y, z), H, lac, oct); }
float orc_turbulence(float x, float y, float z, int oct, float size, int hard) {
    return turbulence(V(x, y, z), oct, size, hard != 0);
}

}  // extern "C"
