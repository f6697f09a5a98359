// Ray queries on the device: slab test, kd-tree traversal (closest and any
// hit), triangle test, and the front-to-back object-tree iterator.
//
// Each function restates one reference routine; the traversal order, the
// comparisons (strict vs non-strict) and the float expressions are the
// reference's, so a ray visits the same nodes and reports the same triangle
// as kdTree_t::Intersect / IntersectS on the same tree.
#pragma once
#include "dev_common.cuh"

namespace yr {

// A ray with the reciprocals of its direction (1.f/d, correctly rounded,
// which is also kdTree_t::Intersect's invDir: 1.0/d in double narrowed to
// float rounds to the same value).  The exact slab test divides (IEEE) as
// bound_t::cross does; the reciprocals serve the kd split distances and the
// conservative object-tree test.
struct RayR {
    V3 d;
    V3 inv;
};

__device__ __forceinline__ RayR make_rayr(const V3 &d) {
    RayR r;
    r.d = d;
    r.inv = v3(1.f / d.x, 1.f / d.y, 1.f / d.z);
    return r;
}

// bound_t::cross(from, ray, enter, leave, dist) (bound.cc:389-436) as the
// shipped build evaluates it (fast-math: (g - from)/ray instead of
// ((g - a) - (from - a))/ray).
__device__ __forceinline__ bool box_enter_leave(const float *bmin, const float *bmax, const V3 &from,
                                                const RayR &R, float dist, float &enter, float &leave) {
    float lmin = -1.f, lmax = -1.f;
    const V3 &ray = R.d;
    if (ray.x != 0.f) {
        float t1 = (bmin[0] - from.x) / ray.x, t2 = (bmax[0] - from.x) / ray.x;
        if (t1 > t2) { float s = t1; t1 = t2; t2 = s; }
        lmin = t1;
        lmax = t2;
        if ((lmax < 0.f) || (lmin > dist)) return false;
    }
    if (ray.y != 0.f) {
        float t1 = (bmin[1] - from.y) / ray.y, t2 = (bmax[1] - from.y) / ray.y;
        if (t1 > t2) { float s = t1; t1 = t2; t2 = s; }
        if (t1 > lmin) lmin = t1;
        if ((t2 < lmax) || (lmax < 0.f)) lmax = t2;
        if ((lmax < 0.f) || (lmin > dist)) return false;
    }
    if (ray.z != 0.f) {
        float t1 = (bmin[2] - from.z) / ray.z, t2 = (bmax[2] - from.z) / ray.z;
        if (t1 > t2) { float s = t1; t1 = t2; t2 = s; }
        if (t1 > lmin) lmin = t1;
        if ((t2 < lmax) || (lmax < 0.f)) lmax = t2;
    }
    if ((lmin <= lmax) && (lmax >= 0.f) && (lmin <= dist)) {
        enter = lmin;
        leave = lmax;
        return true;
    }
    return false;
}

// bound_t::cross(from, ray, where, dist) (bound.cc:340-387): where = max(enter, 0)
__device__ __forceinline__ bool box_where(const float *bmin, const float *bmax, const V3 &from, const RayR &R,
                                          float dist, float &where) {
    float e, l;
    if (!box_enter_leave(bmin, bmax, from, R, dist, e, l)) return false;
    where = (e > 0.f) ? e : 0.f;
    return true;
}

// A ray prepared for the object-tree walk.  Unless the scene asks for the
// exact order, the walk uses a conservative slab test: per axis the near
// plane's distance is RN(b*y + (nf - e)) and the far plane's RN(b*y + (nf +
// e)), one FMA each, with y = 1/d, nf = RN(-f*y) and e a bound on the
// rounding errors, so that the interval contains the one bound_t::cross
// computes.  Crossing tests then never reject a box that the exact test
// accepts, and entry distances are lower bounds, so pruning by the closest
// hit so far stays safe; only the visiting order of boxes whose entry
// distances agree to within that error can differ (which changes the
// reported object only when two objects are hit at exactly the same
// distance).
struct ObjRay {
    V3 from;
    RayR R;
    float nlo[3];  // RN(RN(-f*y) - e); NaN where y is infinite
    float nhi[3];  // RN(RN(-f*y) + e); NaN where y is infinite
    bool exact;
};

__device__ __forceinline__ ObjRay make_objray(const V3 &from, const RayR &R, float coord_max, bool exact) {
    ObjRay q;
    q.from = from;
    q.R = R;
    q.exact = exact;
    const float f[3] = {from.x, from.y, from.z}, y[3] = {R.inv.x, R.inv.y, R.inv.z};
    const float inf = __int_as_float(0x7f800000), nan = __int_as_float(0x7fffffff);
    for (int k = 0; k < 3; k++) {
        // With b and f bounded by M + |f| in magnitude, bound_t::cross's
        // RN(RN(b - f) / d) is within 2u (M + |f|)|y| of the exact t, and
        // RN(b*y + RN(nf -+ e)) within 2u (M + 2|f|)|y| of t -+ e; e = 2^-20
        // (M + 2|f|)|y| = 16u (M + 2|f|)|y| covers both with a factor of 4
        // to spare.
        const float nf = -f[k] * y[k];
        const float e = (coord_max + 2.f * fabsf(f[k])) * fabsf(y[k]) * 0x1p-20f;
        // An infinite y (d = 0, which bound_t::cross skips, or a subnormal
        // d) gives the axis NaN plane distances, which the fmaxf / fminf
        // below ignore: the axis constrains nothing.  The largest component
        // of a unit direction always has a finite y.
        const bool skip = fabsf(y[k]) == inf;
        q.nlo[k] = skip ? nan : nf - e;
        q.nhi[k] = skip ? nan : nf + e;
    }
    return q;
}

// Conservative crossing test, branch free: the interval is the
// intersection of the widened per-axis intervals.  bound_t::cross's
// running form (lmin / lmax initialised to -1, early exits) accepts
// exactly when max(t_near) <= min(t_far), min(t_far) >= 0 and
// max(t_near) <= dist; widening every interval keeps every such box.
__device__ __forceinline__ bool box_where_obj(const float *bmin, const float *bmax, const ObjRay &q, float dist,
                                              float &where) {
    if (q.exact) return box_where(bmin, bmax, q.from, q.R, dist, where);
    // the near plane is the box's min where y > 0, its max where y < 0
    float n[3], f[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float y = k == 0 ? q.R.inv.x : (k == 1 ? q.R.inv.y : q.R.inv.z);
        const bool ng = y < 0.f;
        n[k] = __fmaf_rn(ng ? bmax[k] : bmin[k], y, q.nlo[k]);
        f[k] = __fmaf_rn(ng ? bmin[k] : bmax[k], y, q.nhi[k]);
    }
    const float lo = fmaxf(fmaxf(n[0], n[1]), n[2]), hi = fminf(fminf(f[0], f[1]), f[2]);
    const bool ok = (lo <= hi) && (hi >= 0.f) && (lo <= dist);
    where = ok ? fmaxf(lo, 0.f) : where;  // untouched on a miss, as box_where
    return ok;
}

struct Tri {
    V3 a, b, c, n;
};

// 3 x 128-bit read-only loads per triangle
__device__ __forceinline__ Tri load_tri(const float4 *tris, uint32_t i) {
    const float4 p = __ldg(tris + 3 * (size_t)i);
    const float4 q = __ldg(tris + 3 * (size_t)i + 1);
    const float4 r = __ldg(tris + 3 * (size_t)i + 2);
    Tri t;
    t.a = v3(p.x, p.y, p.z);
    t.b = v3(q.x, q.y, q.z);
    t.c = v3(r.x, r.y, r.z);
    t.n = v3(p.w, q.w, r.w);
    return t;
}

// triangle_t::hit (triangle.h:48-58): edge signs, no epsilon.  Returns the
// hit distance triangle_t::intersect (triangle.h:83-86) through `t`.
__device__ __forceinline__ bool tri_hit(const Tri &tr, const V3 &from, const V3 &ray, float &t) {
    const V3 va = tr.a - from, vb = tr.b - from, vc = tr.c - from;
    const float rn = dot(ray, tr.n);
    const V3 r = (rn < 0.f) ? -ray : ray;
    if (dot(cross(va, vb), r) < 0.f) return false;
    if (dot(cross(vb, vc), r) < 0.f) return false;
    if (dot(cross(vc, va), r) < 0.f) return false;
    t = dot(tr.n, va) / rn;
    return true;
}

// Per-thread kd stack.  kdTree_t keeps exit points in an array linked by
// `prev` indices and protects the current entry slot (kdtree.cc:606-624,
// 660-676, 720-723); the links always form a last-in first-out chain whose
// head is the current exit, so a plain stack of exits reproduces it: push a
// far child's exit, and on leaving a leaf the head becomes the entry point
// and the next exit is the new head.  The current exit point lives in
// registers; an entry keeps (far node | axis << 30, t) and the split, from
// which the exit point is recomputed exactly as it was first computed.
// Capacity: one entry per level of the deepest tree plus the initial exit.
constexpr int kKdStackCap = 66;

struct KdStack {
    uint2 *nt;     // far node | axis << 30, bits of t
    float *split;
    int cap;       // entries (depth of the deepest tree + 2 must fit)
};

__device__ __forceinline__ void exit_point(uint32_t node_axis, float t, float split, const float *fr,
                                           const float *rr, float *pb) {
    const uint32_t axis = node_axis >> 30;
    if (axis == 3u) {  // initial exit: from + ray*t on every axis
        pb[0] = fr[0] + t * rr[0];
        pb[1] = fr[1] + t * rr[1];
        pb[2] = fr[2] + t * rr[2];
    } else {
        const int ax = (int)axis, na = ax == 2 ? 0 : ax + 1, pa = ax == 0 ? 2 : ax - 1;
        pb[ax] = split;
        pb[na] = fr[na] + t * rr[na];
        pb[pa] = fr[pa] + t * rr[pa];
    }
}

struct KdResult {
    uint32_t tri;
    uint32_t nodes;   // interior + leaf nodes visited
    uint32_t tests;   // triangle tests
};

constexpr uint32_t kNodeMask = 0x3fffffffu;

// kdTree_t::Intersect (kdtree.cc:591-727, ANY=false) and IntersectS
// (kdtree.cc:730-866, ANY=true).  Z is in/out (closest hit only).  Child
// links and leaf contents were checked against the array sizes when the
// scene was created, so the walk follows them unchecked.

__device__ __forceinline__ float sel3(int a, float v0, float v1, float v2) {
    return a == 0 ? v0 : (a == 1 ? v1 : v2);
}

template <bool ANY>
__device__ inline bool kd_trace(const DevScene &S, const DevObject &obj, const V3 &from, const RayR &R, float dist,
                                float &Z, KdResult &res, const KdStack &stk) {
    float a, b;
    if (!box_enter_leave(obj.tb, obj.tb + 3, from, R, dist, a, b)) return false;
    const V3 &ray = R.d;
    const float f0 = from.x, f1 = from.y, f2 = from.z, r0 = ray.x, r1 = ray.y, r2 = ray.z;
    bool hit = false;
    uint32_t curr = obj.root;
    // entry and exit points; a coordinate off the split axis is always
    // from + t*ray, computed for every axis and replaced on the split axis
    float en_t = a, en0, en1, en2;
    if (a >= 0.f) {
        en0 = f0 + a * r0;
        en1 = f1 + a * r1;
        en2 = f2 + a * r2;
    } else {
        en0 = f0;
        en1 = f1;
        en2 = f2;
    }
    float ex_t = b, ex0 = f0 + b * r0, ex1 = f1 + b * r1, ex2 = f2 + b * r2;
    // stack[0] = initial exit (no node); sp = number of exits on the stack
    stk.nt[0] = make_uint2(kNodeMask | (3u << 30), __float_as_uint(b));
    int sp = 1;
    uint32_t leaves = 0;
    while (curr != kNodeMask) {
        if (dist < en_t) break;
        if (++leaves > kMaxLeafVisits) {
            dev_fail(S.status, kDevIterationCap);
            return false;
        }
        uint2 nd = __ldg(S.nodes + curr);
        while ((nd.y & 3u) != 3u) {
            res.nodes++;
            const int axis = (int)(nd.y & 3u);
            const float split = __uint_as_float(nd.x);
            const uint32_t right = nd.y >> 2;
            // both children are fetched before the side is decided, so the
            // next level's load overlaps this level's arithmetic
            const uint2 nl = __ldg(S.nodes + curr + 1), nr = __ldg(S.nodes + right);
            uint32_t far_child;
            if (sel3(axis, en0, en1, en2) <= split) {
                if (sel3(axis, ex0, ex1, ex2) <= split) {
                    curr = curr + 1;
                    nd = nl;
                    continue;
                }
                far_child = right;
                curr = curr + 1;
            } else {
                if (split < sel3(axis, ex0, ex1, ex2)) {
                    curr = right;
                    nd = nr;
                    continue;
                }
                far_child = curr + 1;
                curr = right;
            }
            const float t = (split - sel3(axis, f0, f1, f2)) * sel3(axis, R.inv.x, R.inv.y, R.inv.z);
            if (sp >= stk.cap) {
                dev_fail(S.status, kDevStackOverflow);
                return false;
            }
            stk.nt[sp] = make_uint2(far_child | ((uint32_t)axis << 30), __float_as_uint(t));
            stk.split[sp] = split;
            sp++;
            ex_t = t;
            ex0 = axis == 0 ? split : f0 + t * r0;
            ex1 = axis == 1 ? split : f1 + t * r1;
            ex2 = axis == 2 ? split : f2 + t * r2;
            nd = curr == right ? nr : nl;
        }
        res.nodes++;
        // leaf
        const uint32_t np = nd.y >> 2;
        for (uint32_t k = 0; k < np; k++) {
            const uint32_t ti = (np == 1) ? nd.x : __ldg(S.prims + nd.x + k);
            res.tests++;
            const Tri tr = load_tri(S.tris, ti);
            float rt;
            if (tri_hit(tr, from, ray, rt)) {
                if (ANY) {
                    if (rt < dist && rt > 0.f) {
                        res.tri = ti;
                        return true;
                    }
                } else if (rt < Z && rt >= 0.f) {
                    Z = rt;
                    res.tri = ti;
                    hit = true;
                }
            }
        }
        if (!ANY && hit && Z <= ex_t) return true;
        // the exit point becomes the entry point; descend into its far node
        en_t = ex_t;
        en0 = ex0;
        en1 = ex1;
        en2 = ex2;
        sp--;
        curr = stk.nt[sp].x & kNodeMask;
        if (curr != kNodeMask) {
            const uint2 nx = stk.nt[sp - 1];
            ex_t = __uint_as_float(nx.y);
            const uint32_t ax = nx.x >> 30;  // 3: the initial exit, from + ray*t on every axis
            const float sp_split = stk.split[sp - 1];
            ex0 = ax == 0u ? sp_split : f0 + ex_t * r0;
            ex1 = ax == 1u ? sp_split : f1 + ex_t * r1;
            ex2 = ax == 2u ? sp_split : f2 + ex_t * r2;
        }
    }
    return hit;
}

// geomeIterator_t (geometree.h:36-157) in its front-to-back mode: yields
// objects whose bound the ray crosses before `maximun`, nearest entry first.
struct ObjIter {
    int2 st[kMaxObjStack];   // (node code, bits of the entry distance)  (host checks the tree depth)
    int sp;
    int current;             // object index or -1
    float maximun;
    const float4 *recs;      // interior records of the tree walked
#ifdef YR_COUNT_OBJ
    uint32_t steps = 0;      // interior records loaded (instrumented builds only)
#endif

    __device__ __forceinline__ void down(const DevScene &S, int code, const ObjRay &ray) {
        for (;;) {
            if (code < 0) {
                current = ~code;
                return;
            }
            const float4 *rec = recs + 4 * (size_t)code;
#ifdef YR_COUNT_OBJ
            steps++;
#endif
            const float4 q0 = __ldg(rec), q1 = __ldg(rec + 1), q2 = __ldg(rec + 2), q3 = __ldg(rec + 3);
            const float lmin[3] = {q0.x, q0.y, q0.z}, lmax[3] = {q0.w, q1.x, q1.y};
            const float rmin[3] = {q1.z, q1.w, q2.x}, rmax[3] = {q2.y, q2.z, q2.w};
            float hl = __int_as_float(0x7f800000), hr = __int_as_float(0x7f800000);
            const bool hitl = box_where_obj(lmin, lmax, ray, maximun, hl);
            const bool hitr = box_where_obj(rmin, rmax, ray, maximun, hr);
            if (!hitl && !hitr) {
                if (sp == 0) {
                    current = -1;
                    return;
                }
                code = st[--sp].x;
                continue;
            }
            if (sp >= kMaxObjStack) {
                dev_fail(S.status, kDevStackOverflow);
                current = -1;
                return;
            }
            const int lc = __float_as_int(q3.x), rc = __float_as_int(q3.y);
            if (hl < hr) {
                if (hitr) st[sp++] = make_int2(rc, __float_as_int(hr));
                code = lc;
            } else {
                if (hitl) st[sp++] = make_int2(lc, __float_as_int(hl));
                code = rc;
            }
        }
    }

    // walk the tree given by its records, root box and root code (n = 0: empty)
    __device__ __forceinline__ void start_tree(const DevScene &S, const float4 *r, const float *rootbox, int root,
                                               uint32_t n, const ObjRay &ray, float maxd) {
        maximun = maxd;
        sp = 0;
        current = -1;
        recs = r;
        if (n == 0) return;
        float w = 0.f;
        if (box_where_obj(rootbox, rootbox + 3, ray, maximun, w)) down(S, root, ray);
    }

    // the scene's object tree (geomeTree_t)
    __device__ __forceinline__ void start(const DevScene &S, const ObjRay &ray, float maxd) {
        start_tree(S, S.onodes, S.otb, S.oroot, S.notree, ray, maxd);
    }

    __device__ __forceinline__ void next(const DevScene &S, const ObjRay &ray) {
        current = -1;
        while (sp > 0 && __int_as_float(st[sp - 1].y) > maximun) sp--;
        if (sp > 0) {
            const int node = st[--sp].x;
            down(S, node, ray);
        }
    }

    __device__ __forceinline__ void limit(float z) {
        if (z < maximun) maximun = z;
    }
};

// The casters' BVH walk of a shadow ray: ObjIter's nearest-first descent
// without its pruning by distance, which never applies to a shadow ray
// (the segment's end `dist` stays fixed, and every pushed child was
// crossed before it), so the stack holds node codes only.
struct CasterIter {
    int st[kMaxObjStack];
    int sp;
    int current;             // object index or -1
#ifdef YR_COUNT_OBJ
    uint32_t steps = 0;
#endif

    __device__ __forceinline__ void down(const DevScene &S, int code, const ObjRay &ray, float dist) {
        for (;;) {
            if (code < 0) {
                current = ~code;
                return;
            }
            const float4 *rec = S.sonodes + 4 * (size_t)code;
#ifdef YR_COUNT_OBJ
            steps++;
#endif
            const float4 q0 = __ldg(rec), q1 = __ldg(rec + 1), q2 = __ldg(rec + 2), q3 = __ldg(rec + 3);
            const float lmin[3] = {q0.x, q0.y, q0.z}, lmax[3] = {q0.w, q1.x, q1.y};
            const float rmin[3] = {q1.z, q1.w, q2.x}, rmax[3] = {q2.y, q2.z, q2.w};
            float hl = __int_as_float(0x7f800000), hr = __int_as_float(0x7f800000);
            const bool hitl = box_where_obj(lmin, lmax, ray, dist, hl);
            const bool hitr = box_where_obj(rmin, rmax, ray, dist, hr);
            if (!hitl && !hitr) {
                if (sp == 0) {
                    current = -1;
                    return;
                }
                code = st[--sp];
                continue;
            }
            const int lc = __float_as_int(q3.x), rc = __float_as_int(q3.y);
            if (hitl && hitr) {
                if (sp >= kMaxObjStack) {
                    dev_fail(S.status, kDevStackOverflow);
                    current = -1;
                    return;
                }
                st[sp++] = hl < hr ? rc : lc;
                code = hl < hr ? lc : rc;
            } else {
                code = hitl ? lc : rc;
            }
        }
    }

    __device__ __forceinline__ void start(const DevScene &S, const ObjRay &ray, float dist) {
        sp = 0;
        current = -1;
        if (S.nsotree == 0) return;
        float w = 0.f;
        if (box_where_obj(S.sotb, S.sotb + 3, ray, dist, w)) down(S, S.soroot, ray, dist);
    }

    __device__ __forceinline__ void next(const DevScene &S, const ObjRay &ray, float dist) {
        current = -1;
        if (sp > 0) down(S, st[--sp], ray, dist);
    }
};

// scene_t::isShadowed answered with the shadow-ray tree.  The reference
// shoots each shadow-casting object whose bound the ray crosses, from
// p + dir*self_bias for the point's own object and from p + dir*MIN_RAYDIST
// for the others, and reports whether any kdTree_t::IntersectS finds a
// triangle with 0 < t < dist (scene.cc:107-185, kdtree.cc:730-866).  That
// is a yes/no question about single triangles, so it does not depend on
// the order in which objects or leaves are visited: here one traversal of
// the merged tree covers the segment that both origins can reach (from the
// earlier origin, up to dist plus the gap between the two offsets), and
// each triangle is tested from its own object's origin with the same
// triangle_t::hit / intersect arithmetic - the answer is bit-identical.
__device__ inline bool scene_occluded_merged(const DevScene &S, const V3 &p, int own, const V3 &dir, float dist,
                                             float self_bias, const KdStack &stk, uint32_t &nodes_out,
                                             uint32_t &tests_out) {
    const V3 self = p + dir * self_bias;
    const V3 p2 = p + dir * kMinRayDist;
    const bool self_first = self_bias < kMinRayDist;
    const V3 q = self_first ? self : p2;
    const float tdist = (dist + fabsf(self_bias - kMinRayDist)) * 1.000001f + 1e-6f;
    const RayR R = make_rayr(dir);
    float a, b;
    if (!box_enter_leave(S.sh_tb, S.sh_tb + 3, q, R, tdist, a, b)) return false;
    const V3 &ray = R.d;
    const float inv[3] = {R.inv.x, R.inv.y, R.inv.z};
    const float fr[3] = {q.x, q.y, q.z};
    const float rr[3] = {ray.x, ray.y, ray.z};
    uint32_t curr = 0;
    float en_t = a, en_pb[3];
    if (a >= 0.f) {
        en_pb[0] = fr[0] + a * rr[0];
        en_pb[1] = fr[1] + a * rr[1];
        en_pb[2] = fr[2] + a * rr[2];
    } else {
        en_pb[0] = fr[0];
        en_pb[1] = fr[1];
        en_pb[2] = fr[2];
    }
    float ex_pb[3];
    ex_pb[0] = fr[0] + b * rr[0];
    ex_pb[1] = fr[1] + b * rr[1];
    ex_pb[2] = fr[2] + b * rr[2];
    float ex_t = b;
    stk.nt[0] = make_uint2(kNodeMask | (3u << 30), __float_as_uint(b));
    int sp = 1;
    uint32_t leaves = 0, nodes = 0, tests = 0;
    bool occluded = false;
    while (curr != kNodeMask) {
        if (tdist < en_t) break;
        if (++leaves > kMaxLeafVisits) {
            dev_fail(S.status, kDevIterationCap);
            break;
        }
        if (curr >= S.sh_nnodes) {
            dev_fail(S.status, kDevBadTree);
            break;
        }
        uint2 nd = __ldg(S.sh_nodes + curr);
        bool bad = false;
        while ((nd.y & 3u) != 3u) {
            nodes++;
            const int axis = (int)(nd.y & 3u);
            const float split = __uint_as_float(nd.x);
            const uint32_t right = nd.y >> 2;
            uint32_t far_child;
            if (curr + 1 >= S.sh_nnodes || right >= S.sh_nnodes) {
                bad = true;
                break;
            }
            if (en_pb[axis] <= split) {
                if (ex_pb[axis] <= split) {
                    curr = curr + 1;
                    nd = __ldg(S.sh_nodes + curr);
                    continue;
                }
                far_child = right;
                curr = curr + 1;
            } else {
                if (split < ex_pb[axis]) {
                    curr = right;
                    nd = __ldg(S.sh_nodes + curr);
                    continue;
                }
                far_child = curr + 1;
                curr = right;
            }
            const float t = (split - fr[axis]) * inv[axis];
            if (sp >= stk.cap) {
                bad = true;
                break;
            }
            stk.nt[sp] = make_uint2(far_child | ((uint32_t)axis << 30), __float_as_uint(t));
            stk.split[sp] = split;
            sp++;
            const int na = axis == 2 ? 0 : axis + 1, pa = axis == 0 ? 2 : axis - 1;
            ex_t = t;
            ex_pb[axis] = split;
            ex_pb[na] = fr[na] + t * rr[na];
            ex_pb[pa] = fr[pa] + t * rr[pa];
            nd = __ldg(S.sh_nodes + curr);
        }
        if (bad) {
            dev_fail(S.status, sp >= stk.cap ? kDevStackOverflow : kDevBadTree);
            break;
        }
        nodes++;
        const uint32_t np = nd.y >> 2;
        for (uint32_t k = 0; k < np; k++) {
            const uint32_t ti = (np == 1) ? nd.x : __ldg(S.sh_prims + nd.x + k);
            if (ti >= S.ntris) {
                bad = true;
                break;
            }
            tests++;
            const Tri tr = load_tri(S.tris, ti);
            const int obj = (int)__ldg(S.tri_obj + ti);
            float rt;
            if (tri_hit(tr, obj == own ? self : p2, ray, rt) && rt < dist && rt > 0.f) {
                // the reference shoots an object only when the ray from p2
                // crosses its bound before dist (geometree.h:86-135); the
                // enclosing object-tree boxes then pass too (same ray, larger
                // boxes, monotonic slab arithmetic)
                const DevObject &ob = S.objects[obj];
                float w;
                if (box_where(ob.ob, ob.ob + 3, p2, R, dist, w)) {
                    occluded = true;
                    break;
                }
            }
        }
        if (bad) {
            dev_fail(S.status, kDevBadTree);
            break;
        }
        if (occluded) break;
        en_t = ex_t;
        en_pb[0] = ex_pb[0];
        en_pb[1] = ex_pb[1];
        en_pb[2] = ex_pb[2];
        sp--;
        curr = stk.nt[sp].x & kNodeMask;
        if (curr != kNodeMask) {
            const uint2 nx = stk.nt[sp - 1];
            ex_t = __uint_as_float(nx.y);
            exit_point(nx.x, ex_t, stk.split[sp - 1], fr, rr, ex_pb);
        }
    }
    nodes_out += nodes;
    tests_out += tests;
    return occluded;
}

struct SceneHit {
    float t;
    int object;       // -1 = miss
    uint32_t tri;     // global triangle index
    uint32_t nodes;
    uint32_t tests;
};

// object3d_t::shoot with shadow = true: the any-hit walk of the object's
// tree; a reference (referenceObject_t::shoot, reference.cc:95-114) walks its
// original's tree with origin and direction taken into the original's space
// by M's inverse (not renormalised, so the distances stay the world's)
template <bool INST>
__device__ __forceinline__ bool shoot_any(const DevScene &S, const DevObject &obj, const V3 &from, const RayR &ray,
                                          float dist, float &Z, KdResult &r, const KdStack &stk) {
    if (!INST) return kd_trace<true>(S, obj, from, ray, dist, Z, r, stk);
    V3 f = from;
    RayR rr = ray;
    if (obj.inst >= 0) {
        const DevInst &I = S.insts[obj.inst];
        f = xf_point(I.back, from);
        rr = make_rayr(xf_vec(I.back, ray.d));
    }
    return kd_trace<true>(S, obj, f, rr, dist, Z, r, stk);
}

// Closest hit over all objects.  `f` is the already offset origin.
//   pass_limit = true : scene_t::raytrace (scene.cc:210-233) - each object
//                       is shot with the current closest distance
//   pass_limit = false: scene_t::firstHit (scene.cc:688-707)
//   shadow_only: skip objects that do not cast shadows (firstHit's shadow arg)
template <bool INST>
__device__ inline SceneHit scene_closest_t(const DevScene &S, const V3 &f, const V3 &dir, bool pass_limit,
                                           bool shadow_only, const KdStack &stk) {
    const RayR ray = make_rayr(dir);
    const ObjRay oray = make_objray(f, ray, S.coord_max, S.exact_order != 0);
    SceneHit best;
    best.t = 0.f;
    best.object = -1;
    best.tri = kNone;
    best.nodes = 0;
    best.tests = 0;
    const float inf = __int_as_float(0x7f800000);
    float limit = inf;
    ObjIter it;
    it.start(S, oray, inf);
    while (it.current >= 0) {
        const int o = it.current;
        const DevObject &obj = S.objects[o];
        if (!(shadow_only && !(obj.flags & 1u))) {
            const float dis = pass_limit ? limit : inf;
            float Z = dis;
            KdResult r{kNone, 0, 0};
            bool h;
            if (!INST) {
                h = kd_trace<false>(S, obj, f, ray, dis, Z, r, stk);
            } else {
                V3 fo = f;
                RayR ro = ray;
                if (obj.inst >= 0) {  // referenceObject_t::shoot: the ray in the original's space
                    const DevInst &I = S.insts[obj.inst];
                    fo = xf_point(I.back, f);
                    ro = make_rayr(xf_vec(I.back, dir));
                }
                h = kd_trace<false>(S, obj, fo, ro, dis, Z, r, stk);
            }
            best.nodes += r.nodes;
            best.tests += r.tests;
            if (h && Z > 0.f) {
                if (pass_limit) limit = Z;
                it.limit(Z);
                if (best.object < 0 || Z < best.t) {
                    best.t = Z;
                    best.object = o;
                    best.tri = r.tri;
                }
            }
        }
        it.next(S, oray);
    }
    return best;
}

__device__ inline SceneHit scene_closest(const DevScene &S, const V3 &f, const V3 &dir, bool pass_limit,
                                         bool shadow_only, const KdStack &stk) {
    if (S.insts) return scene_closest_t<true>(S, f, dir, pass_limit, shadow_only, stk);
    return scene_closest_t<false>(S, f, dir, pass_limit, shadow_only, stk);
}

// scene_t::isShadowed (scene.cc:107-185).  p: shading point, own: its
// object, ray: unit direction, dist: |l - p| (or infinity).
template <bool INST>
__device__ inline bool scene_occluded_ref(const DevScene &S, const V3 &p, int own, const V3 &dir, float dist,
                                          float self_bias, const KdStack &stk, uint32_t &nodes, uint32_t &tests) {
    const V3 self = p + dir * self_bias;
    const V3 p2 = p + dir * kMinRayDist;
    const RayR ray = make_rayr(dir);
    const ObjRay oray = make_objray(p2, ray, S.coord_max, S.exact_order != 0);
    ObjIter it;
    it.start(S, oray, dist);
    while (it.current >= 0) {
        const int o = it.current;
        const DevObject &obj = S.objects[o];
        if (obj.flags & 1u) {
            float Z = dist;
            KdResult r{kNone, 0, 0};
            const bool h = shoot_any<INST>(S, obj, (o == own) ? self : p2, ray, dist, Z, r, stk);
#ifdef YR_COUNT_OBJ
            tests += 1;  // objects shot
            if (h) {
                nodes += it.steps;
                return true;
            }
#else
            nodes += r.nodes;
            tests += r.tests;
            if (h) return true;
#endif
        }
        it.next(S, oray);
    }
#ifdef YR_COUNT_OBJ
    nodes += it.steps;
#endif
    return false;
}

// scene_t::isShadowed with the objects found through the SAH BVH over the
// shadow casters.  The reference's answer is whether some casting object o
// has (a) a bound that the ray from p2 crosses before dist (the object tree
// reaches o exactly then: every enclosing box is larger, the slab
// arithmetic is monotonic) and (b) an IntersectS hit from its origin.  The
// BVH's conservative walk reaches every object with (a) (and possibly a
// few more); (b) is the same kd walk; (a) is checked exactly for an
// object with a hit before it counts.  The answer is therefore the
// reference's, whatever the order in which objects are reached.
template <bool INST>
__device__ inline bool scene_occluded_bvh(const DevScene &S, const V3 &p, int own, const V3 &dir, float dist,
                                          float self_bias, const KdStack &stk, uint32_t &nodes, uint32_t &tests) {
    const V3 self = p + dir * self_bias;
    const V3 p2 = p + dir * kMinRayDist;
    const RayR ray = make_rayr(dir);
    const ObjRay oray = make_objray(p2, ray, S.coord_max, false);
    CasterIter it;
    it.start(S, oray, dist);
    while (it.current >= 0) {
        const int o = it.current;
        const DevObject &obj = S.objects[o];
        float Z = dist;
        KdResult r{kNone, 0, 0};
        const bool h = shoot_any<INST>(S, obj, (o == own) ? self : p2, ray, dist, Z, r, stk);
#ifdef YR_COUNT_OBJ
        tests += 1;  // objects shot
#else
        nodes += r.nodes;
        tests += r.tests;
#endif
        if (h) {
            float w;
            if (box_where(obj.ob, obj.ob + 3, p2, ray, dist, w)) {
#ifdef YR_COUNT_OBJ
                nodes += it.steps;
#endif
                return true;
            }
        }
        it.next(S, oray, dist);
    }
#ifdef YR_COUNT_OBJ
    nodes += it.steps;
#endif
    return false;
}

// isShadowed through the shadow-ray tree, through the object tree in the
// reference's order when the scene asks for exact order, else through the
// shadow casters' BVH (yr_render_params.flags)
template <bool INST>
__device__ inline bool scene_occluded_t(const DevScene &S, const V3 &p, int own, const V3 &dir, float dist,
                                        float self_bias, const KdStack &stk, uint32_t &nodes, uint32_t &tests) {
    if (S.use_sh_tree) {
        if (S.sh_nnodes == 0) return false;  // nothing casts shadows
        return scene_occluded_merged(S, p, own, dir, dist, self_bias, stk, nodes, tests);
    }
    if (S.exact_order) return scene_occluded_ref<INST>(S, p, own, dir, dist, self_bias, stk, nodes, tests);
    return scene_occluded_bvh<INST>(S, p, own, dir, dist, self_bias, stk, nodes, tests);
}

// the same, choosing the loops with or without references at run time
// (kernels on the render path are instantiated for each instead)
__device__ inline bool scene_occluded(const DevScene &S, const V3 &p, int own, const V3 &dir, float dist,
                                      float self_bias, const KdStack &stk, uint32_t &nodes, uint32_t &tests) {
    if (S.insts) return scene_occluded_t<true>(S, p, own, dir, dist, self_bias, stk, nodes, tests);
    return scene_occluded_t<false>(S, p, own, dir, dist, self_bias, stk, nodes, tests);
}

}  // namespace yr
