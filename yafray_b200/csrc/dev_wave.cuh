// Wavefront stages shared by the per-scene renderer (render.cu) and the
// batched persistent renderer (batch.cu).
#pragma once
#include <algorithm>
#include <cstring>
#include <mutex>

#include "dev_shade.cuh"
#include "dev_trace.cuh"
#include "scene.h"

namespace yr {

constexpr int kBlock = 128;
#ifndef YR_DYN_FETCH
#define YR_DYN_FETCH 1  // traversal kernels take 32-ray chunks from a counter instead of a fixed stride
#endif
#ifndef YR_TRACE_GRID_PERSIST
#define YR_TRACE_GRID_PERSIST 1  // traversal grids: one block per resident slot of every SM
#endif
#ifndef YR_SHADE_MINB
#define YR_SHADE_MINB 6  // minimum resident blocks per SM for the shading kernels (80 registers)
#endif
#ifndef YR_TRACE_MINB
#define YR_TRACE_MINB 10  // minimum resident blocks per SM for the traversal kernels (48 registers)
#endif

enum SlotFlag : uint8_t { kSlotNone = 0, kSlotLit = 1, kSlotShadowed = 2, kSlotPending = 3 };

struct Wave {
    uint32_t base;       // first camera sample (pixel*spp + s) of the wave
    uint32_t count;      // camera samples in the wave
    uint32_t ns;         // shadow slots per vertex
    uint32_t nv;         // vertices the slot arrays hold (slot s of vertex v at s*nv + v)
    uint32_t npath;      // path samples per camera sample (0: no path light)
    // per camera sample
    float4 *hit0;        // t, object, triangle, (ray count)
    float4 *lterm;       // [count * nlights] per-light terms (rgb)
    float4 *aux;         // [count * nlights] area: plane_at; hemi: fromLight(fake)
    float4 *diff0;       // path light: getDiffuse(sp)*power factor and validity
    // per path (count * npath)
    float4 *p_where;     // origin of the next bounce (xyz), startray.N (w)
    float4 *p_ray;       // direction (xyz), alive flag (w)
    float4 *p_col;       // raycolor (xyz)
    float4 *p_next;      // pending raycolor after the vertex (xyz)
    float4 *p_nray;      // pending direction
    float4 *p_hit;       // bounce hit: t, object, triangle
    float4 *p_contri;    // [count * npath * depth] contributions (rgb)
    float4 *p_aux;       // [count * npath * nlights]
    // slots and queues
    float4 *slot_c;      // [max(count, count*npath) * ns] contribution if lit
    uint8_t *slot_f;     // flags
    float4 *shq0;        // shadow queue: p.xyz, own object
    float4 *shq1;        // dir.xyz, dist
    uint32_t *shq_slot;
    uint32_t *bq;        // bounce queue (path indices)
    uint32_t *bq2;
    uint32_t *sq;        // [count * npath] the bounce queue in shading order: hits first, then misses
    uint32_t part;       // 1: the bounce walk writes sq and the path shading takes its order
    float4 *ptot;        // [count] path light: the rounds' sum of path contributions (adaptive rounds)
    uint32_t *nrep;      // [count] path light: extra rounds of the camera sample
    uint32_t rep;        // the round of paths being traced (0 = the first)
    uint32_t *counters;  // [16]: [0] shadow queue, [1] bounce queue, [2] next bounce queue,
                         // [3..5] ray totals (primary, shadow, bounce) as 2x u32 lo/hi pairs,
                         // [6] / [7] traversal fetch counters, [8] empty shadow-queue places,
                         // [9] / [10] hits / misses placed in sq
    unsigned long long *rays;  // [3] primary, shadow, bounce
    unsigned long long *kst;   // [YR_K_COUNT][3]: rays, nodes, tests per kernel class
    float *out;          // RGBA image (device)
};

// Slot s of vertex v.  Slots are stored sample-major, so that the lanes of
// a warp (consecutive vertices) write and read one slot of neighbouring
// vertices at neighbouring addresses.
__host__ __device__ __forceinline__ uint32_t slot_of(const Wave &W, uint32_t v, uint32_t s) { return s * W.nv + v; }

// Extra per-wave state of the adjoint recompute (yr_backward).
struct AdjWave {
    float4 *slot_s;        // [slots] specular factor per light sample (slot_c: diffuse factor)
    float4 *v0;            // [count] camera vertex: diffuse colour, shader (bits)
    float4 *v0m;           // [2*count] camera vertex texture: (d colour / d intensity, d colour / d color1), (colour, 0)
    float4 *pv;            // [count*npath*depth] path vertex: diffuse colour, shader (bits); w = -1: none
    float4 *pm;            // [2*count*npath*depth] path vertex texture, as v0m
    float4 *pG;            // [count*npath*depth] direct light (or background) at the vertex; w = 1: present
    const float4 *gpix;    // per image pixel: dL/d(pixel rgb)
    float *grad;           // parameter gradient (global)
    const int *sh_pbase;   // first parameter of each shader
    const int *li_pidx;    // parameter of each light (its power)
    const float4 *spec_dir;// unit specular direction of each shader
    uint32_t nparams;
};

// warp-reduced traversal counters, one atomic per warp (all lanes must call)
__device__ __forceinline__ void count_work(const Wave &W, int cls, uint32_t rays, uint32_t nodes, uint32_t tests) {
    const uint32_t r = __reduce_add_sync(0xffffffffu, rays);
    const uint32_t n = __reduce_add_sync(0xffffffffu, nodes);
    const uint32_t t = __reduce_add_sync(0xffffffffu, tests);
    if ((threadIdx.x & 31) == 0 && r) {
        atomicAdd(&W.kst[3 * cls + 0], (unsigned long long)r);
        atomicAdd(&W.kst[3 * cls + 1], (unsigned long long)n);
        atomicAdd(&W.kst[3 * cls + 2], (unsigned long long)t);
    }
}

// camera sample cs -> image pixel (row-major index) inside the region
__device__ __forceinline__ uint32_t cs_pixel(const DevRender &R, uint32_t cs, int &x, int &y) {
    const uint32_t lp = cs / R.spp;
    x = R.rx0 + (int)(lp % (uint32_t)R.rw);
    y = R.ry0 + (int)(lp / (uint32_t)R.rw);
    return (uint32_t)y * (uint32_t)R.cam.resx + (uint32_t)x;
}

// QMC index of path pi of camera sample s (s = sample within its pixel) in
// the current round of paths: (round * spp + s) * P + pi
__device__ __forceinline__ uint32_t path_index(const DevRender &R, const Wave &W, uint32_t s, uint32_t pi) {
    return (W.rep * R.spp + s) * W.npath + pi;
}

// ---------------------------------------------------------------- camera
// state.screenpos of a camera sample at pixel (x, y), sub-pixel (fx, fy),
// given to its camera hit (scene.cc:234, 749-750, 798-799)
__device__ __forceinline__ void screen_pos(const DevRender &R, int x, int y, float fx, float fy, Surf &sp) {
    sp.sx = (float)(2.0 * (double)(((float)x + fx) / (float)R.cam.resx) - 1.0);
    sp.sy = (float)(1.0 - 2.0 * (double)(((float)y + fy) / (float)R.cam.resy));
}

// camera_t::shootRay, CM_PERSPECTIVE (camera.cc:184-188)
__device__ __forceinline__ V3 camera_ray(const DevCamera &c, float px, float py) {
    return normalize(c.vto + (c.vright * px + c.vup * py));
}

// sub-pixel position of camera sample s (scene.cc:741-799 with all pixels
// resampled in one AA pass of spp-1 samples)
__device__ __forceinline__ void sample_pos(const DevRender &R, uint32_t pixel, uint32_t s, float &fx, float &fy) {
    if (s == 0) {
        fx = 0.5f;
        fy = 0.5f;
        return;
    }
    const uint32_t c = s - 1;
    // RI_LP (mcqmc.h:73-78)
    uint32_t r = 0, i = c + pixel;
    for (uint32_t v = 1u << 31; i; i >>= 1, v |= v >> 1)
        if (i & 1) r ^= v;
    const float lp = (float)((double)r / 4294967296.0);
    // the float terms are promoted by the double literals 0.5
    fx = (float)(0.5 + (double)R.pw * ((double)lp - 0.5));
    fy = (float)(0.5 + (double)R.pw * ((double)((float)c * R.totsamdiv) - 0.5));
}

// ------------------------------------------------------------ warp append
__device__ __forceinline__ uint32_t warp_append(uint32_t *counter, bool pred) {
    const unsigned mask = __activemask();
    const unsigned ball = __ballot_sync(mask, pred);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader && ball) base = atomicAdd(counter, (uint32_t)__popc(ball));
    base = __shfl_sync(mask, base, leader);
    return base + (uint32_t)__popc(ball & ((1u << lane) - 1u));
}

// A shadow-queue entry without a ray (a reserved place that its lane did
// not fill): the traversal skips it and the ray count leaves it out.
constexpr uint32_t kNoSlot = 0xffffffffu;

__device__ __forceinline__ void put_shadow(const Wave &W, uint32_t q, const V3 &p, int own, const V3 &dir,
                                           float dist, uint32_t slot) {
    W.shq0[q] = make_float4(p.x, p.y, p.z, __int_as_float(own));
    W.shq1[q] = make_float4(dir.x, dir.y, dir.z, dist);
    W.shq_slot[q] = slot;
}

__device__ __forceinline__ void emit_shadow(const Wave &W, bool pred, const V3 &p, int own, const V3 &dir,
                                            float dist, uint32_t slot) {
    const uint32_t q = warp_append(&W.counters[0], pred);
    if (pred) put_shadow(W, q, p, own, dir, dist, slot);
}

// One shadow-queue reservation per warp for one light's `n` sample rays:
// every lane that samples the light takes n places, and the warp pays one
// atomic instead of n.  The places are arranged for the walk, whose warps
// take the queue 32 places at a time:
//   at camera hits, sample-major (sample j of the r-th such lane at
//   j*nw + r): the warp's lanes are neighbouring camera samples, so 32
//   places are rays from nearly one point into one cell of the light's
//   sample grid;
//   at path vertices, lane-major (at r*n + j): the lanes are unrelated
//   paths, so 32 places are the rays of one or two points.
// A sample that turns out to need no ray leaves its place empty (kNoSlot);
// the empty places are counted for the ray totals.  Whole warp.
struct WarpPlaces {
    unsigned mask;
    uint32_t base, nw, rank, holes, n;
    int lane, leader;
    bool sampling, lane_major;
    __device__ __forceinline__ WarpPlaces(const Wave &W, bool s, uint32_t n_, bool path_vertex)
        : holes(0), n(n_), sampling(s), lane_major(path_vertex) {
        mask = __activemask();
        const unsigned ball = __ballot_sync(mask, s);
        lane = threadIdx.x & 31;
        leader = __ffs(mask) - 1;
        nw = (uint32_t)__popc(ball);
        rank = (uint32_t)__popc(ball & ((1u << lane) - 1u));
        base = 0;
        if (lane == leader && nw) base = atomicAdd(&W.counters[0], nw * n);
        base = __shfl_sync(mask, base, leader);
    }
    // sample j's ray (emit) or its empty place
    __device__ __forceinline__ void put(const Wave &W, uint32_t j, bool emit, const V3 &p, int own, const V3 &dir,
                                        float dist, uint32_t slot) {
        if (!sampling) return;
        const uint32_t q = lane_major ? base + rank * n + j : base + j * nw + rank;
        if (emit) {
            put_shadow(W, q, p, own, dir, dist, slot);
        } else {
            W.shq_slot[q] = kNoSlot;
            holes++;
        }
    }
    __device__ __forceinline__ void finish(const Wave &W) {
        const uint32_t h = __reduce_add_sync(mask, holes);
        if (lane == leader && h) atomicAdd(&W.counters[8], h);
    }
};

// --------------------------------------------------------------- kernels
// Stage bodies.  Each wavefront kernel runs one stage over the whole wave;
// the batched persistent kernel runs the same stages over one tile inside
// a block.  Stages marked "whole warp" must be called by all 32 lanes.
// INST: the scene has references (instanced objects); the traversal loops
// that transform rays are compiled only into those instantiations.
template <bool INST>
__device__ __forceinline__ void st_primary(const DevScene &S, const DevRender &R, const Wave &W, uint32_t i,
                                           const KdStack &stk, uint32_t &nodes, uint32_t &tests) {
    {
        const uint32_t cs = W.base + i;
        int x, y;
        const uint32_t pixel = cs_pixel(R, cs, x, y), s = cs % R.spp;
        float fx, fy;
        sample_pos(R, pixel, s, fx, fy);
        const V3 ray = camera_ray(R.cam, (float)x + fx, (float)y + fy);
        const V3 f = R.cam.pos + ray * kMinRayDist;  // scene.cc:211
        const SceneHit h = scene_closest_t<INST>(S, f, ray, true, false, stk);
        W.hit0[i] = make_float4(h.t, __int_as_float(h.object), __uint_as_float(h.tri), 0.f);
        nodes += h.nodes;
        tests += h.tests;
    }
}

#ifdef YR_WAVE_KERNELS
template <bool INST>
static __global__ void __launch_bounds__(kBlock, YR_TRACE_MINB) k_primary(DevScene S, DevRender R, Wave W) {
    uint2 stk_nt[kKdStackCap];
    float stk_split[kKdStackCap];
    const KdStack stk{stk_nt, stk_split, kKdStackCap};
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t nodes = 0, tests = 0;
    if (i < W.count) st_primary<INST>(S, R, W, i, stk, nodes, tests);
    count_work(W, YR_K_PRIMARY, i < W.count ? 1u : 0u, nodes, tests);
}
#endif

// sample slots of a light at one vertex (a point light's one, an area or
// hemi light's samples); the penumbra guess's probe slots come after all
__device__ __forceinline__ uint32_t light_slots(const DevLight &L) {
    if (L.type == YR_LIGHT_POINT) return 1;
    if (L.type == YR_LIGHT_AREA || L.type == YR_LIGHT_HEMI) return (uint32_t)L.samples;
    return 0;
}

// Grid point of probe j of the penumbra guess (areaLight_t::guessLight,
// arealight.cc:176-198, which draws rand() % samples): floor(samples * u),
// u = halton(5, m0*psamples + j) rotated like the light's first dimension.
__device__ __forceinline__ int guess_point(const DevLight &L, uint32_t m0, int j, float r0) {
    const float u = cp_add(halton(5, m0 * (uint32_t)L.psamples + (uint32_t)j), r0);
    const int rs = (int)(u * (float)L.samples);
    return rs < L.samples ? rs : L.samples - 1;
}

enum GuessStatus { kGuessShadow = 0, kGuessPenumbra = 1, kGuessLight = 2 };

// per-light sampling at one shading vertex; writes slots, aux and queue
// entries.  vtx = vertex index for slots/aux, v = QMC vertex level,
// m0 = QMC sample index of this vertex.
// Area lights with a penumbra guess (psamples > 0) take two stages:
// stage 0 queues the guess's probe rays (and does every other light);
// stage 1, once the probes are answered, decides each guess light
// (guessLight's order, with its early stop once light and shadow were
// both seen) and queues the light's sample rays in penumbra, or counts every
// grid point lit without a shadow ray, or none in shadow.
// ADJ (adjoint recompute): slot_c / slot_s receive the diffuse and specular
// factors per unit light power instead of the light sample's colour, hemi
// aux holds (diffuse factor, specular factor, 0, go), and the vertex's
// diffuse colour and noise value are returned.
template <bool ADJ = false>
__device__ __forceinline__ void shade_lights(const DevScene &S, const DevRender &R, const Wave &W, bool active,
                                             const Surf &sp, const V3 &eye, uint32_t vtx, int v, uint32_t m0,
                                             uint32_t pixel, float4 *aux, float4 *slot_s = nullptr,
                                             C3 *lkc_out = nullptr, TexDeriv *td_out = nullptr, int stage = 0) {
    DevShader sh;
    C3 lkc = c3(0.f, 0.f, 0.f);
    if (active) {
        sh = R.shaders[sp.shader];
        if (!ADJ && (sh.mod_spec > 0.f || sh.mod_hard > 0.f)) {
            // the modulator also sets this point's specular colour and
            // Phong exponent (fromLight, basicshaders.cc:55-62)
            modulated_all(R.shaders + sp.shader, sp, eye, lkc, sh.specular, sh.hard);
        } else {
            lkc = modulated_color(R.shaders + sp.shader, sp, eye, ADJ ? td_out : nullptr);
        }
        if (ADJ) *lkc_out = lkc;
    }
    V3 N = sp.N;
    LitPre pre;
    if (active) {
        pre = lit_pre(sh, sp, eye);
        N = pre.N;  // FACE_FORWARD(Ng, N, normalize(eye)), as fromLight forms it
    }
    uint32_t off = 0;
    for (int k = 0; k < R.nlights; k++) {
        const DevLight L = R.lights[k];
        const bool guess = !ADJ && L.type == YR_LIGHT_AREA && L.psamples > 0;
        if (stage == 1 && !guess) {  // the second stage handles the guessing lights only
            off += light_slots(L);
            continue;
        }
        if (L.type == YR_LIGHT_POINT) {
            const uint32_t slot = slot_of(W, vtx, off);
            bool emit = false;
            V3 rdir;
            float dist = 0.f;
            if (active) {
                // pointLight_t::illuminate (pointlight.cc:27-46)
                const V3 Lv = L.from - sp.P;
                const V3 dir = normalize(Lv);
                float id2 = dot(Lv, Lv);
                if (id2 != 0.f) id2 = 1.f / id2;
                if (ADJ) {
                    C3 D, Sp;
                    from_light_parts(sh, pre, dir, L.rawc * id2, D, Sp);
                    W.slot_c[slot] = make_float4(D.r, D.g, D.b, 0.f);
                    slot_s[slot] = make_float4(Sp.r, Sp.g, Sp.b, 0.f);
                } else {
                    const C3 c = from_light(sh, lkc, pre, dir, L.color * id2);
                    W.slot_c[slot] = make_float4(c.r, c.g, c.b, 0.f);
                }
                if (L.cast) {
                    // isShadowed(sp, from): ray = l - p, dist = |l - p|
                    rdir = L.from - sp.P;
                    dist = length(rdir);
                    rdir = normalize(rdir);
                    emit = true;
                    W.slot_f[slot] = kSlotPending;
                } else {
                    W.slot_f[slot] = kSlotLit;
                }
            }
            emit_shadow(W, emit, sp.P, sp.object, rdir, dist, slot);
            off += 1;
        } else if (L.type == YR_LIGHT_AREA) {
            // areaLight_t::illuminate (arealight.cc:93-174): the penumbra
            // branch with explicit QMC jitter; with psamples > 0 the guess
            // (arealight.cc:176-198) decides it first
            float plane_at = 0.f;
            bool lit_side = false;
            if (active) {
                plane_at = dot(sp.P - L.from, L.direction);
                lit_side = plane_at > 0.f;
                if (stage == 0) aux[vtx * R.nlights + k] = make_float4(plane_at, lit_side ? 1.f : 0.f, 0.f, 0.f);
            }
            const uint32_t d = light_dim(k, v);
            const float r0 = cp_rot(R.seed, pixel, d), r1 = cp_rot(R.seed, pixel, d + 1);
            if (guess && stage == 0) {
                // the guess's probes: unjittered grid points; a point behind
                // the surface counts as shadow without a ray (an empty place)
                WarpPlaces wp(W, active && lit_side, (uint32_t)L.psamples, v > 0);
                for (int j = 0; j < L.psamples; j++) {
                    const uint32_t slot = slot_of(W, vtx, (uint32_t)L.probe_off + (uint32_t)j);
                    bool emit = false;
                    V3 rdir;
                    float dist = 0.f;
                    if (active) {
                        W.slot_f[slot] = kSlotNone;
                        if (lit_side) {
                            const float *pt = R.area_pts + 9 * (size_t)(L.pt_base + guess_point(L, m0, j, r0));
                            const V3 gp = v3(pt[0], pt[1], pt[2]);
                            if (dot(gp - sp.P, N) < 0.f) {
                                W.slot_f[slot] = kSlotShadowed;
                            } else {
                                rdir = gp - sp.P;
                                dist = length(rdir);
                                rdir = normalize(rdir);
                                emit = true;
                                W.slot_f[slot] = kSlotPending;
                            }
                        }
                    }
                    wp.put(W, (uint32_t)j, emit, sp.P, sp.object, rdir, dist, slot);
                }
                wp.finish(W);
                if (active)
                    for (int jj = 0; jj < L.samples; jj++) W.slot_f[slot_of(W, vtx, off + (uint32_t)jj)] = kSlotNone;
                off += (uint32_t)L.samples;
                continue;
            }
            int status = kGuessPenumbra;
            if (guess && active && lit_side) {
                bool luz = false, sombra = false;
                int decided = -1;
                for (int j = 0; j < L.psamples; j++) {
                    if (luz && sombra) {
                        decided = kGuessPenumbra;
                        break;
                    }
                    if (W.slot_f[slot_of(W, vtx, (uint32_t)L.probe_off + (uint32_t)j)] == kSlotLit) luz = true;
                    else sombra = true;
                }
                status = decided >= 0 ? decided : ((luz && sombra) ? kGuessPenumbra : (luz ? kGuessLight : kGuessShadow));
            }
            // the light's sample rays in one reservation per warp; a sample
            // behind the point's tangent plane leaves its place empty
            WarpPlaces wp(W, active && lit_side && status == kGuessPenumbra, (uint32_t)L.samples, v > 0);
            for (int jj = 0; jj < L.samples; jj++) {
                const uint32_t slot = slot_of(W, vtx, off + (uint32_t)jj);
                bool emit = false;
                V3 rdir;
                float dist = 0.f;
                if (active && status == kGuessLight) {
                    // every grid point, unjittered, no shadow test (arealight.cc:156-166)
                    const float *pt = R.area_pts + 9 * (size_t)(L.pt_base + jj);
                    V3 dir = v3(pt[0], pt[1], pt[2]) - sp.P;
                    float ld2 = norm_len_sqr(dir);
                    ld2 = (ld2 != 0.f) ? (1.f / ld2) : 1.f;
                    const C3 c = from_light(sh, lkc, pre, dir, (L.power * L.color) * ld2);
                    W.slot_c[slot] = make_float4(c.r, c.g, c.b, 0.f);
                    W.slot_f[slot] = kSlotLit;
                } else if (active) {
                    W.slot_f[slot] = kSlotNone;
                    if (lit_side && status == kGuessPenumbra) {
                        const uint32_t m = m0 * (uint32_t)L.samples + (uint32_t)jj;
                        const float h2 = cp_add(halton(2, m), r0), h3 = cp_add(halton(3, m), r1);
                        V3 sampleP;
                        if (L.samples == 1) {
                            sampleP = (L.corner + L.tox * h2) + L.toy * h3;
                        } else {
                            const float dish = h2 - 0.5f, disv = h3 - 0.5f;
                            const float *pt = R.area_pts + 9 * (size_t)(L.pt_base + jj);
                            sampleP = (v3(pt[0], pt[1], pt[2]) + v3(pt[3], pt[4], pt[5]) * dish) +
                                      v3(pt[6], pt[7], pt[8]) * disv;
                        }
                        V3 Lv = sampleP - sp.P;
                        if (!(dot(Lv, N) < 0.f)) {
                            V3 dir = Lv;
                            float ld2 = norm_len_sqr(dir);
                            ld2 = (ld2 != 0.f) ? (1.f / ld2) : 1.f;
                            if (ADJ) {
                                C3 D, Sp;
                                from_light_parts(sh, pre, dir, L.color * ld2, D, Sp);
                                W.slot_c[slot] = make_float4(D.r, D.g, D.b, 0.f);
                                slot_s[slot] = make_float4(Sp.r, Sp.g, Sp.b, 0.f);
                            } else {
                                const C3 c = from_light(sh, lkc, pre, dir, (L.power * L.color) * ld2);
                                W.slot_c[slot] = make_float4(c.r, c.g, c.b, 0.f);
                            }
                            W.slot_f[slot] = kSlotPending;
                            rdir = sampleP - sp.P;
                            dist = length(rdir);
                            rdir = normalize(rdir);
                            emit = true;
                        }
                    }
                }
                wp.put(W, (uint32_t)jj, emit, sp.P, sp.object, rdir, dist, slot);
            }
            wp.finish(W);
            off += (uint32_t)L.samples;
        } else if (L.type == YR_LIGHT_HEMI) {
            // hemiLight_t::illuminate (hemilight.cc:58-100), QMC
            bool go = false;
            C3 fl = c3(0.f, 0.f, 0.f);
            V3 Nh = sp.N;
            if (active) {
                Nh = face_forward(sp.Ng, sp.N, eye);
                fl = from_light(sh, lkc, pre, Nh, c3(1.f, 1.f, 1.f));
                const float mad = fmaxf(fabsf(fl.r), fmaxf(fabsf(fl.g), fabsf(fl.b)));
                go = !(mad < 0.05f);
                if (ADJ) {
                    C3 D, Sp;
                    from_light_parts(sh, pre, Nh, c3(1.f, 1.f, 1.f), D, Sp);
                    aux[vtx * R.nlights + k] = make_float4(D.r, Sp.r, 0.f, go ? 1.f : 0.f);
                } else {
                    aux[vtx * R.nlights + k] = make_float4(fl.r, fl.g, fl.b, go ? 1.f : 0.f);
                }
            }
            const uint32_t d = light_dim(k, v);
            const float r0 = cp_rot(R.seed, pixel, d), r1 = cp_rot(R.seed, pixel, d + 1);
            // one reservation per warp; a direction below the horizon leaves
            // its place empty
            WarpPlaces wp(W, active && go, (uint32_t)L.samples, v > 0);
            for (int jj = 0; jj < L.samples; jj++) {
                const uint32_t slot = slot_of(W, vtx, off + (uint32_t)jj);
                bool emit = false;
                V3 rdir;
                float dist = 0.f;
                if (active) {
                    W.slot_f[slot] = kSlotNone;
                    if (go) {
                        const uint32_t m = m0 * (uint32_t)L.samples + (uint32_t)jj;
                        const float z1 = cp_add(halton(2, m), r0), z2 = cp_add(halton(3, m), r1);
                        const V3 dir = uni_hemi_dir(Nh, sp.NU, sp.NV, z1, z2);
                        const float occ = dot(dir, Nh);
                        if (occ > 0.f) {
                            const C3 c = L.color * occ;
                            W.slot_c[slot] = make_float4(c.r, c.g, c.b, 0.f);
                            W.slot_f[slot] = kSlotPending;
                            if (L.maxdist > 0.f) {
                                rdir = (sp.P + L.maxdist * dir) - sp.P;
                                dist = length(rdir);
                                rdir = normalize(rdir);
                            } else {
                                rdir = normalize(dir);
                                dist = __int_as_float(0x7f800000);
                            }
                            emit = true;
                        }
                    }
                }
                wp.put(W, (uint32_t)jj, emit, sp.P, sp.object, rdir, dist, slot);
            }
            wp.finish(W);
            off += (uint32_t)L.samples;
        }
    }
}

// light terms of one vertex from its slots, in light order (scene.cc:267-272)
__device__ __forceinline__ C3 gather_term(const DevRender &R, const Wave &W, const DevLight &L, int k, uint32_t vtx,
                                          uint32_t off, const float4 *aux) {
    if (L.type == YR_LIGHT_POINT) {
        const uint32_t slot = slot_of(W, vtx, off);
        if (W.slot_f[slot] == kSlotLit) {
            const float4 c = W.slot_c[slot];
            return c3(c.x, c.y, c.z);
        }
        return c3(0.f, 0.f, 0.f);
    }
    if (L.type == YR_LIGHT_AREA) {
        const float4 a = aux[vtx * R.nlights + k];
        if (a.y == 0.f) return c3(0.f, 0.f, 0.f);
        C3 resul = c3(0.f, 0.f, 0.f);
        for (int jj = 0; jj < L.samples; jj++) {
            const uint32_t slot = slot_of(W, vtx, off + (uint32_t)jj);
            if (W.slot_f[slot] == kSlotLit) {
                const float4 c = W.slot_c[slot];
                resul = resul + c3(c.x, c.y, c.z);
            }
        }
        return (a.x * resul) / (float)L.samples;
    }
    if (L.type == YR_LIGHT_HEMI) {
        const float4 a = aux[vtx * R.nlights + k];
        if (a.w == 0.f) return c3(0.f, 0.f, 0.f);
        C3 total = c3(0.f, 0.f, 0.f);
        for (int jj = 0; jj < L.samples; jj++) {
            const uint32_t slot = slot_of(W, vtx, off + (uint32_t)jj);
            if (W.slot_f[slot] == kSlotLit) {
                const float4 c = W.slot_c[slot];
                total = total + c3(c.x, c.y, c.z);
            }
        }
        return (L.sampdiv * total) * c3(a.x, a.y, a.z);
    }
    return c3(0.f, 0.f, 0.f);
}

// whole warp
template <bool ADJ = false>
__device__ __forceinline__ void st_shade_camera(const DevScene &S, const DevRender &R, const Wave &W, uint32_t i,
                                                const AdjWave *A = nullptr) {
    const bool inb = i < W.count;
    const uint32_t cs = W.base + (inb ? i : 0);
    int x, y;
    const uint32_t pixel = cs_pixel(R, cs, x, y), s = cs % R.spp;
    bool active = false;
    Surf sp;
    V3 eye = v3(0.f, 0.f, 0.f);
    if (inb) {
        const float4 h = W.hit0[i];
        const int obj = __float_as_int(h.y);
        if (obj >= 0) {
            float fx, fy;
            sample_pos(R, pixel, s, fx, fy);
            const V3 ray = camera_ray(R.cam, (float)x + fx, (float)y + fy);
            const V3 f = R.cam.pos + ray * kMinRayDist;
            sp = make_surface(S, R, obj, __float_as_uint(h.z), h.x, f, ray);
            screen_pos(R, x, y, fx, fy, sp);
            eye = R.cam.pos - sp.P;  // scene_t::light: eye = from - sp.P()
            active = true;
        }
    }
    if (ADJ) {
        C3 lkc = c3(0.f, 0.f, 0.f);
        TexDeriv td{};
        shade_lights<true>(S, R, W, active, sp, eye, inb ? i : 0, 0, s, pixel, W.aux, A->slot_s, &lkc, &td);
        if (active) {
            A->v0[i] = make_float4(lkc.r, lkc.g, lkc.b, __int_as_float(sp.shader));
            A->v0m[2 * (size_t)i] = make_float4(td.dint.r, td.dint.g, td.dint.b, td.dc1);
            A->v0m[2 * (size_t)i + 1] = make_float4(td.tex.r, td.tex.g, td.tex.b, 0.f);
        }
    } else {
        shade_lights(S, R, W, active, sp, eye, inb ? i : 0, 0, s, pixel, W.aux);
    }
    if (!inb || R.path_light < 0) return;
    // pathLight_t::normalSample (pathlight.cc:389-403) + the first
    // directions of takeSample (pathlight.cc:305-312)
    bool paths = false;
    if (active) {
        const C3 dif = modulated_color(R.shaders + sp.shader, sp, eye);  // getDiffuse(sp, eye)
        paths = !(energy(dif) < 0.05f);
        const DevLight PL = R.lights[R.path_light];
        W.diff0[i] = make_float4(dif.r, dif.g, dif.b, paths ? PL.power : 0.f);
        if (paths) {
            const V3 N0 = face_forward(sp.Ng, sp.N, eye);
            const float r0 = cp_rot(R.seed, pixel, 0), r1 = cp_rot(R.seed, pixel, 1);
            for (uint32_t pi = 0; pi < W.npath; pi++) {
                const uint32_t n = path_index(R, W, s, pi);
                const float z1 = cp_add(halton(kPrimes[0], n), r0), z2 = cp_add(halton(kPrimes[1], n), r1);
                const V3 ray = cos_hemi_dir(N0, sp.NU, sp.NV, z1, z2);
                const uint32_t p = i * W.npath + pi;
                W.p_where[p] = make_float4(sp.P.x, sp.P.y, sp.P.z, dot(ray, N0));
                W.p_ray[p] = make_float4(ray.x, ray.y, ray.z, 1.f);
                W.p_col[p] = make_float4(1.f, 1.f, 1.f, 0.f);
            }
        }
    } else {
        W.diff0[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    // queue the paths (in path order within a warp)
    for (uint32_t pi = 0; pi < W.npath; pi++) {
        const uint32_t q = warp_append(&W.counters[1], paths);
        if (paths) W.bq[q] = i * W.npath + pi;
    }
}

#ifdef YR_WAVE_KERNELS
static __global__ void __launch_bounds__(kBlock, YR_SHADE_MINB) k_shade_camera(DevScene S, DevRender R, Wave W) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W.count && (i & ~31u) >= W.count) return;  // whole warps past the end leave
    st_shade_camera(S, R, W, i);
}
#endif

// one queued shadow ray; false for a place without a ray (kNoSlot).  BVH:
// the scene uses the casters' BVH (neither the shadow-ray tree nor the
// exact order), so the kernel holds that walk alone
template <bool INST, bool BVH = false>
__device__ __forceinline__ bool st_trace_shadow(const DevScene &S, const Wave &W, uint32_t q, float self_bias,
                                                const KdStack &stk, uint32_t &nodes, uint32_t &tests) {
    const uint32_t slot = W.shq_slot[q];
    if (slot == kNoSlot) return false;
    const float4 a = W.shq0[q], b = W.shq1[q];
    const V3 p = v3(a.x, a.y, a.z), l = v3(b.x, b.y, b.z);
    const int own = __float_as_int(a.w);
    const bool occ = BVH ? scene_occluded_bvh<INST>(S, p, own, l, b.w, self_bias, stk, nodes, tests)
                         : scene_occluded_t<INST>(S, p, own, l, b.w, self_bias, stk, nodes, tests);
    W.slot_f[slot] = occ ? kSlotShadowed : kSlotLit;
    return true;
}

#ifdef YR_WAVE_KERNELS
template <bool INST, bool BVH>
static __global__ void __launch_bounds__(kBlock, YR_TRACE_MINB) k_trace_shadow_q(DevScene S, Wave W, float self_bias) {
    uint2 stk_nt[kKdStackCap];
    float stk_split[kKdStackCap];
    const KdStack stk{stk_nt, stk_split, kKdStackCap};
    const uint32_t n = W.counters[0];
    uint32_t rays = 0, nodes = 0, tests = 0;
#if YR_DYN_FETCH
    // each warp takes the next 32 queue entries until the queue is done, so
    // warps that drew short rays take more of them (counters[6] starts at 0)
    for (;;) {
        uint32_t base = 0;
        if ((threadIdx.x & 31u) == 0) base = atomicAdd(&W.counters[6], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const uint32_t q = base + (threadIdx.x & 31u);
        if (q < n && st_trace_shadow<INST, BVH>(S, W, q, self_bias, stk, nodes, tests)) rays++;
    }
#else
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        if (st_trace_shadow<INST, BVH>(S, W, q, self_bias, stk, nodes, tests)) rays++;
#endif
    count_work(W, YR_K_SHADOW, rays, nodes, tests);
}
#endif

__device__ __forceinline__ void st_gather_camera(const DevRender &R, const Wave &W, uint32_t i) {
    const float4 h = W.hit0[i];
    const bool hit = __float_as_int(h.y) >= 0;
    uint32_t off = 0;
    for (int k = 0; k < R.nlights; k++) {
        const DevLight L = R.lights[k];
        C3 t = c3(0.f, 0.f, 0.f);
        if (hit && L.type != YR_LIGHT_PATH) t = gather_term(R, W, L, k, i, off, W.aux);
        W.lterm[(size_t)i * R.nlights + k] = make_float4(t.r, t.g, t.b, 0.f);
        off += light_slots(L);
    }
}

#ifdef YR_WAVE_KERNELS
static __global__ void __launch_bounds__(kBlock) k_gather_camera(DevRender R, Wave W) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < W.count) st_gather_camera(R, W, i);
}
#endif

template <bool INST>
__device__ __forceinline__ void st_trace_bounce(const DevScene &S, const Wave &W, uint32_t q, const KdStack &stk,
                                                uint32_t &nodes, uint32_t &tests) {
    const uint32_t p = W.bq[q];
    const float4 wh = W.p_where[p], rr = W.p_ray[p];
    const V3 ray = v3(rr.x, rr.y, rr.z);
    const V3 f = v3(wh.x, wh.y, wh.z) + ray * kMinRayDist;  // scene.cc:693
    const SceneHit h = scene_closest_t<INST>(S, f, ray, false, true, stk);
    W.p_hit[p] = make_float4(h.t, __int_as_float(h.object), __uint_as_float(h.tri), 0.f);
    nodes += h.nodes;
    tests += h.tests;
}

#ifdef YR_WAVE_KERNELS
template <bool INST>
static __global__ void __launch_bounds__(kBlock, YR_TRACE_MINB) k_trace_bounce(DevScene S, Wave W) {
    uint2 stk_nt[kKdStackCap];
    float stk_split[kKdStackCap];
    const KdStack stk{stk_nt, stk_split, kKdStackCap};
    const uint32_t n = W.counters[1];
    uint32_t rays = 0, nodes = 0, tests = 0;
#if YR_DYN_FETCH
    for (;;) {  // as k_trace_shadow_q, on counters[7]
        uint32_t base = 0;
        if ((threadIdx.x & 31u) == 0) base = atomicAdd(&W.counters[7], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const uint32_t q = base + (threadIdx.x & 31u);
        bool hit = false;
        if (q < n) {
            st_trace_bounce<INST>(S, W, q, stk, nodes, tests);
            hit = __float_as_int(W.p_hit[W.bq[q]].y) >= 0;
            rays++;
        }
        if (W.part) {
            // the shading order: hits from the front, misses from the
            // back, so that a shading warp takes paths of one kind and its
            // light reservations hold full warps of points (whole warp)
            const uint32_t ph = warp_append(&W.counters[9], q < n && hit);
            const uint32_t pm = warp_append(&W.counters[10], q < n && !hit);
            if (q < n) W.sq[hit ? ph : n - 1u - pm] = W.bq[q];
        }
    }
#else
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        st_trace_bounce<INST>(S, W, q, stk, nodes, tests);
        rays++;
    }
#endif
    count_work(W, YR_K_BOUNCE, rays, nodes, tests);
}
#endif

// shading at bounce vertex j (pathlight.cc:313-346): light samples, next
// direction and pending raycolor
// whole warp; q indexes the bounce queue (lanes past its end are inactive)
template <bool ADJ = false>
__device__ __forceinline__ void st_shade_path(const DevScene &S, const DevRender &R, const Wave &W, int j,
                                              uint32_t q, uint32_t n, const AdjWave *A = nullptr) {
    const bool inq = q < n;
    const uint32_t p = inq ? (W.part ? W.sq[q] : W.bq[q]) : 0;
    const uint32_t i = p / W.npath, pi = p % W.npath;
    const uint32_t cs = W.base + i;
    int px_x, px_y;
    const uint32_t pixel = cs_pixel(R, cs, px_x, px_y), s = cs % R.spp;
    bool active = false;
    Surf sp;
    V3 eye = v3(0.f, 0.f, 0.f), ray = v3(0.f, 0.f, 1.f);
    if (inq) {
        const float4 h = W.p_hit[p];
        const int obj = __float_as_int(h.y);
        const float4 wh = W.p_where[p], rr = W.p_ray[p];
        ray = v3(rr.x, rr.y, rr.z);
        if (obj >= 0) {
            const V3 f = v3(wh.x, wh.y, wh.z) + ray * kMinRayDist;
            sp = make_surface(S, R, obj, __float_as_uint(h.z), h.x, f, ray);
            // getLight: scene_t::light(state, sp, sp.P()+eye, true) with
            // eye = -ray, and light() forms eye = from - sp.P() (scene.cc:264)
            eye = (sp.P + (-ray)) - sp.P;
            active = true;
        }
    }
    C3 dif = c3(0.f, 0.f, 0.f);
    if (ADJ) {
        TexDeriv td{};
        shade_lights<true>(S, R, W, active, sp, eye, p, j + 1, path_index(R, W, s, pi), pixel, W.p_aux, A->slot_s, &dif,
                           &td);
        if (active) {
            const size_t ci = (size_t)p * R.path_depth + j;
            A->pv[ci] = make_float4(dif.r, dif.g, dif.b, __int_as_float(sp.shader));
            A->pm[2 * ci] = make_float4(td.dint.r, td.dint.g, td.dint.b, td.dc1);
            A->pm[2 * ci + 1] = make_float4(td.tex.r, td.tex.g, td.tex.b, 0.f);
        }
    } else {
        shade_lights(S, R, W, active, sp, eye, p, j + 1, path_index(R, W, s, pi), pixel, W.p_aux);
    }
    if (active) {
        if (!ADJ) dif = modulated_color(R.shaders + sp.shader, sp, -ray);  // getDiffuse(tempsp, -ray)
        const float4 col = W.p_col[p];
        const C3 nc = c3(col.x, col.y, col.z) * dif;
        W.p_next[p] = make_float4(nc.r, nc.g, nc.b, 0.f);
        const V3 HN = face_forward(sp.Ng, sp.N, -ray);
        const int lev = j + 1;
        if (j + 1 < R.path_depth) {
            const float r0 = cp_rot(R.seed, pixel, 2 * lev), r1 = cp_rot(R.seed, pixel, 2 * lev + 1);
            const uint32_t nidx = path_index(R, W, s, pi);
            const float z1 = cp_add(halton(kPrimes[2 * lev], nidx), r0);
            const float z2 = cp_add(halton(kPrimes[2 * lev + 1], nidx), r1);
            const V3 nr = cos_hemi_dir(HN, sp.NU, sp.NV, z1, z2);
            W.p_nray[p] = make_float4(nr.x, nr.y, nr.z, 0.f);
        }
        // with a penumbra guess the guess stage needs the bounce origin
        // still: it moves the path there itself
        if (!R.has_guess) W.p_where[p] = make_float4(sp.P.x, sp.P.y, sp.P.z, W.p_where[p].w);
    }
}

// The penumbra guess's second stage at the camera vertex of sample i (whole
// warp): the vertex is set up again as st_shade_camera does, and the
// guessing area lights are decided from their answered probes.
__device__ __forceinline__ void st_guess_camera(const DevScene &S, const DevRender &R, const Wave &W, uint32_t i) {
    const bool inb = i < W.count;
    const uint32_t cs = W.base + (inb ? i : 0);
    int x, y;
    const uint32_t pixel = cs_pixel(R, cs, x, y), s = cs % R.spp;
    bool active = false;
    Surf sp;
    V3 eye = v3(0.f, 0.f, 0.f);
    if (inb) {
        const float4 h = W.hit0[i];
        const int obj = __float_as_int(h.y);
        if (obj >= 0) {
            float fx, fy;
            sample_pos(R, pixel, s, fx, fy);
            const V3 ray = camera_ray(R.cam, (float)x + fx, (float)y + fy);
            const V3 f = R.cam.pos + ray * kMinRayDist;
            sp = make_surface(S, R, obj, __float_as_uint(h.z), h.x, f, ray);
            screen_pos(R, x, y, fx, fy, sp);
            eye = R.cam.pos - sp.P;
            active = true;
        }
    }
    shade_lights(S, R, W, active, sp, eye, inb ? i : 0, 0, s, pixel, W.aux, nullptr, nullptr, nullptr, 1);
}

// The same at path vertex j (bounce queue entry q, whole warp); it then
// moves the path to the vertex, as st_shade_path does without a guess.
__device__ __forceinline__ void st_guess_path(const DevScene &S, const DevRender &R, const Wave &W, int j, uint32_t q,
                                              uint32_t n) {
    const bool inq = q < n;
    const uint32_t p = inq ? W.bq[q] : 0;
    const uint32_t i = p / W.npath, pi = p % W.npath;
    const uint32_t cs = W.base + i;
    int px_x, px_y;
    const uint32_t pixel = cs_pixel(R, cs, px_x, px_y), s = cs % R.spp;
    bool active = false;
    Surf sp;
    V3 eye = v3(0.f, 0.f, 0.f);
    float4 wh = make_float4(0.f, 0.f, 0.f, 0.f);
    if (inq) {
        const float4 h = W.p_hit[p];
        const int obj = __float_as_int(h.y);
        wh = W.p_where[p];
        const float4 rr = W.p_ray[p];
        const V3 ray = v3(rr.x, rr.y, rr.z);
        if (obj >= 0) {
            const V3 f = v3(wh.x, wh.y, wh.z) + ray * kMinRayDist;
            sp = make_surface(S, R, obj, __float_as_uint(h.z), h.x, f, ray);
            eye = (sp.P + (-ray)) - sp.P;
            active = true;
        }
    }
    shade_lights(S, R, W, active, sp, eye, p, j + 1, path_index(R, W, s, pi), pixel, W.p_aux, nullptr, nullptr, nullptr,
                 1);
    if (active) W.p_where[p] = make_float4(sp.P.x, sp.P.y, sp.P.z, wh.w);
}

#ifdef YR_WAVE_KERNELS
static __global__ void __launch_bounds__(kBlock, YR_SHADE_MINB) k_guess_camera(DevScene S, DevRender R, Wave W) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W.count && (i & ~31u) >= W.count) return;  // whole warps past the end leave
    st_guess_camera(S, R, W, i);
}

static __global__ void __launch_bounds__(kBlock, YR_SHADE_MINB) k_guess_path(DevScene S, DevRender R, Wave W, int j) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = W.counters[1];
    if (q >= n && (q & ~31u) >= n) return;
    st_guess_path(S, R, W, j, q, n);
}

static __global__ void __launch_bounds__(kBlock, YR_SHADE_MINB) k_shade_path(DevScene S, DevRender R, Wave W, int j) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = W.counters[1];
    if (q >= n && (q & ~31u) >= n) return;
    st_shade_path(S, R, W, j, q, n);
}
#endif

// whole warp
__device__ __forceinline__ void st_gather_path(const DevRender &R, const Wave &W, int j, const C3 &bg, uint32_t q,
                                               uint32_t n) {
    const bool inq = q < n;
    const uint32_t p = inq ? W.bq[q] : 0;
    bool requeue = false;
    if (inq) {
        const float4 h = W.p_hit[p];
        const float4 col = W.p_col[p];
        const float startN = W.p_where[p].w;
        const C3 rc = c3(col.x, col.y, col.z);
        C3 contri;
        const size_t ci = ((size_t)p * R.path_depth + j);
        if (__float_as_int(h.y) < 0) {
            // background reached (pathlight.cc:318-324)
            contri = (startN * rc) * bg;
        } else {
            C3 light = c3(0.f, 0.f, 0.f);
            uint32_t off = 0;
            for (int k = 0; k < R.nlights; k++) {
                const DevLight L = R.lights[k];
                if (L.type != YR_LIGHT_PATH) light = light + gather_term(R, W, L, k, p, off, W.p_aux);
                off += light_slots(L);
            }
            contri = (startN * rc) * light;
            const float4 nc = W.p_next[p];
            const C3 ncol = c3(nc.x, nc.y, nc.z);
            W.p_col[p] = make_float4(ncol.r, ncol.g, ncol.b, 0.f);
            if (j + 1 < R.path_depth && !(energy(ncol) < 0.05f)) {
                const float4 nr = W.p_nray[p];
                W.p_ray[p] = make_float4(nr.x, nr.y, nr.z, 1.f);
                requeue = true;
            }
        }
        W.p_contri[ci] = make_float4(contri.r, contri.g, contri.b, 1.f);
    }
    const uint32_t nq = warp_append(&W.counters[2], requeue);
    if (requeue) W.bq2[nq] = p;
}

#ifdef YR_WAVE_KERNELS
static __global__ void __launch_bounds__(kBlock) k_gather_path(DevRender R, Wave W, int j, C3 bg) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = W.counters[1];
    if (q >= n && (q & ~31u) >= n) return;
    st_gather_path(R, W, j, bg, q, n);
}
#endif

// color_t::expgam_Adjust (color.h:175-195) in the shipped build's form:
// with exposure e != 0, x = 1 - exp(e*max(x,0)) (the product in float, exp in
// double); with gamma_R != 1, x = pow(max(x,0), gamma_R) in double; with
// neither, clamp to [0,1] when clamp_rgb.
__device__ __forceinline__ C3 expgam_adjust(const C3 &c, float e, float g, bool clamp_rgb) {
    float v[3] = {c.r, c.g, c.b};
    if (e == 0.0f && g == 1.0f) {
        if (clamp_rgb)
#pragma unroll
            for (int k = 0; k < 3; k++) v[k] = fmaxf(fminf(v[k], 1.0f), 0.0f);
        return c3(v[0], v[1], v[2]);
    }
    if (e != 0.0f)
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = (float)(1.0 - exp((double)(e * fmaxf(v[k], 0.0f))));
    if (g != 1.0f)
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = (float)pow((double)fmaxf(v[k], 0.0f), (double)g);
    return c3(v[0], v[1], v[2]);
}

// one pixel of the wave: AA average of its camera samples
__device__ __forceinline__ void st_finish(const DevRender &R, const Wave &W, uint32_t px) {
    float4 first = make_float4(0.f, 0.f, 0.f, 0.f), tot = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t s = 0; s < R.spp; s++) {
        const uint32_t i = px * R.spp + s;
        const float4 h = W.hit0[i];
        const bool hit = __float_as_int(h.y) >= 0;
        C3 col;
        if (hit) {
            C3 fl = c3(0.f, 0.f, 0.f);
            for (int k = 0; k < R.nlights; k++) {
                if (k == R.path_light) {
                    // normalSample: getDiffuse * (total * multiplier) * power
                    const float4 d0 = W.diff0[i];
                    C3 pt = c3(0.f, 0.f, 0.f);
                    if (d0.w != 0.f) {
                        C3 total = c3(0.f, 0.f, 0.f);
                        float rounds = 1.0f;
                        if (R.path_threshold > 0.f) {  // the rounds' sum, formed round by round
                            const float4 t = W.ptot[i];
                            total = c3(t.x, t.y, t.z);
                            rounds = (float)(1u + W.nrep[i]);
                        } else {
                            for (uint32_t pi = 0; pi < W.npath; pi++)
                                for (int j = 0; j < R.path_depth; j++) {
                                    const float4 c = W.p_contri[((size_t)(i * W.npath + pi)) * R.path_depth + j];
                                    if (c.w == 0.f) break;
                                    total = total + c3(c.x, c.y, c.z);
                                }
                        }
                        // multiplier() = 1/(taken+1), divided by the rounds taken
                        const float mult = (float)(1.0 / (double)(float)W.npath);
                        total = total * (mult / rounds);
                        pt = (c3(d0.x, d0.y, d0.z) * total) * d0.w;
                    }
                    fl = fl + pt;
                } else {
                    const float4 t = W.lterm[(size_t)i * R.nlights + k];
                    fl = fl + c3(t.x, t.y, t.z);
                }
            }
            col = fl;
        } else {
            col = R.background;
        }
        if (R.tonemap) col = expgam_adjust(col, R.exposure, R.gamma_r, R.clamp_rgb != 0);
        const float4 c4 = make_float4(col.r, col.g, col.b, hit ? 1.f : 0.f);
        if (s == 0) {
            first = c4;
        } else {
            tot.x += c4.x;
            tot.y += c4.y;
            tot.z += c4.z;
            tot.w += c4.w;
        }
    }
    float4 o = first;
    if (R.spp > 1) {
        // (mf*img + totcol) / (mf + totnumsam) with mf = 1 (scene.cc:810-812)
        const float d = (float)(1 + (R.spp - 1));
        o = make_float4((first.x + tot.x) / d, (first.y + tot.y) / d, (first.z + tot.z) / d, (first.w + tot.w) / d);
    }
    if (R.premultiply) o = make_float4(o.x * o.w, o.y * o.w, o.z * o.w, o.w);  // colorA_t::alphaPremultiply
    int x, y;
    const uint32_t pixel = cs_pixel(R, W.base + px * R.spp, x, y);
    reinterpret_cast<float4 *>(W.out)[pixel] = o;
}

// The path light's adaptive rounds (pathLight_t::takeSample,
// pathlight.cc:349-374), per camera sample i once round W.rep of its paths
// is gathered.  Round 0: the contributions summed in the reference's order
// (path by path, vertex by vertex) and, per partial sum i % 4, the extra
// rounds: the sums times multiplier() = 1/P, their per-channel minimum and
// maximum after the scene's tone adjustment (scene_t::adjustColor),
// diff = maxAbsDiff(max, min) / (max(ene, 1) * 4) / threshold with
// ene = maxAbsDiff(min, 0), extra = int(diff^2) - 1 in [0, 3].  Later
// rounds: their contributions added in the same order.
__device__ __forceinline__ void st_path_round(const DevRender &R, const Wave &W, uint32_t i) {
    if (W.diff0[i].w == 0.f) return;  // no paths from this point
    if (W.rep > 0 && W.nrep[i] < W.rep) return;
    C3 total = c3(0.f, 0.f, 0.f), sub[4];
    for (int k = 0; k < 4; k++) sub[k] = c3(0.f, 0.f, 0.f);
    if (W.rep > 0) {
        const float4 t = W.ptot[i];
        total = c3(t.x, t.y, t.z);
    }
    for (uint32_t pi = 0; pi < W.npath; pi++)
        for (int j = 0; j < R.path_depth; j++) {
            const float4 c = W.p_contri[((size_t)(i * W.npath + pi)) * R.path_depth + j];
            if (c.w == 0.f) break;
            total = total + c3(c.x, c.y, c.z);
            sub[pi & 3u] = sub[pi & 3u] + c3(c.x, c.y, c.z);
        }
    W.ptot[i] = make_float4(total.r, total.g, total.b, 0.f);
    if (W.rep > 0) return;
    const float mult = (float)(1.0 / (double)(float)W.npath);
    float mn[3] = {1000.f, 1000.f, 1000.f}, mx[3] = {0.f, 0.f, 0.f};
    for (int k = 0; k < 4; k++) {
        const C3 c = sub[k] * mult;
        const float v[3] = {c.r, c.g, c.b};
        for (int ch = 0; ch < 3; ch++) {
            if (v[ch] > mx[ch]) mx[ch] = v[ch];
            if (v[ch] < mn[ch]) mn[ch] = v[ch];
        }
    }
    const C3 lo = expgam_adjust(c3(mn[0], mn[1], mn[2]), R.exposure, R.gamma_r, R.clamp_rgb != 0);
    const C3 hi = expgam_adjust(c3(mx[0], mx[1], mx[2]), R.exposure, R.gamma_r, R.clamp_rgb != 0);
    const float ene = fmaxf(fabsf(lo.r), fmaxf(fabsf(lo.g), fabsf(lo.b)));
    const float mad = fmaxf(fabsf(hi.r - lo.r), fmaxf(fabsf(hi.g - lo.g), fabsf(hi.b - lo.b)));
    float diff = (float)((double)mad / (((ene < 1.0f) ? 1.0 : (double)ene) * 2.0 * 2.0));
    diff /= R.path_threshold;
    int extra = (int)(diff * diff) - 1;
    extra = extra > 3 ? 3 : (extra < 0 ? 0 : extra);
    W.nrep[i] = (uint32_t)extra;
}

// The first directions of round W.rep (> 0) for the camera samples that
// take it: the camera vertex set up again as st_shade_camera does, then
// its paths queued (whole warp).
__device__ __forceinline__ void st_path_restart(const DevScene &S, const DevRender &R, const Wave &W, uint32_t i) {
    const bool inb = i < W.count;
    bool paths = false;
    if (inb && W.diff0[i].w != 0.f && W.nrep[i] >= W.rep) {
        const uint32_t cs = W.base + i;
        int x, y;
        const uint32_t pixel = cs_pixel(R, cs, x, y), s = cs % R.spp;
        const float4 h = W.hit0[i];
        float fx, fy;
        sample_pos(R, pixel, s, fx, fy);
        const V3 ray0 = camera_ray(R.cam, (float)x + fx, (float)y + fy);
        const V3 f = R.cam.pos + ray0 * kMinRayDist;
        const Surf sp = make_surface(S, R, __float_as_int(h.y), __float_as_uint(h.z), h.x, f, ray0);
        const V3 eye = R.cam.pos - sp.P;
        const V3 N0 = face_forward(sp.Ng, sp.N, eye);
        const float r0 = cp_rot(R.seed, pixel, 0), r1 = cp_rot(R.seed, pixel, 1);
        for (uint32_t pi = 0; pi < W.npath; pi++) {
            const uint32_t n = path_index(R, W, s, pi);
            const float z1 = cp_add(halton(kPrimes[0], n), r0), z2 = cp_add(halton(kPrimes[1], n), r1);
            const V3 ray = cos_hemi_dir(N0, sp.NU, sp.NV, z1, z2);
            const uint32_t p = i * W.npath + pi;
            W.p_where[p] = make_float4(sp.P.x, sp.P.y, sp.P.z, dot(ray, N0));
            W.p_ray[p] = make_float4(ray.x, ray.y, ray.z, 1.f);
            W.p_col[p] = make_float4(1.f, 1.f, 1.f, 0.f);
        }
        paths = true;
    }
    for (uint32_t pi = 0; pi < W.npath; pi++) {
        const uint32_t q = warp_append(&W.counters[1], paths);
        if (paths) W.bq[q] = i * W.npath + pi;
    }
}

#ifdef YR_WAVE_KERNELS
static __global__ void __launch_bounds__(kBlock) k_path_round(DevRender R, Wave W) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < W.count) st_path_round(R, W, i);
}

static __global__ void __launch_bounds__(kBlock, YR_SHADE_MINB) k_path_restart(DevScene S, DevRender R, Wave W) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W.count && (i & ~31u) >= W.count) return;  // whole warps past the end leave
    st_path_restart(S, R, W, i);
}
#endif

#ifdef YR_WAVE_KERNELS
static __global__ void __launch_bounds__(kBlock) k_finish(DevRender R, Wave W) {
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x;
    if (px < W.count / R.spp) st_finish(R, W, px);
}
#endif

#ifdef YR_WAVE_KERNELS
static __global__ void k_clear_contri(Wave W, size_t n) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        W.p_contri[q] = make_float4(0.f, 0.f, 0.f, 0.f);
}
#endif

#ifdef YR_WAVE_KERNELS
static __global__ void k_swap_queues(Wave W) {
    // bounce queue <- next queue (the caller swaps the pointers)
    W.counters[1] = W.counters[2];
    W.counters[2] = 0;
}
#endif

#ifdef YR_WAVE_KERNELS
static __global__ void k_count(Wave W, int which) {
    // accumulate queue lengths into the 64-bit ray totals
    if (which == 0) {  // the queue's rays: its places less the empty ones
        W.rays[1] += W.counters[0] - W.counters[8];
        W.counters[8] = 0;
    }
    if (which == 1) W.rays[2] += W.counters[1];
}
#endif


// ------------------------------------------------------------ wave layout
// Shape of a render: slots per vertex, paths per camera sample, lights.
struct Plan {
    uint32_t npix;    // image pixels
    uint32_t rpix;    // region pixels
    uint64_t total;   // camera samples to render
    uint32_t ns;      // shadow slots per vertex
    uint32_t npath;   // path samples per camera sample
    uint32_t nl;      // lights (>= 1 for sizing)
    int depth;        // path depth (>= 1 for sizing)
};

inline yr_status make_plan(const yr_scene *scene, Plan &P) {
    const DevRender &R = scene->rdr;
    P.npix = (uint32_t)R.cam.resx * (uint32_t)R.cam.resy;
    P.rpix = (uint32_t)R.rw * (uint32_t)R.rh;
    P.total = (uint64_t)P.rpix * R.spp;
    if (P.total >= (1ull << 32)) return YR_ERR_TOO_LARGE;
    if (R.path_light >= 0 && R.path_depth > 15) return YR_ERR_UNSUPPORTED;
    P.ns = 0;
    for (const DevLight &L : scene->lights) {
        if (L.type == YR_LIGHT_POINT) P.ns += 1;
        else if (L.type == YR_LIGHT_AREA || L.type == YR_LIGHT_HEMI) P.ns += (uint32_t)L.samples;
        P.ns += (uint32_t)L.psamples;  // the penumbra guess's probe slots, after the sample slots
    }
    P.npath = R.path_light >= 0 ? (uint32_t)R.path_samples : 0;
    P.nl = (uint32_t)std::max(1, R.nlights);
    P.depth = std::max(1, R.path_depth);
    return YR_OK;
}

constexpr int kNumBufs = 25;
constexpr size_t kBufAlign = 256;

// Bytes of each scratch buffer for a wave of `wcap` camera samples, in the
// order assign_wave() hands them out.
__host__ __device__ inline void wave_sizes(const Plan &P, uint32_t wcap, size_t *b) {
    const size_t w = wcap, pc = (size_t)wcap * (P.npath > 1u ? P.npath : 1u), vc = w > pc ? w : pc;
    const size_t slots = vc * (P.ns > 1u ? P.ns : 1u);
    const size_t f4 = sizeof(float4);
    size_t sizes[kNumBufs] = {f4 * w,  f4 * w * P.nl, f4 * w * P.nl, f4 * w,  f4 * pc, f4 * pc,
                              f4 * pc, f4 * pc,       f4 * pc,       f4 * pc, f4 * pc * P.depth, f4 * pc * P.nl,
                              f4 * slots, slots,      f4 * slots,    f4 * slots, 4 * slots, 4 * pc,
                              4 * pc,  4 * 16,        8 * 4,         8 * 3 * YR_K_COUNT,
                              f4 * w,  4 * w,         4 * pc};
    for (int i = 0; i < kNumBufs; i++) b[i] = sizes[i];
}

__host__ __device__ inline size_t wave_bytes(const Plan &P, uint32_t wcap) {
    size_t b[kNumBufs], t = 0;
    wave_sizes(P, wcap, b);
    for (int i = 0; i < kNumBufs; i++) t += (b[i] + kBufAlign - 1) / kBufAlign * kBufAlign;
    return t;
}

// Point the wave's arrays into one block of at least wave_bytes(P, wcap).
__host__ __device__ inline void assign_wave(const Plan &P, uint32_t wcap, char *base, Wave &W) {
    size_t b[kNumBufs];
    wave_sizes(P, wcap, b);
    void *ptr[kNumBufs];
    size_t off = 0;
    for (int i = 0; i < kNumBufs; i++) {
        ptr[i] = base + off;
        off += (b[i] + kBufAlign - 1) / kBufAlign * kBufAlign;
    }
    int k = 0;
    W.hit0 = (float4 *)ptr[k++];
    W.lterm = (float4 *)ptr[k++];
    W.aux = (float4 *)ptr[k++];
    W.diff0 = (float4 *)ptr[k++];
    W.p_where = (float4 *)ptr[k++];
    W.p_ray = (float4 *)ptr[k++];
    W.p_col = (float4 *)ptr[k++];
    W.p_next = (float4 *)ptr[k++];
    W.p_nray = (float4 *)ptr[k++];
    W.p_hit = (float4 *)ptr[k++];
    W.p_contri = (float4 *)ptr[k++];
    W.p_aux = (float4 *)ptr[k++];
    W.slot_c = (float4 *)ptr[k++];
    W.slot_f = (uint8_t *)ptr[k++];
    W.shq0 = (float4 *)ptr[k++];
    W.shq1 = (float4 *)ptr[k++];
    W.shq_slot = (uint32_t *)ptr[k++];
    W.bq = (uint32_t *)ptr[k++];
    W.bq2 = (uint32_t *)ptr[k++];
    W.counters = (uint32_t *)ptr[k++];
    W.rays = (unsigned long long *)ptr[k++];
    W.kst = (unsigned long long *)ptr[k++];
    W.ptot = (float4 *)ptr[k++];
    W.nrep = (uint32_t *)ptr[k++];
    W.sq = (uint32_t *)ptr[k++];
    W.part = 0;
    W.rep = 0;
    W.ns = P.ns;
    W.npath = P.npath;
    W.nv = P.npath > 1u ? wcap * P.npath : wcap;  // as wave_sizes' vc
}

// Blocks of kBlock threads that fill every SM once for `kernel` (queried
// once per device and kernel), the grid of the traversal kernels.
// The per-device caches below are filled under one lock: the first renders
// on a device may come from several host threads at once.
inline std::mutex &device_cache_mutex() {
    static std::mutex mu;
    return mu;
}

template <class K>
inline int resident_grid(K kernel) {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    std::lock_guard<std::mutex> lock(device_cache_mutex());
    if (!cached[dev]) {
        int sms = 148, per = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kBlock, 0) != cudaSuccess || per < 1) per = 1;
        cached[dev] = sms * per;
    }
    return cached[dev];
}

// Enqueue every launch of one render of `scene` on `st` (no synchronization,
// capturable): waves of `wcap` camera samples through the scratch that
// `W` points to (render.cu).
yr_status enqueue_render(yr_scene *scene, const Plan &P, uint32_t wcap, Wave &W, float *out, cudaStream_t st);

// Scratch budget of one wavefront when `sharers` of them run at once on the
// current device: a quarter of the free memory shared out, at least 1.5 GB
// and at most 16 GB each.  Larger waves keep more rays in every launch
// (fewer, fuller launches: 1.5 GB -> 16 GB is +12% on a 1920x1080, 16 spp
// GI frame).
// The free memory is read once per device (the first render on it).
inline size_t render_budget(int sharers) {
    static size_t free_at_start[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    std::lock_guard<std::mutex> lock(device_cache_mutex());
    if (!free_at_start[dev]) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b == 0) free_b = 1;
        free_at_start[dev] = free_b;
    }
    const size_t lo = 1536ull << 20, hi = 16384ull << 20;
    const size_t b = free_at_start[dev] / 4 / (size_t)(sharers > 0 ? sharers : 1);
    return std::min(hi, std::max(lo, b));
}

// Largest wave (whole pixels) whose scratch fits in `budget` bytes.
inline uint32_t wave_for_budget(const Plan &P, const DevRender &R, size_t budget) {
    uint64_t lo = 0, hi = P.rpix;
    while (lo < hi) {  // largest pixel count that fits
        const uint64_t mid = (lo + hi + 1) / 2;
        if (wave_bytes(P, (uint32_t)(mid * R.spp)) <= budget) lo = mid;
        else hi = mid - 1;
    }
    return (uint32_t)(lo * R.spp);
}


}  // namespace yr
