// yr_backward: gradient of an image loss with respect to the shaders'
// colours, specular weights and texture parameters and the lights' powers.
//
// Geometry is fixed, so every ray, hit and shadow answer of the forward
// render is a constant of the parameters; the pixel value is then a
// polynomial in them.  For one camera sample with diffuse colour C0 and
// specular colour S0 at its hit:
//   c = sum_k pow_k (C0 . D_k + S0 . Sp_k)                  direct light k
//     + pow_path / P * C0 . sum_paths sum_j cosN * (prod_{i<j} C_i) . G_j
// where D_k / Sp_k are the diffuse / specular factors of light k per unit
// power (fromLight split, basicshaders.cc:46-70), C_i the diffuse colour at
// bounce vertex i and G_j the direct light at vertex j (or the background
// on a miss), as pathLight_t::takeSample accumulates them
// (pathlight.cc:303-347).  The adjoint re-runs the wavefront of yr_render
// with the same QMC indices (the recompute stands in for stored paths),
// keeps each light sample's D / Sp factors instead of its colour, and
// accumulates dL/dparam: direct-light terms at the gather of each vertex,
// the path products backwards (Horner) per camera sample at the end of the
// wave.  Texture chain: C = mix(color1 + f (color2 - color1), C_base, w)
// with f = intensity * fBm (basictex.cc:656-709, color.cc:103-109).
//
// The energy cut-offs of the forward (paths stop below 0.05; hemi lights
// skip weak points) are treated as fixed decisions.  Gradients are
// accumulated in FP32 per block in shared memory, then added to the global
// vector with one atomic per parameter per block.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#define YR_WAVE_KERNELS 1
#include "dev_wave.cuh"

namespace yr {

constexpr uint32_t kSmemParams = 8192;  // gradients kept in shared memory up to this many parameters

struct GradAcc {
    float *acc;  // shared-memory copy, or the global vector
    __device__ __forceinline__ void add(int i, float v) const {
        if (v != 0.f) atomicAdd(acc + i, v);
    }
};

__device__ __forceinline__ GradAcc grad_begin(const AdjWave &A, float *smem) {
    const bool use = A.nparams <= kSmemParams;
    if (use)
        for (uint32_t i = threadIdx.x; i < A.nparams; i += blockDim.x) smem[i] = 0.f;
    __syncthreads();
    return GradAcc{use ? smem : A.grad};
}

__device__ __forceinline__ void grad_end(const AdjWave &A, const GradAcc &g) {
    __syncthreads();
    if (g.acc != A.grad)
        for (uint32_t i = threadIdx.x; i < A.nparams; i += blockDim.x) {
            const float v = g.acc[i];
            if (v != 0.f) atomicAdd(A.grad + i, v);
        }
}

__device__ __forceinline__ float dot3(const C3 &a, const C3 &b) { return a.r * b.r + a.g * b.g + a.b * b.b; }

// dL/dC and dL/dS at a vertex of shader `sid` -> the shader's parameters.
// C is the modulated diffuse colour; md[0] = (d tex / d intensity, d tex /
// d color1), md[1] = (tex, 0) at the vertex (modulated_color's TexDeriv).
__device__ __forceinline__ void chain_shader(const DevRender &R, const AdjWave &A, const GradAcc &acc, int sid,
                                             const float4 *md, const C3 &dC, const C3 &dS) {
    const DevShader &sh = R.shaders[sid];
    const int b = A.sh_pbase[sid];
    C3 dCb = dC;
    if (sh.tex_type != YR_TEX_NONE && sh.mod_color > 0.f) {
        const float4 m0 = md[0], m1 = md[1];
        const C3 tex = c3(m1.x, m1.y, m1.z);
        const float w = sh.mod_color;
        C3 dtex;
        switch (sh.mod_mode) {
        case YR_MOD_MUL:  // C' = mix(tex, 1, w) * C
            dtex = w > 1.f ? dC * sh.color : (dC * sh.color) * w;
            dCb = dC * (w > 1.f ? tex : tex * w + (1 - w) * c3(1.f, 1.f, 1.f));
            break;
        case YR_MOD_ADD: dtex = dC * w; break;
        case YR_MOD_SUB: dtex = dC * -w; break;
        default:  // mix(tex, C, w)
            dtex = w > 1.f ? dC : dC * w;
            dCb = w > 1.f ? c3(0.f, 0.f, 0.f) : dC * (1.f - w);
        }
        acc.add(b + 4, dot3(dtex, c3(m0.x, m0.y, m0.z)));
        const C3 dtc1 = dtex * m0.w;
        acc.add(b + 5, dtc1.r);
        acc.add(b + 6, dtc1.g);
        acc.add(b + 7, dtc1.b);
    }
    acc.add(b + 0, dCb.r);
    acc.add(b + 1, dCb.g);
    acc.add(b + 2, dCb.b);
    const float4 sd = A.spec_dir[sid];
    acc.add(b + 3, dS.r * sd.x + dS.g * sd.y + dS.b * sd.z);
}

// Direct light at one vertex from its slots (adjoint form of gather_term):
// accumulates the light-power and shader gradients for adjoint weight Wv
// and returns the direct light sum G.
__device__ __forceinline__ C3 adj_vertex_direct(const DevRender &R, const Wave &W, const AdjWave &A,
                                                const GradAcc &acc, uint32_t vtx, const float4 *aux, const C3 &lkc,
                                                int sid, const float4 *md, const C3 &Wv) {
    const C3 spec = R.shaders[sid].specular;
    C3 Dt = c3(0.f, 0.f, 0.f), St = c3(0.f, 0.f, 0.f);
    uint32_t off = 0;
    for (int k = 0; k < R.nlights; k++) {
        const DevLight L = R.lights[k];
        C3 Dk = c3(0.f, 0.f, 0.f), Sk = c3(0.f, 0.f, 0.f);
        if (L.type == YR_LIGHT_POINT) {
            const uint32_t slot = slot_of(W, vtx, off);
            if (W.slot_f[slot] == kSlotLit) {
                const float4 d = W.slot_c[slot], e = A.slot_s[slot];
                Dk = c3(d.x, d.y, d.z);
                Sk = c3(e.x, e.y, e.z);
            }
        } else if (L.type == YR_LIGHT_AREA) {
            const float4 a = aux[vtx * R.nlights + k];
            if (a.y != 0.f) {
                for (int jj = 0; jj < L.samples; jj++) {
                    const uint32_t slot = slot_of(W, vtx, off + (uint32_t)jj);
                    if (W.slot_f[slot] == kSlotLit) {
                        const float4 d = W.slot_c[slot], e = A.slot_s[slot];
                        Dk = Dk + c3(d.x, d.y, d.z);
                        Sk = Sk + c3(e.x, e.y, e.z);
                    }
                }
                const float f = a.x / (float)L.samples;
                Dk = Dk * f;
                Sk = Sk * f;
            }
        } else if (L.type == YR_LIGHT_HEMI) {
            const float4 a = aux[vtx * R.nlights + k];
            if (a.w != 0.f) {
                C3 total = c3(0.f, 0.f, 0.f);
                for (int jj = 0; jj < L.samples; jj++) {
                    const uint32_t slot = slot_of(W, vtx, off + (uint32_t)jj);
                    if (W.slot_f[slot] == kSlotLit) {
                        const float4 d = W.slot_c[slot];
                        total = total + c3(d.x, d.y, d.z);
                    }
                }
                Dk = total * (a.x / (float)L.samples);
                Sk = total * (a.y / (float)L.samples);
            }
        }
        if (L.type != YR_LIGHT_PATH) {
            acc.add(A.li_pidx[k], dot3(Wv, lkc * Dk + spec * Sk));
            Dt = Dt + L.power * Dk;
            St = St + L.power * Sk;
        }
        off += light_slots(L);
    }
    chain_shader(R, A, acc, sid, md, Wv * Dt, Wv * St);
    return lkc * Dt + spec * St;
}

__device__ __forceinline__ C3 sample_weight(const DevRender &R, const AdjWave &A, uint32_t cs) {
    int x, y;
    const uint32_t pixel = cs_pixel(R, cs, x, y);
    const float4 g = A.gpix[pixel];
    const float inv = 1.f / (float)R.spp;  // the pixel is the mean of its spp samples
    return c3(g.x * inv, g.y * inv, g.z * inv);
}

// --------------------------------------------------------------- kernels
// dL/dpixel = 2 * scale * (img - target) over RGB; loss in double.  With
// alpha premultiply the image is the average times its alpha, so the
// gradient of the average is alpha times that.
__global__ void __launch_bounds__(kBlock) k_adj_loss(const float4 *img, const float4 *target, uint32_t npix,
                                                      float scale, int premultiply, float4 *gpix, double *loss) {
    double part = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        const float4 a = img[i], b = target[i];
        const float r = a.x - b.x, g = a.y - b.y, bl = a.z - b.z;
        part += (double)scale * ((double)r * r + (double)g * g + (double)bl * bl);
        const float s2 = premultiply ? 2.f * scale * a.w : 2.f * scale;
        gpix[i] = make_float4(s2 * r, s2 * g, s2 * bl, 0.f);
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0 && part != 0.0) atomicAdd(loss, part);
}

__global__ void __launch_bounds__(kBlock) k_adj_shade_camera(DevScene S, DevRender R, Wave W, AdjWave A) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W.count && (i & ~31u) >= W.count) return;  // whole warps past the end leave
    st_shade_camera<true>(S, R, W, i, &A);
}

__global__ void __launch_bounds__(kBlock) k_adj_gather_camera(DevRender R, Wave W, AdjWave A) {
    extern __shared__ float smem[];
    const GradAcc acc = grad_begin(A, smem);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < W.count) {
        const float4 h = W.hit0[i];
        if (__float_as_int(h.y) >= 0) {
            const float4 v = A.v0[i];
            adj_vertex_direct(R, W, A, acc, i, W.aux, c3(v.x, v.y, v.z), __float_as_int(v.w), A.v0m + 2 * (size_t)i,
                              sample_weight(R, A, W.base + i));
        }
    }
    grad_end(A, acc);
}

__global__ void k_adj_clear(AdjWave A, size_t n) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        A.pG[q] = make_float4(0.f, 0.f, 0.f, 0.f);
        A.pv[q] = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
    }
}

__global__ void __launch_bounds__(kBlock) k_adj_shade_path(DevScene S, DevRender R, Wave W, int j, AdjWave A) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = W.counters[1];
    if (q >= n && (q & ~31u) >= n) return;
    st_shade_path<true>(S, R, W, j, q, n, &A);
}

// adjoint of st_gather_path: direct-light gradients at bounce vertex j,
// the vertex's direct light kept for the backward pass, and the same
// continuation decision as the forward
__global__ void __launch_bounds__(kBlock) k_adj_gather_path(DevRender R, Wave W, int j, C3 bg, AdjWave A) {
    extern __shared__ float smem[];
    const GradAcc acc = grad_begin(A, smem);
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = W.counters[1];
    if (q < n || (q & ~31u) < n) {
        const bool inq = q < n;
        const uint32_t p = inq ? W.bq[q] : 0;
        bool requeue = false;
        if (inq) {
            const uint32_t i = p / W.npath;
            const float4 h = W.p_hit[p];
            const float4 col = W.p_col[p];
            const float startN = W.p_where[p].w;
            const size_t ci = (size_t)p * R.path_depth + j;
            if (__float_as_int(h.y) < 0) {
                A.pG[ci] = make_float4(bg.r, bg.g, bg.b, 1.f);
            } else {
                const float4 d0 = W.diff0[i];
                const float mult = (float)(1.0 / (double)(float)W.npath);
                const C3 g = sample_weight(R, A, W.base + i);
                const C3 Wv = ((g * c3(d0.x, d0.y, d0.z)) * (d0.w * mult * startN)) * c3(col.x, col.y, col.z);
                const float4 v = A.pv[ci];
                const C3 G = adj_vertex_direct(R, W, A, acc, p, W.p_aux, c3(v.x, v.y, v.z), __float_as_int(v.w),
                                               A.pm + 2 * ci, Wv);
                A.pG[ci] = make_float4(G.r, G.g, G.b, 1.f);
                const float4 nc = W.p_next[p];
                const C3 ncol = c3(nc.x, nc.y, nc.z);
                W.p_col[p] = make_float4(ncol.r, ncol.g, ncol.b, 0.f);
                if (j + 1 < R.path_depth && !(energy(ncol) < 0.05f)) {
                    const float4 nr = W.p_nray[p];
                    W.p_ray[p] = make_float4(nr.x, nr.y, nr.z, 1.f);
                    requeue = true;
                }
            }
        }
        const uint32_t nq = warp_append(&W.counters[2], requeue);
        if (requeue) W.bq2[nq] = p;
    }
    grad_end(A, acc);
}

// per camera sample: path products backwards, the camera vertex's diffuse
// colour and the path light's power
__global__ void __launch_bounds__(kBlock) k_adj_finish(DevRender R, Wave W, AdjWave A) {
    extern __shared__ float smem[];
    const GradAcc acc = grad_begin(A, smem);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < W.count && R.path_light >= 0) {
        const float4 h = W.hit0[i], d0 = W.diff0[i];
        if (__float_as_int(h.y) >= 0 && d0.w != 0.f) {
            const C3 g = sample_weight(R, A, W.base + i), dif0 = c3(d0.x, d0.y, d0.z);
            const float mult = (float)(1.0 / (double)(float)W.npath);
            const C3 Acol = (g * dif0) * (d0.w * mult);
            C3 Tsum = c3(0.f, 0.f, 0.f);
            C3 rc[16];
            for (uint32_t pi = 0; pi < W.npath; pi++) {
                const uint32_t p = i * W.npath + pi;
                const float startN = W.p_where[p].w;
                const size_t c0 = (size_t)p * R.path_depth;
                int J = 0;
                rc[0] = c3(1.f, 1.f, 1.f);
                while (J < R.path_depth && A.pG[c0 + J].w != 0.f) {
                    const float4 v = A.pv[c0 + J];
                    rc[J + 1] = __float_as_int(v.w) >= 0 ? rc[J] * c3(v.x, v.y, v.z) : c3(0.f, 0.f, 0.f);
                    J++;
                }
                C3 U = c3(0.f, 0.f, 0.f);  // sum over later vertices, Horner form
                for (int jj = J - 1; jj >= 0; jj--) {
                    const float4 v = A.pv[c0 + jj], G = A.pG[c0 + jj];
                    const int sid = __float_as_int(v.w);
                    if (sid >= 0) {
                        if (U.r != 0.f || U.g != 0.f || U.b != 0.f)
                            chain_shader(R, A, acc, sid, A.pm + 2 * (c0 + jj), (Acol * startN) * (rc[jj] * U),
                                         c3(0.f, 0.f, 0.f));
                        U = c3(G.x, G.y, G.z) + c3(v.x, v.y, v.z) * U;
                    } else {
                        U = c3(G.x, G.y, G.z);
                    }
                }
                Tsum = Tsum + startN * U;
            }
            const float4 v = A.v0[i];
            chain_shader(R, A, acc, __float_as_int(v.w), A.v0m + 2 * (size_t)i, g * (Tsum * (d0.w * mult)),
                         c3(0.f, 0.f, 0.f));
            acc.add(A.li_pidx[R.path_light], dot3(g, dif0 * (Tsum * mult)));
        }
    }
    grad_end(A, acc);
}

// ------------------------------------------------------------ layout
constexpr int kNumAdjBufs = 7;

static void adj_sizes(const Plan &P, uint32_t wcap, uint32_t npix, size_t *b) {
    const size_t w = wcap, pc = (size_t)wcap * (P.npath > 1u ? P.npath : 1u), vc = w > pc ? w : pc;
    const size_t slots = vc * (P.ns > 1u ? P.ns : 1u), pd = pc * (size_t)P.depth;
    const size_t f4 = sizeof(float4);
    const size_t sizes[kNumAdjBufs] = {f4 * slots, f4 * w, 2 * f4 * w, f4 * pd, 2 * f4 * pd, f4 * pd, f4 * (size_t)npix};
    for (int i = 0; i < kNumAdjBufs; i++) b[i] = sizes[i];
}

static size_t adj_bytes(const Plan &P, uint32_t wcap, uint32_t npix) {
    size_t b[kNumAdjBufs], t = 0;
    adj_sizes(P, wcap, npix, b);
    for (int i = 0; i < kNumAdjBufs; i++) t += (b[i] + kBufAlign - 1) / kBufAlign * kBufAlign;
    return t;
}

static void assign_adj(const Plan &P, uint32_t wcap, uint32_t npix, char *base, AdjWave &A) {
    size_t b[kNumAdjBufs];
    adj_sizes(P, wcap, npix, b);
    void *ptr[kNumAdjBufs];
    size_t off = 0;
    for (int i = 0; i < kNumAdjBufs; i++) {
        ptr[i] = base + off;
        off += (b[i] + kBufAlign - 1) / kBufAlign * kBufAlign;
    }
    A.slot_s = (float4 *)ptr[0];
    A.v0 = (float4 *)ptr[1];
    A.v0m = (float4 *)ptr[2];
    A.pv = (float4 *)ptr[3];
    A.pm = (float4 *)ptr[4];
    A.pG = (float4 *)ptr[5];
    A.gpix = (const float4 *)ptr[6];
}


int grid_for(uint32_t n, int block);



// Wave size and scratch bytes of one backward pass.
struct AdjPlan {
    Plan P;
    uint32_t wcap = 0;
    size_t wave = 0;    // bytes of the wave buffers (256-aligned)
    size_t bytes = 0;   // wave + adjoint buffers
};

static yr_status adj_plan(const yr_scene *scene, size_t budget, AdjPlan &A) {
    const DevRender &R = scene->rdr;
    yr_status ret = make_plan(scene, A.P);
    if (ret != YR_OK) return ret;
    if (R.raydepth <= 0) return YR_ERR_UNSUPPORTED;
    // per-sample exposure / gamma is not differentiated
    if (R.tonemap && !(R.exposure == 0.f && R.gamma_r == 1.f && !R.clamp_rgb)) return YR_ERR_UNSUPPORTED;
    // nor the penumbra guess's decisions or the path light's adaptive
    // rounds, nor a texture's modulation of
    // the specular colour or exponent
    if (R.has_guess || R.path_threshold > 0.f) return YR_ERR_UNSUPPORTED;
    for (const yr_shader_desc &d : scene->shader_desc)
        if (d.tex_type != YR_TEX_NONE &&
            (d.mod_specular > 0.f || d.mod_hard > 0.f || (d.tex_map & 0xffu) == YR_TEXCO_REFLECT))
            return YR_ERR_UNSUPPORTED;  // (a reflected-eye texture differs between a vertex's shading calls)
    const Plan &P = A.P;
    uint64_t lo = 1, hi = P.rpix;
    while (lo < hi) {
        const uint64_t mid = (lo + hi + 1) / 2;
        const uint32_t w = (uint32_t)(mid * R.spp);
        if (wave_bytes(P, w) + adj_bytes(P, w, P.npix) <= budget) lo = mid;
        else hi = mid - 1;
    }
    A.wcap = (uint32_t)(lo * R.spp);
    A.wave = (wave_bytes(P, A.wcap) + 255) / 256 * 256;
    A.bytes = A.wave + adj_bytes(P, A.wcap, P.npix);
    return YR_OK;
}

// Every launch of one backward pass on `st` (capturable, no synchronization);
// `blk` holds A.bytes of scratch; the loss is added to *d_loss.
static yr_status enqueue_backward(yr_scene *scene, const AdjPlan &AP, char *blk, const yr_backward_desc *desc,
                                  float *dparams, double *d_loss, cudaStream_t st) {
    const DevRender &R = scene->rdr;
    const Plan &P = AP.P;
    const uint32_t wcap = AP.wcap;
    Wave W;
    std::memset(&W, 0, sizeof(W));
    assign_wave(P, wcap, blk, W);
    AdjWave A;
    std::memset(&A, 0, sizeof(A));
    assign_adj(P, wcap, P.npix, blk + AP.wave, A);
    A.grad = dparams;
    A.sh_pbase = scene->d_sh_pbase;
    A.li_pidx = scene->d_li_pidx;
    A.spec_dir = scene->d_spec_dir;
    A.nparams = scene->nparams;
    const size_t smem = A.nparams <= kSmemParams ? sizeof(float) * std::max<uint32_t>(A.nparams, 1u) : 0;

    if (scene->nparams) cudaMemsetAsync(dparams, 0, sizeof(float) * scene->nparams, st);
    cudaMemsetAsync(W.rays, 0, sizeof(unsigned long long) * 4, st);
    cudaMemsetAsync(W.kst, 0, sizeof(unsigned long long) * 3 * YR_K_COUNT, st);
    k_adj_loss<<<grid_for(P.npix, kBlock), kBlock, 0, st>>>((const float4 *)desc->image,
                                                             (const float4 *)desc->target, P.npix, desc->loss_scale,
                                                             scene->rdr.premultiply, (float4 *)A.gpix, d_loss);
    const DevScene &D = scene->dev;
    const uint32_t vcap = std::max(wcap, wcap * std::max(1u, P.npath));
#if YR_TRACE_GRID_PERSIST
    const int gq = std::min(grid_for(vcap * std::max(P.ns, 1u), kBlock), resident_grid(k_trace_shadow_q<false, true>));
    const int gb = std::min(grid_for(vcap, kBlock), resident_grid(k_trace_bounce<false>));
#else
    const int gq = grid_for(vcap * std::max(P.ns, 1u), kBlock), gb = gq;
#endif
    const bool inst = D.insts != nullptr;
    auto k_prim = inst ? k_primary<true> : k_primary<false>;
    // the shadow queue kernel with the casters' BVH walk alone when the
    // scene uses it (no shadow-ray tree, no exact order)
    const bool bvh = !D.use_sh_tree && !D.exact_order;
    auto k_shadow = inst ? (bvh ? k_trace_shadow_q<true, true> : k_trace_shadow_q<true, false>)
                         : (bvh ? k_trace_shadow_q<false, true> : k_trace_shadow_q<false, false>);
    auto k_bounce = inst ? k_trace_bounce<true> : k_trace_bounce<false>;
    for (uint64_t b = 0; b < P.total; b += wcap) {
        W.base = (uint32_t)b;
        W.count = (uint32_t)std::min<uint64_t>(wcap, P.total - b);
        const int g = (int)((W.count + kBlock - 1) / kBlock);
        cudaMemsetAsync(W.counters, 0, sizeof(uint32_t) * 16, st);
        k_prim<<<g, kBlock, 0, st>>>(D, R, W);
        k_adj_shade_camera<<<g, kBlock, 0, st>>>(D, R, W, A);
        cudaMemsetAsync(W.counters + 6, 0, sizeof(uint32_t), st);
        k_shadow<<<gq, kBlock, 0, st>>>(D, W, R.self_bias);
        k_adj_gather_camera<<<g, kBlock, smem, st>>>(R, W, A);
        if (P.npath > 0) {
            const size_t nc = (size_t)W.count * P.npath * P.depth;
            k_adj_clear<<<grid_for((uint32_t)std::min<size_t>(nc, 1u << 30), kBlock), kBlock, 0, st>>>(A, nc);
            const int gp = (int)(((size_t)W.count * P.npath + kBlock - 1) / kBlock);
            for (int j = 0; j < R.path_depth; j++) {
                cudaMemsetAsync(W.counters + 7, 0, sizeof(uint32_t), st);
                k_bounce<<<gb, kBlock, 0, st>>>(D, W);
                cudaMemsetAsync(W.counters, 0, sizeof(uint32_t), st);
                k_adj_shade_path<<<gp, kBlock, 0, st>>>(D, R, W, j, A);
                cudaMemsetAsync(W.counters + 6, 0, sizeof(uint32_t), st);
                k_shadow<<<gq, kBlock, 0, st>>>(D, W, R.self_bias);
                k_adj_gather_path<<<gp, kBlock, smem, st>>>(R, W, j, R.background, A);
                std::swap(W.bq, W.bq2);
                k_swap_queues<<<1, 1, 0, st>>>(W);
            }
            k_adj_finish<<<g, kBlock, smem, st>>>(R, W, A);
        }
    }
    return cudaGetLastError() == cudaSuccess ? YR_OK : YR_ERR_CUDA;
}

// ------------------------------------------------ batched forward + backward
// One optimisation step of many scenes as one CUDA graph: each scene's
// forward render into its image, then its backward pass, on one of a few
// concurrent streams (longest scenes first onto the least loaded stream);
// scenes on one stream share one scratch block.
struct AdjLane {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<uint32_t> scenes;
    char *scratch = nullptr;
};

struct AdjBatch {
    int device = -1;
    std::vector<yr_scene *> scenes;
    std::vector<DevScene> h_scenes;
    std::vector<DevRender> h_renders;
    std::vector<yr_backward_desc> descs;
    std::vector<float *> grads;
    std::vector<AdjPlan> plans;
    std::vector<uint32_t> fwave;   // forward wave of each scene
    std::vector<AdjLane> lanes;
    double *d_loss = nullptr;
    unsigned long long *d_rays = nullptr;  // 4 per scene
    unsigned long long *d_kst = nullptr;
    cudaEvent_t fork = nullptr;
    cudaGraphExec_t graph = nullptr;
    ~AdjBatch() {
        if (graph) cudaGraphExecDestroy(graph);
        for (AdjLane &l : lanes) {
            if (l.stream) cudaStreamDestroy(l.stream);
            if (l.done) cudaEventDestroy(l.done);
            cudaFree(l.scratch);
        }
        if (fork) cudaEventDestroy(fork);
        cudaFree(d_loss);
        cudaFree(d_rays);
        cudaFree(d_kst);
    }
};

static std::mutex g_adj_mu;
static std::map<std::vector<uintptr_t>, std::unique_ptr<AdjBatch>> g_adj_batches;

void adj_batch_forget(const yr_scene *s) {
    std::lock_guard<std::mutex> lock(g_adj_mu);
    for (auto it = g_adj_batches.begin(); it != g_adj_batches.end();) {
        if (std::find(it->second->scenes.begin(), it->second->scenes.end(), s) != it->second->scenes.end()) {
            int prev = 0;
            cudaGetDevice(&prev);
            cudaSetDevice(it->second->device);
            it = g_adj_batches.erase(it);
            cudaSetDevice(prev);
        } else {
            ++it;
        }
    }
}

static yr_status adj_batch_capture(AdjBatch &B) {
    if (B.graph) cudaGraphExecDestroy(B.graph);
    B.graph = nullptr;
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return YR_ERR_CUDA;
    yr_status ret = YR_OK;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaStreamDestroy(cs);
        return YR_ERR_CUDA;
    }
    const size_t n = B.scenes.size();
    cudaMemsetAsync(B.d_loss, 0, sizeof(double) * n, cs);
    cudaEventRecord(B.fork, cs);
    for (AdjLane &l : B.lanes) {
        cudaStreamWaitEvent(l.stream, B.fork, 0);
        for (uint32_t s : l.scenes) {
            yr_scene *sc = B.scenes[s];
            const AdjPlan &A = B.plans[s];
            Wave W;
            std::memset(&W, 0, sizeof(W));
            assign_wave(A.P, B.fwave[s], l.scratch, W);
            W.rays = B.d_rays + 4 * (size_t)s;
            W.kst = B.d_kst;
            if (ret == YR_OK) ret = enqueue_render(sc, A.P, B.fwave[s], W, (float *)B.descs[s].image, l.stream);
            if (ret == YR_OK)
                ret = enqueue_backward(sc, A, l.scratch, &B.descs[s], B.grads[s], B.d_loss + s, l.stream);
        }
        cudaEventRecord(l.done, l.stream);
        cudaStreamWaitEvent(cs, l.done, 0);
    }
    const cudaError_t ee = cudaStreamEndCapture(cs, &g);
    if (ret == YR_OK && ee != cudaSuccess) ret = YR_ERR_CUDA;
    if (ret == YR_OK && cudaGraphInstantiate(&B.graph, g, 0) != cudaSuccess) ret = YR_ERR_CUDA;
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    return ret;
}

}  // namespace yr

using namespace yr;

extern "C" {

YR_API uint32_t yr_param_count(const yr_scene *scene) { return scene ? scene->nparams : 0u; }

YR_API yr_status yr_params_get(const yr_scene *scene, float *params) {
    if (!scene || !params) return YR_ERR_INVALID_ARG;
    for (size_t i = 0; i < scene->shader_desc.size(); i++) {
        const yr_shader_desc &d = scene->shader_desc[i];
        float *o = params + scene->sh_pbase[i];
        o[0] = d.color[0];
        o[1] = d.color[1];
        o[2] = d.color[2];
        o[3] = std::max(d.specular[0], std::max(d.specular[1], d.specular[2]));
        if (d.tex_type != YR_TEX_NONE) {
            o[4] = d.tex_intensity;
            o[5] = d.tex_color1[0];
            o[6] = d.tex_color1[1];
            o[7] = d.tex_color1[2];
        }
    }
    for (size_t k = 0; k < scene->light_desc.size(); k++) params[scene->li_pidx[k]] = scene->light_desc[k].power;
    return YR_OK;
}

YR_API yr_status yr_params_set(yr_scene *scene, const float *params) {
    if (!scene || !params) return YR_ERR_INVALID_ARG;
    std::vector<yr_shader_desc> sh = scene->shader_desc;
    std::vector<yr_light_desc> li = scene->light_desc;
    for (size_t i = 0; i < sh.size(); i++) {
        const float *o = params + scene->sh_pbase[i];
        for (int c = 0; c < 3; c++) {
            sh[i].color[c] = o[c];
            sh[i].specular[c] = o[3] * scene->spec_dir[4 * i + c];
        }
        if (sh[i].tex_type != YR_TEX_NONE) {
            sh[i].tex_intensity = o[4];
            for (int c = 0; c < 3; c++) sh[i].tex_color1[c] = o[5 + c];
        }
    }
    for (size_t k = 0; k < li.size(); k++) li[k].power = params[scene->li_pidx[k]];
    return yr_scene_set_params(scene, sh.empty() ? nullptr : sh.data(), li.empty() ? nullptr : li.data());
}

YR_API yr_status yr_backward(yr_scene *scene, const yr_backward_desc *desc, float *dparams, float *loss_out,
                             void *stream) {
    if (!scene || !desc || !desc->target || !desc->image || (!dparams && scene->nparams)) return YR_ERR_INVALID_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(scene->device);
    auto done = [&](yr_status e) {
        cudaSetDevice(prev);
        return e;
    };
    cudaStream_t st = (cudaStream_t)stream;
    AdjPlan A;
    yr_status ret = adj_plan(scene, render_budget(1), A);
    if (ret != YR_OK) return done(ret);
    PoolBlock pb(scene->device, st);  // given back (after a stream sync) when this call returns
    if ((ret = pool_acquire(scene->device, 256 + A.bytes, pb.buf)) != YR_OK) return done(ret);
    char *blk = (char *)pb.buf.p;
    double *d_loss = (double *)blk;
    cudaMemsetAsync(d_loss, 0, sizeof(double), st);
    if ((ret = enqueue_backward(scene, A, blk + 256, desc, dparams, d_loss, st)) != YR_OK) return done(ret);
    if (loss_out) {
        double l = 0.0;
        if (cudaMemcpyAsync(&l, d_loss, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return done(YR_ERR_CUDA);
        *loss_out = (float)l;
    }
    return done(take_status(scene, st));
}

YR_API yr_status yr_backward_batch(yr_scene *const *scenes, uint32_t count, const yr_backward_desc *descs,
                                   float *const *dparams, float *losses, int32_t streams, void *stream) {
    if (!scenes || !descs || !dparams || count == 0) return YR_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < count; i++)
        if (!scenes[i] || !descs[i].image || !descs[i].target || (!dparams[i] && scenes[i]->nparams) ||
            scenes[i]->device != scenes[0]->device)
            return YR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_adj_mu);
    int prev = 0;
    cudaGetDevice(&prev);
    const int device = scenes[0]->device;
    cudaSetDevice(device);
    auto done = [&](yr_status e) {
        cudaSetDevice(prev);
        return e;
    };
    cudaStream_t st = (cudaStream_t)stream;
    const int nl = std::max(1, std::min<int>(streams > 0 ? streams : 8, (int)count));
    std::vector<uintptr_t> key{(uintptr_t)device, (uintptr_t)nl};
    for (uint32_t i = 0; i < count; i++) key.push_back((uintptr_t)scenes[i]);
    std::unique_ptr<AdjBatch> &slot = g_adj_batches[key];
    const size_t lane_budget = render_budget(nl);
    yr_status ret;
    if (slot)
        for (uint32_t i = 0; i < count && slot; i++)
            if (std::memcmp(&slot->h_scenes[i], &scenes[i]->dev, sizeof(DevScene)) ||
                std::memcmp(&slot->h_renders[i], &scenes[i]->rdr, sizeof(DevRender)))
                slot.reset();
    if (!slot) {
        std::unique_ptr<AdjBatch> B(new AdjBatch);
        B->device = device;
        B->scenes.assign(scenes, scenes + count);
        B->plans.resize(count);
        B->fwave.resize(count);
        B->h_scenes.resize(count);
        B->h_renders.resize(count);
        std::vector<double> cost(count);
        for (uint32_t i = 0; i < count; i++) {
            if ((ret = adj_plan(scenes[i], lane_budget, B->plans[i])) != YR_OK) return done(ret);
            const Plan &P = B->plans[i].P;
            B->fwave[i] = std::max(scenes[i]->rdr.spp, wave_for_budget(P, scenes[i]->rdr, lane_budget));
            std::memcpy(&B->h_scenes[i], &scenes[i]->dev, sizeof(DevScene));
            std::memcpy(&B->h_renders[i], &scenes[i]->rdr, sizeof(DevRender));
            cost[i] = (double)P.total * (1.0 + P.ns) * (1.0 + P.npath * (double)P.depth * (1.0 + P.ns));
        }
        if (cudaMalloc(&B->d_loss, sizeof(double) * count) != cudaSuccess ||
            cudaMalloc(&B->d_rays, sizeof(unsigned long long) * 4 * count) != cudaSuccess ||
            cudaMalloc(&B->d_kst, sizeof(unsigned long long) * 3 * YR_K_COUNT) != cudaSuccess ||
            cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming) != cudaSuccess)
            return done(YR_ERR_OUT_OF_MEMORY);
        std::vector<uint32_t> order(count);
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
        B->lanes.resize(nl);
        std::vector<double> load(nl, 0.0);
        for (uint32_t s : order) {
            const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            B->lanes[k].scenes.push_back(s);
            load[k] += cost[s];
        }
        for (AdjLane &l : B->lanes) {
            if (cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) != cudaSuccess)
                return done(YR_ERR_CUDA);
            size_t need = 0;
            for (uint32_t s : l.scenes)
                need = std::max(need, std::max(B->plans[s].bytes, wave_bytes(B->plans[s].P, B->fwave[s])));
            if (need && cudaMalloc(&l.scratch, need) != cudaSuccess) return done(YR_ERR_OUT_OF_MEMORY);
        }
        slot = std::move(B);
    }
    AdjBatch &B = *slot;
    bool same = B.descs.size() == count && B.grads.size() == count;
    for (uint32_t i = 0; same && i < count; i++)
        same = B.descs[i].image == descs[i].image && B.descs[i].target == descs[i].target &&
               B.descs[i].loss_scale == descs[i].loss_scale && B.grads[i] == dparams[i];
    if (!same || !B.graph) {
        B.descs.assign(descs, descs + count);
        B.grads.assign(dparams, dparams + count);
        if ((ret = adj_batch_capture(B)) != YR_OK) return done(ret);
    }
    if (cudaGraphLaunch(B.graph, st) != cudaSuccess) return done(YR_ERR_CUDA);
    for (yr_scene *sc : B.scenes)
        if ((ret = take_status(sc, st)) != YR_OK) return done(ret);
    if (losses) {
        std::vector<double> l(count);
        if (cudaMemcpy(l.data(), B.d_loss, sizeof(double) * count, cudaMemcpyDeviceToHost) != cudaSuccess)
            return done(YR_ERR_CUDA);
        for (uint32_t i = 0; i < count; i++) losses[i] = (float)l[i];
    }
    return done(YR_OK);
}

}  // extern "C"
