// kd-tree build on the GPU: the trees of the host build (kdTree_t,
// kdtree.cc:57-582, node for node, leaf lists in the same order) for many
// meshes at once.
//
// The build goes down the trees one depth at a time over all meshes:
//   - nodes of more than 128 triangles (the binned "pigeonhole" sweep,
//     kdTree_t::pigeonMinCost, kdtree.cc:167-304): one CTA per (node, axis)
//     bins the node's triangles in list order, one CTA per node partitions
//     them (stable: the reference's child lists keep the parent's order);
//   - nodes of at most 128 triangles: one thread per node clips
//     (triBoxClip for at most 32, kdtree.cc:430-470), runs the exact sorted
//     sweep (kdTree_t::minimalCost, kdtree.cc:311-406) and writes the
//     child lists in the sorted-edge order the reference builds them in.
// Every node gets a record (split or leaf); subtree sizes bottom-up and
// depth-first positions top-down then give the reference's node order
// (left child next, right child index stored) and leaf list offsets.
//
// Exactness.  The bin bookkeeping of the binned sweep depends on the order
// in which a bin sees its edges (a flat triangle above the bin's current
// split value moves it without flushing the counters), so each batch of
// 512 triangles sorts its 1024 edge events by (bin, event index) and the
// first thread of each bin's run applies them in list order.  Costs are
// the host build's float expressions (the shipped build's -ffast-math
// forms), compiled unfused; the best split is the earliest one with the
// lowest cost, as the sequential loops keep it.  The sorted sweep uses
// kd_sort (the reference library's std::sort permutation, which fixes the
// order of equal edges and so of the child lists) and kd_clip_triangle,
// both shared with the host build.  Node ids and list offsets come from
// atomic counters; they only label records, the output order comes from
// the tree shape alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "host_build.h"
#include "kd_clip.h"
#include "kd_sort.h"

namespace yr {
namespace {

constexpr int kBins = 1024;             // KD_BINS (kdtree.cc:17)
constexpr uint32_t kClipThresh = 32;    // TRI_CLIP_THRESH (kdtree.cc:16)
constexpr uint32_t kPigeonThresh = 128;
constexpr int kBinThreads = 512;        // one CTA per (node, axis)
constexpr int kChunk = 512;             // triangles per binning batch
constexpr int kEvents = 2 * kChunk;     // lower and upper edge of each
constexpr int kPartThreads = 1024;
constexpr int kScanThreads = 1024;
constexpr int kSmallThreads = 128;
constexpr int kSmallCtasPerSm = 8;
constexpr uint32_t kEdgeCap = 2 * kPigeonThresh;  // candidates of one axis of a small node
constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kSmallList = 0x80000000u;  // list offset flag: next depth's small-node lists
constexpr uint32_t kPoolList = 0x40000000u;   // list offset flag: leaf pool
constexpr int kErrBadTree = 1;

struct ObjP {
    float tb[6];  // grown tree bound: min xyz, max xyz
    float cost_ratio, ebonus;
    int max_depth, max_leaf;
    uint32_t tri_base, ntris;
    uint32_t nbase, pbase;  // first node / triangle of this tree in the output
};

struct BigNode {  // a node and its triangle list (global triangle indices)
    float nb[6];
    uint32_t obj, depth, bad, beg, cnt, id;
};

struct AxisBest {
    float cost, t;
    int found, pad;
};

struct Decision {
    int axis;  // -1: leaf
    float t;
    uint32_t bad, nl, nr;
    uint32_t dst_l, dst_r;  // list offsets with kSmallList / kPoolList, else next big lists
    uint32_t pad;
};

struct NodeRec {
    uint32_t kind;  // 0 split, 1 leaf
    uint32_t axis;
    float t;
    uint32_t left, right;  // children (split)
    uint32_t cnt, pool;    // triangles and their place in the leaf pool (leaf)
    uint32_t obj;
};

// Counters of one depth step: the big nodes of the next depth (from the
// CTA scan), the small nodes of the next depth, the leaf pool and the node
// ids (atomic; pool and ids cumulative).
struct Totals {
    uint32_t nnext, next_refs;
    uint32_t nsmall, small_refs;
    uint32_t pool, nids;
    uint32_t pad[2];
};

__device__ __forceinline__ float dmin3(float a, float b, float c) {
    return (a > b) ? ((b > c) ? c : b) : ((a > c) ? c : a);
}
__device__ __forceinline__ float dmax3(float a, float b, float c) {
    return (a < b) ? ((b > c) ? b : c) : ((a > c) ? a : c);
}

__device__ __forceinline__ uint32_t *list_ptr(uint32_t off, uint32_t *big, uint32_t *small, uint32_t *pool) {
    if (off & kSmallList) return small + (off & ~kSmallList);
    if (off & kPoolList) return pool + (off & ~kPoolList);
    return big + off;
}

// Exclusive scan of K values per thread over a CTA of NT threads;
// `total` receives the CTA sums.  smem: K*32 words.
template <int NT, int K>
__device__ void block_scan(uint32_t (&v)[K], uint32_t (&total)[K], uint32_t *smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl[K];
    for (int k = 0; k < K; k++) {
        uint32_t x = v[k];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        incl[k] = x;
        if (lane == 31) smem[k * 32 + warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        for (int k = 0; k < K; k++) {
            uint32_t x = lane < NT / 32 ? smem[k * 32 + lane] : 0u;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            smem[k * 32 + lane] = x;
        }
    }
    __syncthreads();
    for (int k = 0; k < K; k++) {
        const uint32_t before = warp ? smem[k * 32 + warp - 1] : 0u;
        total[k] = smem[k * 32 + NT / 32 - 1];
        v[k] = before + incl[k] - v[k];
    }
    __syncthreads();
}

// --------------------------------------------------------------- set-up
__global__ void k_tri_bounds(const float *__restrict__ verts, const uint32_t *__restrict__ tris, uint32_t n,
                             float *__restrict__ bnd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *A = verts + 3 * (size_t)tris[3 * (size_t)i];
    const float *B = verts + 3 * (size_t)tris[3 * (size_t)i + 1];
    const float *C = verts + 3 * (size_t)tris[3 * (size_t)i + 2];
    for (int k = 0; k < 3; k++) {
        bnd[6 * (size_t)i + k] = dmin3(A[k], B[k], C[k]);
        bnd[6 * (size_t)i + 3 + k] = dmax3(A[k], B[k], C[k]);
    }
}

// Bound of each mesh's triangle bounds (one CTA per mesh).
__global__ void k_obj_bounds(const float *__restrict__ bnd, const ObjP *__restrict__ op, float *__restrict__ out) {
    __shared__ float red[6][32];
    const ObjP P = op[blockIdx.x];
    float b[6];
    for (int k = 0; k < 6; k++) b[k] = bnd[6 * (size_t)P.tri_base + k];
    for (uint32_t i = threadIdx.x; i < P.ntris; i += blockDim.x) {
        const float *c = bnd + 6 * (size_t)(P.tri_base + i);
        for (int k = 0; k < 3; k++) {
            b[k] = (b[k] < c[k]) ? b[k] : c[k];
            b[3 + k] = (b[3 + k] > c[3 + k]) ? b[3 + k] : c[3 + k];
        }
    }
    for (int o = 16; o > 0; o >>= 1)
        for (int k = 0; k < 6; k++) {
            const float y = __shfl_down_sync(0xffffffffu, b[k], o);
            b[k] = k < 3 ? ((b[k] < y) ? b[k] : y) : ((b[k] > y) ? b[k] : y);
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 6; k++) red[k][warp] = b[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++)
            for (int k = 0; k < 6; k++)
                b[k] = k < 3 ? ((b[k] < red[k][w]) ? b[k] : red[k][w]) : ((b[k] > red[k][w]) ? b[k] : red[k][w]);
        for (int k = 0; k < 6; k++) out[6 * blockIdx.x + k] = b[k];
    }
}

// One edge event of kdTree_t::pigeonMinCost's bin bookkeeping
// (kdtree.cc:191-240) on bin b; kind 0 lower edge, 1 flat triangle, 2 upper
// edge.  The result depends on the order of a bin's events.
__device__ __forceinline__ void bin_apply(uint32_t b, float x, int kind, float *bt, int *bn, int *bcl, int *bcr,
                                          int *bcb, int *bcbl) {
    if (kind == 1) {
        if (bn[b] == 0 || x >= bt[b]) {
            bt[b] = x;
            bcb[b]++;
        } else {
            bcl[b]++;
            bcr[b]++;
        }
        bn[b] += 2;
    } else if (kind == 0) {
        if (bn[b] == 0 || x > bt[b]) {
            bt[b] = x;
            bcl[b] += bcb[b] + bcbl[b];
            bcr[b] += bcb[b];
            bcb[b] = bcbl[b] = 0;
            bcbl[b]++;
        } else if (x == bt[b]) {
            bcbl[b]++;
        } else {
            bcl[b]++;
        }
        bn[b]++;
    } else {
        bcr[b]++;
        if (bn[b] == 0 || x > bt[b]) {
            bt[b] = x;
            bcl[b] += bcb[b] + bcbl[b];
            bcr[b] += bcb[b];
            bcb[b] = bcbl[b] = 0;
        }
        bn[b]++;
    }
}

// The sweep over the 1025 bins of kdTree_t::pigeonMinCost (kdtree.cc:
// 243-300) by a CTA of kBinThreads: thread t owns bins [3t, 3t+3); the
// earliest bin of the lowest cost goes to *outp.
__device__ void bin_sweep(const BigNode &nd, const ObjP &P, int axis, const float *bt, const int *bn, const int *bcl,
                          const int *bcr, const int *bcb, const int *bcbl, uint32_t *scan_smem, float *red_c,
                          int *red_i, AxisBest *outp, int *err) {
    const int tid = threadIdx.x;
    const uint32_t np = nd.cnt;
    const float d[3] = {nd.nb[3] - nd.nb[0], nd.nb[4] - nd.nb[1], nd.nb[5] - nd.nb[2]};
    const float lo = nd.nb[axis], hi = nd.nb[3 + axis];
    const int b0 = 3 * tid, b1 = min(b0 + 3, kBins + 1);
    uint32_t v[2] = {0u, 0u}, tot[2];
    for (int b = b0; b < b1; b++) {
        v[0] += (uint32_t)(bcl[b] + bcb[b] + bcbl[b]);
        v[1] += (uint32_t)(bcr[b] + bcb[b]);
    }
    block_scan<kBinThreads, 2>(v, tot, scan_smem);
    uint32_t below = v[0], above = np - v[1];
    const float eb = (float)((double)P.ebonus * (1.1 - (double)((float)nd.depth / (float)P.max_depth)));
    const float inv_sa = 1.0f / ((d[1] + d[2]) * d[0] + d[1] * d[2]);  // fast-math form
    const float cap_area = d[(axis + 1) % 3] * d[(axis + 2) % 3];
    const float cap_perim = d[(axis + 1) % 3] + d[(axis + 2) % 3];
    const float rd = 1.0f / d[axis];
    float bc = __int_as_float(0x7f800000);
    int bi = 0x7fffffff;
    for (int b = b0; b < b1; b++) {
        if (bn[b] == 0) continue;
        below += (uint32_t)bcl[b];
        above -= (uint32_t)bcr[b];
        const float et = bt[b];
        if (et > lo && et < hi) {
            const float l1 = et - lo, l2 = hi - et;
            const float below_sa = cap_area + l1 * cap_perim;
            const float above_sa = cap_area + l2 * cap_perim;
            const float raw = below_sa * below + above_sa * above;
            float net;
            if (above == 0) net = raw * (1.0f - (l2 * rd + 0.1f) * eb);
            else if (below == 0) net = raw * (1.0f - (l1 * rd + 0.1f) * eb);
            else net = raw;
            const float cost = P.cost_ratio + inv_sa * net;
            if (cost < bc) {
                bc = cost;
                bi = b;
            }
        }
        below += (uint32_t)(bcb[b] + bcbl[b]);
        above -= (uint32_t)bcb[b];
    }
    if (b0 <= kBins && b1 == kBins + 1 && (below != np || above != 0)) atomicExch(err, kErrBadTree);
    // earliest bin of the lowest cost
    for (int o = 16; o > 0; o >>= 1) {
        const float c2 = __shfl_down_sync(0xffffffffu, bc, o);
        const int i2 = __shfl_down_sync(0xffffffffu, bi, o);
        if (c2 < bc || (c2 == bc && i2 < bi)) {
            bc = c2;
            bi = i2;
        }
    }
    if ((tid & 31) == 0) {
        red_c[tid >> 5] = bc;
        red_i[tid >> 5] = bi;
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < kBinThreads / 32; w++)
            if (red_c[w] < bc || (red_c[w] == bc && red_i[w] < bi)) {
                bc = red_c[w];
                bi = red_i[w];
            }
        const bool found = bi <= kBins && bc < __int_as_float(0x7f800000);
        *outp = AxisBest{bc, found ? bt[bi] : 0.f, found ? 1 : 0, 0};
    }
}

// ------------------------------------------------ phase A: binned sweep
// One CTA per (node, axis): the bins of kdTree_t::pigeonMinCost filled in
// list order, then the sweep over the 1025 bins.
__global__ void __launch_bounds__(kBinThreads) k_bin(const BigNode *__restrict__ nodes, const uint32_t *__restrict__ refs,
                                                     const float *__restrict__ bnd, const ObjP *__restrict__ op,
                                                     AxisBest *__restrict__ best, int *__restrict__ err) {
    __shared__ float bt[kBins + 1];
    __shared__ int bn[kBins + 1], bcl[kBins + 1], bcr[kBins + 1], bcb[kBins + 1], bcbl[kBins + 1];
    __shared__ uint32_t key[kEvents];
    __shared__ float epos[kEvents];
    __shared__ uint8_t eflat[kChunk];
    __shared__ uint32_t scan_smem[2 * 32];
    __shared__ float red_c[kBinThreads / 32];
    __shared__ int red_i[kBinThreads / 32];

    const uint32_t node = blockIdx.x / 3;
    const int axis = blockIdx.x % 3;
    const BigNode nd = nodes[node];
    const ObjP P = op[nd.obj];
    AxisBest *outp = best + blockIdx.x;
    if (nd.cnt <= (uint32_t)P.max_leaf || (int)nd.depth >= P.max_depth) {
        if (threadIdx.x == 0) *outp = AxisBest{0.f, 0.f, 0, 0};
        return;
    }
    const int tid = threadIdx.x;
    for (int b = tid; b <= kBins; b += kBinThreads) {
        bt[b] = 0.f;
        bn[b] = bcl[b] = bcr[b] = bcb[b] = bcbl[b] = 0;
    }
    const float d[3] = {nd.nb[3] - nd.nb[0], nd.nb[4] - nd.nb[1], nd.nb[5] - nd.nb[2]};
    const float s = kBins / d[axis];
    const float lo = nd.nb[axis];
    const uint32_t np = nd.cnt;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < np; c0 += kChunk) {
        uint32_t k0 = kNone, k1 = kNone;
        if (c0 + tid < np) {
            const uint32_t p = refs[nd.beg + c0 + tid];
            const float tl = bnd[6 * (size_t)p + axis], tu = bnd[6 * (size_t)p + 3 + axis];
            int bl = (int)((tl - lo) * s), br = (int)((tu - lo) * s);
            bl = bl < 0 ? 0 : (bl > kBins ? kBins : bl);
            br = br < 0 ? 0 : (br > kBins ? kBins : br);
            epos[2 * tid] = tl;
            epos[2 * tid + 1] = tu;
            const bool flat = tl == tu;
            eflat[tid] = flat;
            k0 = ((uint32_t)bl << 11) | (uint32_t)(2 * tid);
            if (!flat) k1 = ((uint32_t)br << 11) | (uint32_t)(2 * tid + 1);
        }
        key[2 * tid] = k0;
        key[2 * tid + 1] = k1;
        __syncthreads();
        // bitonic sort of the 1024 keys (unique: the event index is part of the key)
        for (int k = 2; k <= kEvents; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                const int i = 2 * tid - (tid & (j - 1));
                const int l = i + j;
                const uint32_t a = key[i], b = key[l];
                if ((a > b) == ((i & k) == 0)) {
                    key[i] = b;
                    key[l] = a;
                }
                __syncthreads();
            }
        // the first event of each bin's run applies the run in list order
        for (int q = tid; q < kEvents; q += kBinThreads) {
            const uint32_t kq = key[q];
            if (kq == kNone) continue;
            const uint32_t b = kq >> 11;
            if (q > 0 && (key[q - 1] >> 11) == b) continue;
            for (int m = q; m < kEvents && key[m] != kNone && (key[m] >> 11) == b; m++) {
                const uint32_t ev = key[m] & 2047u;
                bin_apply(b, epos[ev], eflat[ev >> 1] ? 1 : (int)(ev & 1u) * 2, bt, bn, bcl, bcr, bcb, bcbl);
            }
        }
        __syncthreads();
    }
    bin_sweep(nd, P, axis, bt, bn, bcl, bcr, bcb, bcbl, scan_smem, red_c, red_i, outp, err);
}

// The same binned sweep for a depth with few large nodes, spread over all
// SMs: every 512-triangle batch of every (node, axis) sorts its events by
// (bin, event index) in its own CTA (k_wide_sort), the per-batch bin counts
// give every event its place in bin-major, list order (k_wide_offsets,
// k_wide_scatter), and one thread per bin applies its events in that order
// (k_wide_apply) before the usual sweep.
struct WideBatch {
    uint32_t node, axis, c0;  // node, axis, first list position of the batch
    uint32_t row;             // this batch's row in the count / offset tables
};

struct WideSet {  // one (node, axis)
    uint32_t row0, nrows;     // its batches' rows
    uint32_t ev0;             // first of its events in the event array
    uint32_t pad;
};

__global__ void __launch_bounds__(kBinThreads) k_wide_sort(const WideBatch *__restrict__ batches,
                                                           const BigNode *__restrict__ nodes,
                                                           const uint32_t *__restrict__ refs, const float *__restrict__ bnd,
                                                           uint32_t *__restrict__ hist, uint2 *__restrict__ sorted) {
    __shared__ uint32_t key[kEvents];
    __shared__ float epos[kEvents];
    const WideBatch W = batches[blockIdx.x];
    const BigNode nd = nodes[W.node];
    const int axis = (int)W.axis, tid = threadIdx.x;
    const float d = nd.nb[3 + axis] - nd.nb[axis];
    const float s = kBins / d, lo = nd.nb[axis];
    uint32_t k0 = kNone, k1 = kNone;
    if (W.c0 + tid < nd.cnt) {  // as k_bin
        const uint32_t p = refs[nd.beg + W.c0 + tid];
        const float tl = bnd[6 * (size_t)p + axis], tu = bnd[6 * (size_t)p + 3 + axis];
        int bl = (int)((tl - lo) * s), br = (int)((tu - lo) * s);
        bl = bl < 0 ? 0 : (bl > kBins ? kBins : bl);
        br = br < 0 ? 0 : (br > kBins ? kBins : br);
        epos[2 * tid] = tl;
        epos[2 * tid + 1] = tu;
        const bool flat = tl == tu;
        k0 = ((uint32_t)bl << 11) | (uint32_t)(2 * tid) | (flat ? 0x80000000u : 0u);
        if (!flat) k1 = ((uint32_t)br << 11) | (uint32_t)(2 * tid + 1);
    }
    key[2 * tid] = k0;
    key[2 * tid + 1] = k1;
    __syncthreads();
    for (int k = 2; k <= kEvents; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int i = 2 * tid - (tid & (j - 1));
            const int l = i + j;
            const uint32_t a = key[i], b = key[l];
            // the flat flag (bit 31) does not take part in the order
            if (((a & 0x7fffffffu) > (b & 0x7fffffffu) || (a == kNone && b != kNone)) == ((i & k) == 0)) {
                key[i] = b;
                key[l] = a;
            }
            __syncthreads();
        }
    for (int q = tid; q < kEvents; q += kBinThreads) {
        const uint32_t kq = key[q];
        sorted[(size_t)W.row * kEvents + q] = make_uint2(kq, kq == kNone ? 0u : __float_as_uint(epos[kq & 2047u]));
        if (kq == kNone) continue;
        const uint32_t b = (kq & 0x7fffffffu) >> 11;
        if (q > 0 && key[q - 1] != kNone && ((key[q - 1] & 0x7fffffffu) >> 11) == b) continue;
        int m = q;
        while (m < kEvents && key[m] != kNone && ((key[m] & 0x7fffffffu) >> 11) == b) m++;
        hist[(size_t)W.row * (kBins + 1) + b] = (uint32_t)(m - q);
    }
}

// Per (node, axis): where each bin's events start (bin-major) and each
// batch's place inside each bin (offsets, same layout as the counts).
// One thread per bin 0..kBins-1 (bin kBins is summed beside the scan), so
// the block is exactly kBins threads.
constexpr int kWideOffsetThreads = 1024;
static_assert(kBins == kWideOffsetThreads, "k_wide_offsets runs one thread per bin");
__global__ void __launch_bounds__(kWideOffsetThreads) k_wide_offsets(const WideSet *__restrict__ sets, const uint32_t *__restrict__ hist,
                                                       uint32_t *__restrict__ offs, uint32_t *__restrict__ bin_start) {
    __shared__ uint32_t smem[32];
    const WideSet S = sets[blockIdx.x];
    const int t = threadIdx.x;
    uint32_t tot1024 = 0;
    uint32_t v[1] = {0u}, sum[1];
    for (uint32_t r = 0; r < S.nrows; r++) {
        v[0] += hist[(size_t)(S.row0 + r) * (kBins + 1) + t];
        if (t == 0) tot1024 += hist[(size_t)(S.row0 + r) * (kBins + 1) + kBins];
    }
    block_scan<1024, 1>(v, sum, smem);
    uint32_t run = v[0];  // bins 0..1023 in order, bin 1024 last
    uint32_t run1024 = sum[0];
    for (uint32_t r = 0; r < S.nrows; r++) {
        const size_t at = (size_t)(S.row0 + r) * (kBins + 1);
        offs[at + t] = run;
        run += hist[at + t];
        if (t == 0) {
            offs[at + kBins] = run1024;
            run1024 += hist[at + kBins];
        }
    }
    bin_start[(size_t)blockIdx.x * (kBins + 2) + t] = v[0];
    if (t == 0) {
        bin_start[(size_t)blockIdx.x * (kBins + 2) + kBins] = sum[0];
        bin_start[(size_t)blockIdx.x * (kBins + 2) + kBins + 1] = sum[0] + tot1024;
    }
}

__global__ void __launch_bounds__(kBinThreads) k_wide_scatter(const WideBatch *__restrict__ batches,
                                                              const WideSet *__restrict__ sets,
                                                              const uint2 *__restrict__ sorted,
                                                              const uint32_t *__restrict__ offs, uint2 *__restrict__ events) {
    __shared__ uint32_t key[kEvents];
    __shared__ int run_start[kBins + 1];
    const WideBatch W = batches[blockIdx.x];
    const WideSet S = sets[3 * W.node + W.axis];
    const int tid = threadIdx.x;
    for (int q = tid; q < kEvents; q += kBinThreads) key[q] = sorted[(size_t)W.row * kEvents + q].x;
    __syncthreads();
    for (int q = tid; q < kEvents; q += kBinThreads) {
        const uint32_t kq = key[q];
        if (kq == kNone) continue;
        const uint32_t b = (kq & 0x7fffffffu) >> 11;
        if (q == 0 || key[q - 1] == kNone || ((key[q - 1] & 0x7fffffffu) >> 11) != b) run_start[b] = q;
    }
    __syncthreads();
    for (int q = tid; q < kEvents; q += kBinThreads) {
        const uint2 e = sorted[(size_t)W.row * kEvents + q];
        if (e.x == kNone) continue;
        const uint32_t b = (e.x & 0x7fffffffu) >> 11;
        const uint32_t ev = e.x & 2047u;
        const uint32_t kind = (e.x & 0x80000000u) ? 1u : (ev & 1u) * 2u;
        const uint32_t dst = offs[(size_t)W.row * (kBins + 1) + b] + (uint32_t)(q - run_start[b]);
        events[S.ev0 + dst] = make_uint2(e.y, (b << 2) | kind);
    }
}

__global__ void __launch_bounds__(kBinThreads) k_wide_apply(const BigNode *__restrict__ nodes, const WideSet *__restrict__ sets,
                                                            const uint32_t *__restrict__ bin_start,
                                                            const uint2 *__restrict__ events, const ObjP *__restrict__ op,
                                                            AxisBest *__restrict__ best, int *__restrict__ err) {
    __shared__ float bt[kBins + 1];
    __shared__ int bn[kBins + 1], bcl[kBins + 1], bcr[kBins + 1], bcb[kBins + 1], bcbl[kBins + 1];
    __shared__ uint32_t scan_smem[2 * 32];
    __shared__ float red_c[kBinThreads / 32];
    __shared__ int red_i[kBinThreads / 32];
    const uint32_t node = blockIdx.x / 3;
    const int axis = blockIdx.x % 3;
    const BigNode nd = nodes[node];
    const ObjP P = op[nd.obj];
    AxisBest *outp = best + blockIdx.x;
    if (nd.cnt <= (uint32_t)P.max_leaf || (int)nd.depth >= P.max_depth) {
        if (threadIdx.x == 0) *outp = AxisBest{0.f, 0.f, 0, 0};
        return;
    }
    const WideSet S = sets[blockIdx.x];
    const uint32_t *bs = bin_start + (size_t)blockIdx.x * (kBins + 2);
    for (int b = threadIdx.x; b <= kBins; b += kBinThreads) {
        bt[b] = 0.f;
        bn[b] = bcl[b] = bcr[b] = bcb[b] = bcbl[b] = 0;
        for (uint32_t i = bs[b]; i < bs[b + 1]; i++) {
            const uint2 e = events[S.ev0 + i];
            bin_apply((uint32_t)b, __uint_as_float(e.x), (int)(e.y & 3u), bt, bn, bcl, bcr, bcb, bcbl);
        }
    }
    __syncthreads();
    bin_sweep(nd, P, axis, bt, bn, bcl, bcr, bcb, bcbl, scan_smem, red_c, red_i, outp, err);
}

// Split or leaf per node (kdTree_t::buildTree, kdtree.cc:416-520): the best
// axis is the first with the lowest cost, as the sequential sweep over the
// axes keeps it.
__global__ void k_decide(const BigNode *__restrict__ nodes, uint32_t n, const AxisBest *__restrict__ best,
                         const ObjP *__restrict__ op, Decision *__restrict__ dec) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const BigNode nd = nodes[k];
    const ObjP P = op[nd.obj];
    Decision D{};
    D.axis = -1;
    D.bad = nd.bad;
    if (!(nd.cnt <= (uint32_t)P.max_leaf || (int)nd.depth >= P.max_depth)) {
        float bc = __int_as_float(0x7f800000), t = 0.f;
        int ax = -1;
        for (int a = 0; a < 3; a++) {
            const AxisBest B = best[3 * k + a];
            if (B.found && B.cost < bc) {
                bc = B.cost;
                t = B.t;
                ax = a;
            }
        }
        const float old = float(nd.cnt);
        uint32_t bad = nd.bad;
        if (bc > old) ++bad;
        if (!((bc > 1.6f * old && nd.cnt < 16) || ax == -1 || bad == 2)) {
            D.axis = ax;
            D.t = t;
            D.bad = bad;
        }
    }
    dec[k] = D;
}

// Child list sizes of each split (CTA per node).
__global__ void __launch_bounds__(kPartThreads) k_count(const BigNode *__restrict__ nodes, const uint32_t *__restrict__ refs,
                                                        const float *__restrict__ bnd, Decision *__restrict__ dec) {
    __shared__ uint32_t smem[2 * 32];
    const Decision D = dec[blockIdx.x];
    if (D.axis < 0) return;
    const BigNode nd = nodes[blockIdx.x];
    uint32_t v[2] = {0u, 0u}, tot[2];
    for (uint32_t i = threadIdx.x; i < nd.cnt; i += kPartThreads) {
        const uint32_t p = refs[nd.beg + i];
        const float a = bnd[6 * (size_t)p + D.axis], g = bnd[6 * (size_t)p + 3 + D.axis];
        const bool r = a >= D.t;
        v[0] += r ? 0u : 1u;
        v[1] += (r || g > D.t) ? 1u : 0u;
    }
    block_scan<kPartThreads, 2>(v, tot, smem);
    if (threadIdx.x == 0) {
        dec[blockIdx.x].nl = tot[0];
        dec[blockIdx.x].nr = tot[1];
    }
}

// Numbering of the next depth (one CTA): larger children get consecutive
// places among the next depth's big nodes (CTA scan); children of at most
// 128 triangles, leaves and node ids take theirs from atomic counters.
__global__ void __launch_bounds__(kScanThreads) k_level(const BigNode *__restrict__ nodes, uint32_t n,
                                                        Decision *__restrict__ dec, BigNode *__restrict__ next,
                                                        BigNode *__restrict__ small_next, NodeRec *__restrict__ rec,
                                                        Totals *__restrict__ tot) {
    __shared__ uint32_t smem[2 * 32];
    __shared__ uint32_t carry[2];
    if (threadIdx.x < 2) carry[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < n; c0 += kScanThreads) {
        const uint32_t k = c0 + threadIdx.x;
        uint32_t v[2] = {0, 0}, sum[2];  // next big nodes, their triangles
        Decision D{};
        BigNode nd{};
        if (k < n) {
            D = dec[k];
            nd = nodes[k];
            if (D.axis >= 0) {
                if (D.nl > kPigeonThresh) {
                    v[0]++;
                    v[1] += D.nl;
                }
                if (D.nr > kPigeonThresh) {
                    v[0]++;
                    v[1] += D.nr;
                }
            }
        }
        block_scan<kScanThreads, 2>(v, sum, smem);
        if (k < n) {
            if (D.axis < 0) {
                const uint32_t off = atomicAdd(&tot->pool, nd.cnt);
                rec[nd.id] = NodeRec{1u, 0u, 0.f, 0u, 0u, nd.cnt, off, nd.obj};
                dec[k].dst_l = off | kPoolList;
            } else {
                uint32_t ni = carry[0] + v[0], no = carry[1] + v[1];
                const uint32_t id0 = atomicAdd(&tot->nids, 2u);
                rec[nd.id] = NodeRec{0u, (uint32_t)D.axis, D.t, id0, id0 + 1, 0u, 0u, nd.obj};
                const uint32_t c[2] = {D.nl, D.nr};
                uint32_t dst[2];
                for (int s = 0; s < 2; s++) {
                    BigNode b;
                    for (int q = 0; q < 6; q++) b.nb[q] = nd.nb[q];
                    if (s == 0) b.nb[3 + D.axis] = D.t;
                    else b.nb[D.axis] = D.t;
                    b.obj = nd.obj;
                    b.depth = nd.depth + 1;
                    b.bad = D.bad;
                    b.cnt = c[s];
                    b.id = id0 + s;
                    if (c[s] <= kPigeonThresh) {
                        b.beg = atomicAdd(&tot->small_refs, c[s]);
                        small_next[atomicAdd(&tot->nsmall, 1u)] = b;
                        dst[s] = b.beg | kSmallList;
                    } else {
                        b.beg = no;
                        next[ni] = b;
                        dst[s] = no;
                        ni++;
                        no += c[s];
                    }
                }
                dec[k].dst_l = dst[0];
                dec[k].dst_r = dst[1];
            }
        }
        __syncthreads();
        if (threadIdx.x < 2) carry[threadIdx.x] += sum[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        tot->nnext = carry[0];
        tot->next_refs = carry[1];
    }
}

// Child lists of each split in list order (CTA per node); a leaf's list
// goes to the leaf pool as it is.
__global__ void __launch_bounds__(kPartThreads) k_scatter(const BigNode *__restrict__ nodes, const uint32_t *__restrict__ refs,
                                                          const float *__restrict__ bnd, const Decision *__restrict__ dec,
                                                          uint32_t *__restrict__ next_refs, uint32_t *__restrict__ small_refs,
                                                          uint32_t *__restrict__ pool) {
    __shared__ uint32_t smem[2 * 32];
    const Decision D = dec[blockIdx.x];
    const BigNode nd = nodes[blockIdx.x];
    if (D.axis < 0) {
        uint32_t *dst = list_ptr(D.dst_l, next_refs, small_refs, pool);
        for (uint32_t i = threadIdx.x; i < nd.cnt; i += kPartThreads) dst[i] = refs[nd.beg + i];
        return;
    }
    uint32_t *dl = list_ptr(D.dst_l, next_refs, small_refs, pool);
    uint32_t *dr = list_ptr(D.dst_r, next_refs, small_refs, pool);
    uint32_t cl = 0, cr = 0;
    for (uint32_t c0 = 0; c0 < nd.cnt; c0 += kPartThreads) {
        const uint32_t i = c0 + threadIdx.x;
        uint32_t p = 0;
        uint32_t v[2] = {0u, 0u}, tot[2];
        if (i < nd.cnt) {
            p = refs[nd.beg + i];
            const float a = bnd[6 * (size_t)p + D.axis], g = bnd[6 * (size_t)p + 3 + D.axis];
            const bool r = a >= D.t;
            v[0] = r ? 0u : 1u;
            v[1] = (r || g > D.t) ? 1u : 0u;
        }
        const uint32_t fl = v[0], fr = v[1];
        block_scan<kPartThreads, 2>(v, tot, smem);
        if (fl) dl[cl + v[0]] = p;
        if (fr) dr[cr + v[1]] = p;
        cl += tot[0];
        cr += tot[1];
    }
}

// ------------------------------------------------ nodes of <= 128 triangles
// One thread per node runs one step of kdTree_t::buildTree (kdtree.cc:
// 416-582): clip, leaf tests, the exact sorted sweep on each axis, the
// chosen axis sorted again for the partition (the same input order gives
// the same permutation), and the child lists in sorted-edge order.  Each
// thread's candidates and clipped bounds live in `edge_scratch` and
// `clip_scratch`, interleaved across the grid.
__global__ void __launch_bounds__(kSmallThreads) k_small(const BigNode *__restrict__ nodes, uint32_t n,
                                                         uint32_t *__restrict__ refs, const float *__restrict__ bnd,
                                                         const float *__restrict__ verts, const uint32_t *__restrict__ tris,
                                                         const ObjP *__restrict__ op, KdEdge8 *__restrict__ edge_scratch,
                                                         float *__restrict__ clip_scratch, BigNode *__restrict__ small_next,
                                                         uint32_t *__restrict__ small_next_refs, uint32_t *__restrict__ pool,
                                                         NodeRec *__restrict__ rec, Totals *__restrict__ tot,
                                                         const uint32_t *__restrict__ order) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
    const KdStrided<KdEdge8> ed{edge_scratch + g, (int)T};
    const KdStrided<float> clipb{clip_scratch + g, (int)T};
    for (uint32_t k = g; k < n; k += T) {
        const BigNode nd = nodes[order[k]];
        const ObjP P = op[nd.obj];
        uint32_t *L = refs + nd.beg;
        uint32_t np = nd.cnt;
        auto leaf = [&]() {
            const uint32_t off = np ? atomicAdd(&tot->pool, np) : 0u;
            for (uint32_t i = 0; i < np; i++) pool[off + i] = L[i];
            rec[nd.id] = NodeRec{1u, 0u, 0.f, 0u, 0u, np, off, nd.obj};
        };
        bool clipped = false;
        if (np <= kClipThresh) {
            double bmin[3], bmax[3];
            for (int i = 0; i < 3; ++i) {
                const double half = (double)nd.nb[3 + i] - (double)nd.nb[i];
                const double tsize = (double)P.tb[3 + i] - (double)P.tb[i];
                const double grow = 0.021 * half + 0.00001 * tsize;  // fast-math form
                bmin[i] = (double)nd.nb[i] - grow;
                bmax[i] = (double)nd.nb[3 + i] + grow;
            }
            uint32_t kept = 0;
            for (uint32_t i = 0; i < np; i++) {
                const uint32_t pn = L[i];
                double v[3][3];
                for (int j = 0; j < 3; ++j) {
                    const float *V = verts + 3 * (size_t)tris[3 * (size_t)pn + j];
                    v[j][0] = V[0];
                    v[j][1] = V[1];
                    v[j][2] = V[2];
                }
                float cl[3], ch[3];
                const int res = kd_clip_triangle(bmin, bmax, v, cl, ch);
                if (res == 1) continue;
                for (int q = 0; q < 3; q++) {
                    clipb[6 * kept + q] = res == 0 ? cl[q] : bnd[6 * (size_t)pn + q];
                    clipb[6 * kept + 3 + q] = res == 0 ? ch[q] : bnd[6 * (size_t)pn + 3 + q];
                }
                L[kept++] = pn;
            }
            np = kept;
            clipped = true;
        }
        if (np <= (uint32_t)P.max_leaf || (int)nd.depth >= P.max_depth) {
            leaf();
            continue;
        }
        const float eb = (float)((double)P.ebonus * (1.1 - (double)((float)nd.depth / (float)P.max_depth)));
        const float d[3] = {nd.nb[3] - nd.nb[0], nd.nb[4] - nd.nb[1], nd.nb[5] - nd.nb[2]};
        const float old = float(np);
        float bc = __int_as_float(0x7f800000);
        int ax = -1, off = -1, nedge = 0;
        const float inv_sa = 1.0f / ((d[1] + d[2]) * d[0] + d[1] * d[2]);  // fast-math form
        // this node's candidates on `axis`, sorted (kdtree.cc:330-350)
        auto candidates = [&](int axis) {
            int ne = 0;
            for (uint32_t i = 0; i < np; i++) {
                const uint32_t pn = L[i];
                const float a = clipped ? clipb[6 * i + axis] : bnd[6 * (size_t)pn + axis];
                const float gg = clipped ? clipb[6 * i + 3 + axis] : bnd[6 * (size_t)pn + 3 + axis];
                if (a == gg) {
                    ed[ne++] = KdEdge8{a, (pn << 2) | 1u};
                } else {
                    ed[ne++] = KdEdge8{a, pn << 2};
                    ed[ne++] = KdEdge8{gg, (pn << 2) | 2u};
                }
            }
            kd_sort<16>(ed, ne);  // ne <= 256
            return ne;
        };
        for (int axis = 0; axis < 3; axis++) {
            const int ne = candidates(axis);
            const float cap_area = d[(axis + 1) % 3] * d[(axis + 2) % 3];
            const float cap_perim = d[(axis + 1) % 3] + d[(axis + 2) % 3];
            uint32_t below = 0, above = np;
            const float lo = nd.nb[axis], hi = nd.nb[3 + axis];
            for (int i = 0; i < ne; ++i) {
                const KdEdge8 e = ed[i];
                const uint32_t end = e.pe & 3u;
                if (end == 2) --above;
                const float et = e.pos;
                if (et > lo && et < hi) {
                    const float l1 = et - lo, l2 = hi - et;
                    const float below_sa = cap_area + l1 * cap_perim;
                    const float above_sa = cap_area + l2 * cap_perim;
                    const float raw = below_sa * below + above_sa * above;
                    float net;
                    if (above == 0) net = raw * (1.0f - (l2 / d[axis] + 0.1f) * eb);
                    else if (below == 0) net = raw * (1.0f - (l1 / d[axis] + 0.1f) * eb);
                    else net = raw;
                    const float cost = P.cost_ratio + inv_sa * net;
                    if (cost < bc) {
                        bc = cost;
                        ax = axis;
                        off = i;
                        nedge = ne;
                    }
                }
                if (end != 2) {
                    ++below;
                    if (end == 1) --above;
                }
            }
        }
        uint32_t bad = nd.bad;
        if (bc > old) ++bad;
        if ((bc > 1.6f * old && np < 16) || ax == -1 || bad == 2) {
            leaf();
            continue;
        }
        if (ax != 2) candidates(ax);
        const float split = ed[off].pos;
        uint32_t nl = 0, nr = 0;
        for (int i = 0; i < off; ++i)
            if ((ed[i].pe & 3u) != 2) nl++;
        if ((ed[off].pe & 3u) == 1) nr++;
        for (int i = off + 1; i < nedge; ++i)
            if ((ed[i].pe & 3u) != 0) nr++;
        const uint32_t id0 = atomicAdd(&tot->nids, 2u);
        const uint32_t bl = atomicAdd(&tot->small_refs, nl + nr);
        const uint32_t slot = atomicAdd(&tot->nsmall, 2u);
        uint32_t *Lo = small_next_refs + bl, *Ro = Lo + nl;
        uint32_t a = 0, b = 0;
        for (int i = 0; i < off; ++i)
            if ((ed[i].pe & 3u) != 2) Lo[a++] = ed[i].pe >> 2;
        if ((ed[off].pe & 3u) == 1) Ro[b++] = ed[off].pe >> 2;
        for (int i = off + 1; i < nedge; ++i)
            if ((ed[i].pe & 3u) != 0) Ro[b++] = ed[i].pe >> 2;
        rec[nd.id] = NodeRec{0u, (uint32_t)ax, split, id0, id0 + 1, 0u, 0u, nd.obj};
        BigNode c;
        for (int q = 0; q < 6; q++) c.nb[q] = nd.nb[q];
        c.obj = nd.obj;
        c.depth = nd.depth + 1;
        c.bad = bad;
        c.nb[3 + ax] = split;
        c.beg = bl;
        c.cnt = nl;
        c.id = id0;
        small_next[slot] = c;
        c.nb[3 + ax] = nd.nb[3 + ax];
        c.nb[ax] = split;
        c.beg = bl + nl;
        c.cnt = nr;
        c.id = id0 + 1;
        small_next[slot + 1] = c;
    }
}

// Order of the small nodes for k_small: largest lists first, so that the
// threads of a warp get nodes of similar size (their sorts then run for
// similar lengths) and the longest nodes start first.  Counting sort over
// the list sizes 0..128; the order inside a size is free.
// Lanes of a warp holding the same size share one atomic.
__device__ __forceinline__ uint32_t size_slot(uint32_t *hist, uint32_t c) {
    const unsigned m = __match_any_sync(__activemask(), c);
    const int lane = (int)(threadIdx.x & 31u), leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&hist[c], (uint32_t)__popc(m));
    base = __shfl_sync(m, base, leader);
    return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

__global__ void k_size_hist(const BigNode *__restrict__ nodes, uint32_t n, uint32_t *__restrict__ hist) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) size_slot(hist, nodes[i].cnt);
}

__global__ void k_size_scan(uint32_t *__restrict__ hist) {  // one thread
    uint32_t run = 0;
    for (int c = (int)kPigeonThresh; c >= 0; c--) {
        const uint32_t h = hist[c];
        hist[c] = run;
        run += h;
    }
}

__global__ void k_size_scatter(const BigNode *__restrict__ nodes, uint32_t n, uint32_t *__restrict__ hist,
                               uint32_t *__restrict__ perm) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[size_slot(hist, nodes[i].cnt)] = i;
}

// ------------------------------------------------------------ node order
__global__ void k_sizes_up(const NodeRec *__restrict__ rec, uint32_t lo, uint32_t hi, uint2 *__restrict__ size) {
    const uint32_t id = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= hi) return;
    const NodeRec r = rec[id];
    if (r.kind == 1) {
        size[id] = make_uint2(1u, r.cnt > 1 ? r.cnt : 0u);
        return;
    }
    const uint2 a = size[r.left], b = size[r.right];
    size[id] = make_uint2(1u + a.x + b.x, a.y + b.y);
}

__global__ void k_place_down(const NodeRec *__restrict__ rec, uint32_t lo, uint32_t hi, const uint2 *__restrict__ size,
                             uint2 *__restrict__ place) {
    const uint32_t id = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= hi) return;
    const NodeRec r = rec[id];
    if (r.kind != 0) return;
    const uint2 p = place[id], sl = size[r.left];
    place[r.left] = make_uint2(p.x + 1u, p.y);
    place[r.right] = make_uint2(p.x + 1u + sl.x, p.y + sl.y);
}

// Every node in its place (kdTreeNode packing, kdtree.h:23-61): splits
// with the right child's tree-local index, leaves with their triangle or
// their list's offset (the list copied there), mesh-local triangle indices.
__global__ void k_write(const NodeRec *__restrict__ rec, uint32_t nids, const uint2 *__restrict__ place,
                        const ObjP *__restrict__ op, const uint32_t *__restrict__ pool, uint2 *__restrict__ out_nodes,
                        uint32_t *__restrict__ out_prims) {
    const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nids) return;
    const NodeRec r = rec[id];
    const ObjP P = op[r.obj];
    const uint2 p = place[id];
    if (r.kind == 0) {
        out_nodes[P.nbase + p.x] = make_uint2(__float_as_uint(r.t), r.axis | (place[r.right].x << 2));
        return;
    }
    uint32_t word = 0;
    if (r.cnt == 1) word = pool[r.pool] - P.tri_base;
    else if (r.cnt > 1) word = p.y;
    out_nodes[P.nbase + p.x] = make_uint2(word, (r.cnt << 2) | 3u);
    if (r.cnt > 1)
        for (uint32_t i = 0; i < r.cnt; i++) out_prims[P.pbase + p.y + i] = pool[r.pool + i] - P.tri_base;
}

// ------------------------------------------------------------ host side
// Phase timings of a build on stderr, for variant builds only
// (-DYR_KD_PHASE_TIMES): wall time of each phase since the previous mark,
// and the time spent growing device buffers.
#ifdef YR_KD_PHASE_TIMES
static double kd_now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static double g_kd_mark = 0.0, g_kd_alloc = 0.0;
static int g_kd_allocs = 0;
static void kd_phase(const char *name) {
    const double t = kd_now();
    if (name) fprintf(stderr, "kd phase %-14s %8.2f ms (buffer growth so far %d, %.2f ms)\n", name,
                      1e3 * (t - g_kd_mark), g_kd_allocs, 1e3 * g_kd_alloc);
    g_kd_mark = t;
}
#define KD_PHASE(name) kd_phase(name)
#else
#define KD_PHASE(name) ((void)0)
#endif

struct DBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() {
        if (p) cudaFree(p);
    }
    // grow to at least n bytes, keeping the first `keep` bytes
    bool ensure(size_t n, size_t keep, cudaStream_t s) {
        if (n <= bytes) return true;
#ifdef YR_KD_PHASE_TIMES
        const double t0 = kd_now();
        struct Acc {
            double t0;
            ~Acc() {
                g_kd_alloc += kd_now() - t0;
                g_kd_allocs++;
            }
        } acc{t0};
#endif
        const size_t nb = std::max(n, bytes + bytes / 2);
        void *q = nullptr;
        if (cudaMalloc(&q, nb) != cudaSuccess) return false;
        if (keep && p) cudaMemcpyAsync(q, p, std::min(keep, bytes), cudaMemcpyDeviceToDevice, s);
        if (p) {
            cudaStreamSynchronize(s);
            cudaFree(p);
        }
        p = q;
        bytes = nb;
        return true;
    }
    template <class T>
    T *as() const {
        return static_cast<T *>(p);
    }
};

void swap_buf(DBuf &a, DBuf &b) {
    std::swap(a.p, b.p);
    std::swap(a.bytes, b.bytes);
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

inline unsigned blocks(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

namespace {

// Run f(o) for every mesh o on all host cores.
template <class F>
void for_meshes(uint32_t n, F f) {
    unsigned nth = std::thread::hardware_concurrency();
    nth = std::max(1u, std::min(nth ? nth : 1u, n));
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nth; t++)
        pool.emplace_back([&, t] {
            for (uint32_t o = t; o < n; o += nth) f(o);
        });
    for (uint32_t o = 0; o < n; o += nth) f(o);
    for (std::thread &th : pool) th.join();
}

}  // namespace

yr_status build_kdtrees_gpu(const std::vector<KdMesh> &meshes, const KdParams &kp, int device,
                            std::vector<KdTree> &out, yr_kdtree **abi_out) {
    const uint32_t nobj = (uint32_t)meshes.size();
    if (nobj == 0) return YR_ERR_INVALID_ARG;
#ifdef YR_KD_PHASE_TIMES
    g_kd_alloc = 0.0;
    g_kd_allocs = 0;
#endif
    KD_PHASE(nullptr);
    size_t nt = 0, nv = 0;
    for (const KdMesh &m : meshes) {
        if (!m.verts || !m.tris || m.ntris == 0) return YR_ERR_EMPTY_SCENE;
        nt += m.ntris;
        nv += m.nverts;
    }
    {
        std::vector<yr_status> chk(nobj, YR_OK);
        for_meshes(nobj, [&](uint32_t o) {
            const KdMesh &m = meshes[o];
            for (size_t i = 0; i < 3 * (size_t)m.ntris; i++)
                if (m.tris[i] >= m.nverts) {
                    chk[o] = YR_ERR_INVALID_ARG;
                    return;
                }
            // the sweeps need ordered positions: no NaN or infinite coordinate
            for (size_t i = 0; i < 3 * (size_t)m.nverts; i++)
                if (!std::isfinite(m.verts[i])) {
                    chk[o] = YR_ERR_INVALID_ARG;
                    return;
                }
        });
        for (yr_status c : chk)
            if (c != YR_OK) return c;
    }
    KD_PHASE("input checks");
    // candidates pack index << 2; list offsets carry two flag bits
    if (nt >= (1u << 28) || nv >= 0xffffffffu / 3) return YR_ERR_TOO_LARGE;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return YR_ERR_NO_DEVICE;
    DeviceGuard guard(device);
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return YR_ERR_CUDA;
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } sg{st};
    // nodes of at most 128 triangles run on a second stream, beside the
    // binned sweep of the larger ones
    cudaStream_t st2;
    if (cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking) != cudaSuccess) return YR_ERR_CUDA;
    StreamGuard sg2{st2};
    cudaEvent_t ev_go, ev_done;
    if (cudaEventCreateWithFlags(&ev_go, cudaEventDisableTiming) != cudaSuccess) return YR_ERR_CUDA;
    if (cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming) != cudaSuccess) {
        cudaEventDestroy(ev_go);
        return YR_ERR_CUDA;
    }
    struct EventGuard {
        cudaEvent_t a, b;
        ~EventGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } eg{ev_go, ev_done};

    KD_PHASE("streams");
    // inputs: all meshes concatenated, vertex indices made global
    std::vector<float> hv(3 * nv);
    std::vector<uint32_t> ht(3 * nt);
    std::vector<ObjP> hop(nobj);
    {
        std::vector<size_t> vbase(nobj), tbase(nobj);
        size_t vb = 0, tb = 0;
        for (uint32_t o = 0; o < nobj; o++) {
            vbase[o] = vb;
            tbase[o] = tb;
            vb += meshes[o].nverts;
            tb += meshes[o].ntris;
        }
        for_meshes(nobj, [&](uint32_t o) {
            const KdMesh &m = meshes[o];
            std::memcpy(hv.data() + 3 * vbase[o], m.verts, 12 * (size_t)m.nverts);
            for (size_t i = 0; i < 3 * (size_t)m.ntris; i++)
                ht[3 * tbase[o] + i] = (uint32_t)(m.tris[i] + vbase[o]);
            ObjP &P = hop[o];
            std::memset(&P, 0, sizeof(P));
            P.tri_base = (uint32_t)tbase[o];
            P.ntris = m.ntris;
            P.ebonus = kp.empty_bonus;
            kd_limits(m.ntris, kp, P.max_depth, P.max_leaf, P.cost_ratio);
        });
    }
    DBuf d_verts, d_tris, d_bnd, d_op, d_obnd, d_err, d_tot;
    if (!d_verts.ensure(hv.size() * 4, 0, st) || !d_tris.ensure(ht.size() * 4, 0, st) || !d_bnd.ensure(24 * nt, 0, st) ||
        !d_op.ensure(sizeof(ObjP) * nobj, 0, st) || !d_obnd.ensure(24 * (size_t)nobj, 0, st) ||
        !d_err.ensure(4, 0, st) || !d_tot.ensure(sizeof(Totals), 0, st))
        return YR_ERR_OUT_OF_MEMORY;
    cudaMemcpyAsync(d_verts.p, hv.data(), hv.size() * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_tris.p, ht.data(), ht.size() * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_op.p, hop.data(), sizeof(ObjP) * nobj, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_err.p, 0, 4, st);
    k_tri_bounds<<<blocks(nt, 256), 256, 0, st>>>(d_verts.as<float>(), d_tris.as<uint32_t>(), (uint32_t)nt,
                                                  d_bnd.as<float>());
    k_obj_bounds<<<nobj, 256, 0, st>>>(d_bnd.as<float>(), d_op.as<ObjP>(), d_obnd.as<float>());
    std::vector<float> ob(6 * (size_t)nobj);
    cudaMemcpyAsync(ob.data(), d_obnd.p, 24 * (size_t)nobj, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return YR_ERR_CUDA;
    KD_PHASE("pack+upload");
    for (uint32_t o = 0; o < nobj; o++) {
        Box raw;
        std::memcpy(raw.a, &ob[6 * o], 12);
        std::memcpy(raw.g, &ob[6 * o + 3], 12);
        Box g = kd_grow_bound(raw);
        if (g.a[0] == raw.a[0] && g.g[0] == raw.g[0]) {
            // a zero diagonal keeps the bound as accumulated; the signs of
            // its zeros then follow the sequential accumulation order
            const KdMesh &m = meshes[o];
            for (uint32_t i = 0; i < m.ntris; i++)
                for (int k = 0; k < 3; k++) {
                    const float *A = m.verts + 3 * (size_t)m.tris[3 * (size_t)i];
                    const float *B = m.verts + 3 * (size_t)m.tris[3 * (size_t)i + 1];
                    const float *C = m.verts + 3 * (size_t)m.tris[3 * (size_t)i + 2];
                    const float lo = (A[k] > B[k]) ? ((B[k] > C[k]) ? C[k] : B[k]) : ((A[k] > C[k]) ? C[k] : A[k]);
                    const float hi = (A[k] < B[k]) ? ((B[k] > C[k]) ? B[k] : C[k]) : ((A[k] > C[k]) ? A[k] : C[k]);
                    if (i == 0) {
                        raw.a[k] = lo;
                        raw.g[k] = hi;
                    } else {
                        raw.a[k] = (raw.a[k] < lo) ? raw.a[k] : lo;
                        raw.g[k] = (raw.g[k] > hi) ? raw.g[k] : hi;
                    }
                }
            g = kd_grow_bound(raw);
        }
        std::memcpy(hop[o].tb, g.a, 12);
        std::memcpy(hop[o].tb + 3, g.g, 12);
    }

    // depth 0: the roots, above or below the 128-triangle switch
    std::vector<BigNode> hbig, hsmall;
    std::vector<uint32_t> hrefs, hsrefs;
    for (uint32_t o = 0; o < nobj; o++) {
        const ObjP &P = hop[o];
        BigNode b;
        std::memcpy(b.nb, P.tb, 24);
        b.obj = o;
        b.depth = b.bad = 0;
        b.cnt = P.ntris;
        b.id = o;
        std::vector<uint32_t> &r = P.ntris > kPigeonThresh ? hrefs : hsrefs;
        b.beg = (uint32_t)r.size();
        for (uint32_t i = 0; i < P.ntris; i++) r.push_back(P.tri_base + i);
        (P.ntris > kPigeonThresh ? hbig : hsmall).push_back(b);
    }
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
    const size_t small_threads = (size_t)dev_sms * kSmallCtasPerSm * kSmallThreads;
    DBuf d_cur, d_next, d_refs, d_nrefs, d_small, d_small_next, d_srefs, d_srefs_next, d_pool, d_rec, d_best, d_dec,
        d_edges, d_clip, d_hist, d_order, d_wbatch, d_wset, d_whist, d_woffs, d_wsorted, d_wstart, d_wevents;
    if (!d_edges.ensure(sizeof(KdEdge8) * kEdgeCap * small_threads, 0, st) ||
        !d_hist.ensure(4 * (kPigeonThresh + 1), 0, st) ||
        !d_clip.ensure(4 * 6 * kClipThresh * small_threads, 0, st))
        return YR_ERR_OUT_OF_MEMORY;
    uint32_t nbig = (uint32_t)hbig.size(), nsmall = (uint32_t)hsmall.size();
    size_t big_refs = hrefs.size(), small_refs = hsrefs.size();
    if (!d_cur.ensure(sizeof(BigNode) * std::max<size_t>(1, nbig), 0, st) ||
        !d_refs.ensure(4 * std::max<size_t>(1, big_refs), 0, st) ||
        !d_small.ensure(sizeof(BigNode) * std::max<size_t>(1, nsmall), 0, st) ||
        !d_srefs.ensure(4 * std::max<size_t>(1, small_refs), 0, st))
        return YR_ERR_OUT_OF_MEMORY;
    if (nbig) {
        cudaMemcpyAsync(d_cur.p, hbig.data(), sizeof(BigNode) * nbig, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_refs.p, hrefs.data(), 4 * big_refs, cudaMemcpyHostToDevice, st);
    }
    if (nsmall) {
        cudaMemcpyAsync(d_small.p, hsmall.data(), sizeof(BigNode) * nsmall, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_srefs.p, hsrefs.data(), 4 * small_refs, cudaMemcpyHostToDevice, st);
    }
    cudaMemcpyAsync(d_op.p, hop.data(), sizeof(ObjP) * nobj, cudaMemcpyHostToDevice, st);
    Totals T{};
    T.nids = nobj;
    std::vector<uint32_t> level_lo{0}, level_hi{nobj};

    KD_PHASE("roots+buffers");
    // one depth per step, over all meshes
    while (nbig + nsmall > 0) {
        const size_t nodes_now = (size_t)nbig + nsmall, refs_now = big_refs + small_refs;
        if (T.pool + refs_now >= kPoolList || 2 * refs_now >= kPoolList || T.nids + 2 * nodes_now >= 0x7fffffffu)
            return YR_ERR_TOO_LARGE;
        if (!d_rec.ensure(sizeof(NodeRec) * (T.nids + 2 * nodes_now), sizeof(NodeRec) * T.nids, st) ||
            !d_pool.ensure(4 * (T.pool + refs_now), 4 * (size_t)T.pool, st) ||
            !d_small_next.ensure(sizeof(BigNode) * 2 * nodes_now, 0, st) ||
            !d_srefs_next.ensure(4 * 2 * refs_now, 0, st))
            return YR_ERR_OUT_OF_MEMORY;
        if (nsmall && !d_order.ensure(4 * (size_t)nsmall, 0, st)) return YR_ERR_OUT_OF_MEMORY;
        T.nnext = T.next_refs = T.nsmall = T.small_refs = 0;
        cudaMemcpyAsync(d_tot.p, &T, sizeof(T), cudaMemcpyHostToDevice, st);
        cudaEventRecord(ev_go, st);
        cudaStreamWaitEvent(st2, ev_go, 0);
        if (nbig) {
            if (!d_best.ensure(sizeof(AxisBest) * 3 * (size_t)nbig, 0, st) ||
                !d_dec.ensure(sizeof(Decision) * (size_t)nbig, 0, st) ||
                !d_next.ensure(sizeof(BigNode) * 2 * (size_t)nbig, 0, st) || !d_nrefs.ensure(4 * 2 * big_refs, 0, st))
                return YR_ERR_OUT_OF_MEMORY;
            if (big_refs > (size_t)nbig * 8 * kChunk) {
                // large nodes (above 8 batches on average): spread each
                // node's binning over many CTAs
                std::vector<BigNode> hb(nbig);
                cudaMemcpyAsync(hb.data(), d_cur.p, sizeof(BigNode) * nbig, cudaMemcpyDeviceToHost, st);
                if (cudaStreamSynchronize(st) != cudaSuccess) return YR_ERR_CUDA;
                std::vector<WideBatch> wb;
                std::vector<WideSet> ws(3 * (size_t)nbig);
                uint32_t rows = 0, evs = 0;
                for (uint32_t j = 0; j < nbig; j++)
                    for (uint32_t a = 0; a < 3; a++) {
                        WideSet &S = ws[3 * j + a];
                        S.row0 = rows;
                        S.nrows = (hb[j].cnt + kChunk - 1) / kChunk;
                        S.ev0 = evs;
                        S.pad = 0;
                        for (uint32_t r = 0; r < S.nrows; r++) wb.push_back(WideBatch{j, a, r * (uint32_t)kChunk, rows + r});
                        rows += S.nrows;
                        evs += 2 * hb[j].cnt;
                    }
                // twice the need: the next depths' lists are longer (straddling
                // triangles), and each regrowth is a free and a new allocation
                if (!d_wbatch.ensure(2 * sizeof(WideBatch) * wb.size(), 0, st) ||
                    !d_wset.ensure(2 * sizeof(WideSet) * ws.size(), 0, st) ||
                    !d_whist.ensure(2 * 4 * (size_t)rows * (kBins + 1), 0, st) ||
                    !d_woffs.ensure(2 * 4 * (size_t)rows * (kBins + 1), 0, st) ||
                    !d_wsorted.ensure(2 * 8 * (size_t)rows * kEvents, 0, st) ||
                    !d_wstart.ensure(2 * 4 * ws.size() * (kBins + 2), 0, st) ||
                    !d_wevents.ensure(2 * 8 * (size_t)evs, 0, st))
                    return YR_ERR_OUT_OF_MEMORY;
                cudaMemcpyAsync(d_wbatch.p, wb.data(), sizeof(WideBatch) * wb.size(), cudaMemcpyHostToDevice, st);
                cudaMemcpyAsync(d_wset.p, ws.data(), sizeof(WideSet) * ws.size(), cudaMemcpyHostToDevice, st);
                cudaMemsetAsync(d_whist.p, 0, 4 * (size_t)rows * (kBins + 1), st);
                k_wide_sort<<<rows, kBinThreads, 0, st>>>(d_wbatch.as<WideBatch>(), d_cur.as<BigNode>(),
                                                          d_refs.as<uint32_t>(), d_bnd.as<float>(), d_whist.as<uint32_t>(),
                                                          d_wsorted.as<uint2>());
                k_wide_offsets<<<3 * nbig, kWideOffsetThreads, 0, st>>>(d_wset.as<WideSet>(), d_whist.as<uint32_t>(),
                                                          d_woffs.as<uint32_t>(), d_wstart.as<uint32_t>());
                k_wide_scatter<<<rows, kBinThreads, 0, st>>>(d_wbatch.as<WideBatch>(), d_wset.as<WideSet>(),
                                                             d_wsorted.as<uint2>(), d_woffs.as<uint32_t>(),
                                                             d_wevents.as<uint2>());
                k_wide_apply<<<3 * nbig, kBinThreads, 0, st>>>(d_cur.as<BigNode>(), d_wset.as<WideSet>(),
                                                               d_wstart.as<uint32_t>(), d_wevents.as<uint2>(),
                                                               d_op.as<ObjP>(), d_best.as<AxisBest>(), d_err.as<int>());
            } else {
                k_bin<<<3 * nbig, kBinThreads, 0, st>>>(d_cur.as<BigNode>(), d_refs.as<uint32_t>(), d_bnd.as<float>(),
                                                       d_op.as<ObjP>(), d_best.as<AxisBest>(), d_err.as<int>());
            }
            k_decide<<<blocks(nbig, 128), 128, 0, st>>>(d_cur.as<BigNode>(), nbig, d_best.as<AxisBest>(),
                                                        d_op.as<ObjP>(), d_dec.as<Decision>());
            k_count<<<nbig, kPartThreads, 0, st>>>(d_cur.as<BigNode>(), d_refs.as<uint32_t>(), d_bnd.as<float>(),
                                                   d_dec.as<Decision>());
            k_level<<<1, kScanThreads, 0, st>>>(d_cur.as<BigNode>(), nbig, d_dec.as<Decision>(), d_next.as<BigNode>(),
                                                d_small_next.as<BigNode>(), d_rec.as<NodeRec>(), d_tot.as<Totals>());
            k_scatter<<<nbig, kPartThreads, 0, st>>>(d_cur.as<BigNode>(), d_refs.as<uint32_t>(), d_bnd.as<float>(),
                                                     d_dec.as<Decision>(), d_nrefs.as<uint32_t>(),
                                                     d_srefs_next.as<uint32_t>(), d_pool.as<uint32_t>());
        }
        if (nsmall) {
            cudaMemsetAsync(d_hist.p, 0, 4 * (kPigeonThresh + 1), st2);
            k_size_hist<<<blocks(nsmall, 256), 256, 0, st2>>>(d_small.as<BigNode>(), nsmall, d_hist.as<uint32_t>());
            k_size_scan<<<1, 1, 0, st2>>>(d_hist.as<uint32_t>());
            k_size_scatter<<<blocks(nsmall, 256), 256, 0, st2>>>(d_small.as<BigNode>(), nsmall, d_hist.as<uint32_t>(),
                                                                 d_order.as<uint32_t>());
            const unsigned sb = std::min(blocks(nsmall, kSmallThreads), (unsigned)(dev_sms * kSmallCtasPerSm));
            k_small<<<sb, kSmallThreads, 0, st2>>>(
                d_small.as<BigNode>(), nsmall, d_srefs.as<uint32_t>(), d_bnd.as<float>(), d_verts.as<float>(),
                d_tris.as<uint32_t>(), d_op.as<ObjP>(), d_edges.as<KdEdge8>(), d_clip.as<float>(),
                d_small_next.as<BigNode>(), d_srefs_next.as<uint32_t>(), d_pool.as<uint32_t>(), d_rec.as<NodeRec>(),
                d_tot.as<Totals>(), d_order.as<uint32_t>());
        }
        cudaEventRecord(ev_done, st2);
        cudaStreamWaitEvent(st, ev_done, 0);
        const uint32_t nids_before = T.nids;
        int herr = 0;
        cudaMemcpyAsync(&T, d_tot.p, sizeof(T), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&herr, d_err.p, 4, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return YR_ERR_CUDA;
        if (herr) return YR_ERR_BAD_TREE;  // the reference stops there too (kdtree.cc:283-301)
        level_lo.push_back(nids_before);
        level_hi.push_back(T.nids);
        if (nbig) {
            swap_buf(d_cur, d_next);
            swap_buf(d_refs, d_nrefs);
        }
        swap_buf(d_small, d_small_next);
        swap_buf(d_srefs, d_srefs_next);
        nbig = T.nnext;
        big_refs = T.next_refs;
        nsmall = T.nsmall;
        small_refs = T.small_refs;
    }

    KD_PHASE("depths");
    // node order: sizes bottom-up, places top-down, then every node written
    const uint32_t nids = T.nids;
    DBuf d_size, d_place, d_onodes, d_oprims;
    if (!d_size.ensure(8 * (size_t)nids, 0, st) || !d_place.ensure(8 * (size_t)nids, 0, st))
        return YR_ERR_OUT_OF_MEMORY;
    for (size_t L = level_lo.size(); L-- > 0;) {
        const uint32_t lo = level_lo[L], hi = level_hi[L];
        if (hi > lo) k_sizes_up<<<blocks(hi - lo, 256), 256, 0, st>>>(d_rec.as<NodeRec>(), lo, hi, d_size.as<uint2>());
    }
    std::vector<uint2> rs(nobj);
    cudaMemcpyAsync(rs.data(), d_size.p, 8 * (size_t)nobj, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return YR_ERR_CUDA;
    size_t tot_nodes = 0, tot_prims = 0;
    for (uint32_t o = 0; o < nobj; o++) {
        if (rs[o].x >= (1u << 30)) return YR_ERR_TOO_LARGE;
        hop[o].nbase = (uint32_t)tot_nodes;
        hop[o].pbase = (uint32_t)tot_prims;
        tot_nodes += rs[o].x;
        tot_prims += rs[o].y;
    }
    if (tot_nodes >= 0xffffffffu || tot_prims >= 0xffffffffu) return YR_ERR_TOO_LARGE;
    if (!d_onodes.ensure(8 * std::max<size_t>(1, tot_nodes), 0, st) ||
        !d_oprims.ensure(4 * std::max<size_t>(1, tot_prims), 0, st))
        return YR_ERR_OUT_OF_MEMORY;
    cudaMemcpyAsync(d_op.p, hop.data(), sizeof(ObjP) * nobj, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_place.p, 0, 8 * (size_t)nobj, st);
    for (size_t L = 0; L < level_lo.size(); L++) {
        const uint32_t lo = level_lo[L], hi = level_hi[L];
        if (hi > lo)
            k_place_down<<<blocks(hi - lo, 256), 256, 0, st>>>(d_rec.as<NodeRec>(), lo, hi, d_size.as<uint2>(),
                                                               d_place.as<uint2>());
    }
    k_write<<<blocks(nids, 256), 256, 0, st>>>(d_rec.as<NodeRec>(), nids, d_place.as<uint2>(), d_op.as<ObjP>(),
                                               d_pool.as<uint32_t>(), d_onodes.as<uint2>(), d_oprims.as<uint32_t>());
    KD_PHASE("layout");
    // each tree straight into its destination: yr_kdtree records for the
    // caller, or the KdTree vectors
    if (abi_out) {
        for (uint32_t o = 0; o < nobj; o++) abi_out[o] = nullptr;
        for (uint32_t o = 0; o < nobj; o++) {
            yr_kdtree *r = new (std::nothrow) yr_kdtree;
            if (!r) return YR_ERR_OUT_OF_MEMORY;
            std::memset(r, 0, sizeof(*r));
            abi_out[o] = r;
            r->nnodes = rs[o].x;
            r->nprims = rs[o].y;
            r->nodes = new (std::nothrow) yr_kd_node[r->nnodes ? r->nnodes : 1];
            r->prims = new (std::nothrow) uint32_t[r->nprims ? r->nprims : 1];
            if (!r->nodes || !r->prims) return YR_ERR_OUT_OF_MEMORY;
            std::memcpy(r->bound, hop[o].tb, 24);
            r->max_depth = hop[o].max_depth;
            r->max_leaf_size = hop[o].max_leaf;
            r->cost_ratio = hop[o].cost_ratio;
            r->empty_bonus = hop[o].ebonus;
            cudaMemcpyAsync(r->nodes, d_onodes.as<uint2>() + hop[o].nbase, 8 * (size_t)rs[o].x, cudaMemcpyDeviceToHost,
                            st);
            if (rs[o].y)
                cudaMemcpyAsync(r->prims, d_oprims.as<uint32_t>() + hop[o].pbase, 4 * (size_t)rs[o].y,
                                cudaMemcpyDeviceToHost, st);
        }
    } else {
        out.assign(nobj, KdTree());
        for (uint32_t o = 0; o < nobj; o++) {
            KdTree &t = out[o];
            t.nodes.resize(rs[o].x);
            t.prims.resize(rs[o].y);
            cudaMemcpyAsync(t.nodes.data(), d_onodes.as<uint2>() + hop[o].nbase, 8 * (size_t)rs[o].x,
                            cudaMemcpyDeviceToHost, st);
            if (rs[o].y)
                cudaMemcpyAsync(t.prims.data(), d_oprims.as<uint32_t>() + hop[o].pbase, 4 * (size_t)rs[o].y,
                                cudaMemcpyDeviceToHost, st);
            std::memcpy(t.bound.a, hop[o].tb, 12);
            std::memcpy(t.bound.g, hop[o].tb + 3, 12);
            t.max_depth = hop[o].max_depth;
            t.max_leaf_size = hop[o].max_leaf;
            t.cost_ratio = hop[o].cost_ratio;
            t.empty_bonus = hop[o].ebonus;
        }
    }
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return YR_ERR_CUDA;
    KD_PHASE("trees out");
    return YR_OK;
}

}  // namespace yr

YR_API yr_status yr_kdtree_build_gpu(const yr_kdtree_mesh *meshes, uint32_t nmeshes, const yr_kdtree_params *params,
                                     int32_t device, yr_kdtree **out) {
    if (!meshes || !out || nmeshes == 0) return YR_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < nmeshes; i++) out[i] = nullptr;
    yr::KdParams kp;
    if (params) {
        kp.max_depth = params->max_depth;
        kp.max_leaf = params->max_leaf_size;
        kp.cost_ratio = params->cost_ratio;
        kp.empty_bonus = params->empty_bonus;
        kp.large_scene_penalty = params->large_scene_penalty != 0;
    }
    std::vector<yr::KdMesh> ms(nmeshes);
    for (uint32_t i = 0; i < nmeshes; i++) ms[i] = yr::KdMesh{meshes[i].verts, meshes[i].nverts, meshes[i].tris, meshes[i].ntris};
    std::vector<yr::KdTree> unused;
    yr_status st;
    try {
        st = yr::build_kdtrees_gpu(ms, kp, device, unused, out);
    } catch (const std::bad_alloc &) {
        st = YR_ERR_OUT_OF_MEMORY;
    }
    if (st != YR_OK) {
        for (uint32_t j = 0; j < nmeshes; j++) {
            yr_kdtree_free(out[j]);
            out[j] = nullptr;
        }
        return st;
    }
    return YR_OK;
}
