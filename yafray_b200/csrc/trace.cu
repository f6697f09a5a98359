// yr_trace_closest / yr_trace_shadow: batched scene ray queries.
#include <algorithm>

#include "dev_trace.cuh"
#include "scene.h"

namespace yr {

constexpr int kTraceBlock = 128;

// Warps take 32 rays at a time from *fetch (zeroed before the launch) until
// all n are answered, so warps that drew short rays take more of them.
template <class F>
__device__ __forceinline__ void fetch_rays(uint32_t n, uint32_t *fetch, F &&answer) {
    for (;;) {
        uint32_t base = 0;
        if ((threadIdx.x & 31u) == 0) base = atomicAdd(fetch, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const uint32_t i = base + (threadIdx.x & 31u);
        if (i < n) answer(i);
    }
}

__global__ void __launch_bounds__(kTraceBlock, 10) k_trace_closest(DevScene S, const yr_ray *__restrict__ rays, uint32_t n,
                                                                yr_hit *__restrict__ hits, int shadow_only,
                                                                uint32_t *fetch) {
    uint2 stk_nt[kKdStackCap];
    float stk_split[kKdStackCap];
    const KdStack stk{stk_nt, stk_split, kKdStackCap};
    fetch_rays(n, fetch, [&](uint32_t i) {
        const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
        const float4 q0 = __ldg(rp), q1 = __ldg(rp + 1);
        const V3 org = v3(q0.x, q0.y, q0.z), dir = v3(q1.x, q1.y, q1.z);
        // scene_t::firstHit moves the origin by MIN_RAYDIST (scene.cc:693)
        const V3 f = org + dir * kMinRayDist;
        const SceneHit h = scene_closest(S, f, dir, false, shadow_only != 0, stk);
        yr_hit o;
        o.t = h.object >= 0 ? h.t : 0.f;
        o.object = h.object >= 0 ? (uint32_t)h.object : kNone;
        o.triangle = h.object >= 0 ? h.tri - S.objects[h.object].tri_base : kNone;
        o.nodes_visited = h.nodes;
        hits[i] = o;
    });
}

__global__ void __launch_bounds__(kTraceBlock, 10) k_trace_shadow(DevScene S, const yr_shadow_ray *__restrict__ rays,
                                                               uint32_t n, uint8_t *__restrict__ occ, float self_bias,
                                                               uint32_t *fetch) {
    uint2 stk_nt[kKdStackCap];
    float stk_split[kKdStackCap];
    const KdStack stk{stk_nt, stk_split, kKdStackCap};
    fetch_rays(n, fetch, [&](uint32_t i) {
        const float4 *rp = reinterpret_cast<const float4 *>(rays + i);
        const float4 q0 = __ldg(rp), q1 = __ldg(rp + 1);
        const V3 p = v3(q0.x, q0.y, q0.z), l = v3(q1.x, q1.y, q1.z);
        const int own = (int)__float_as_uint(q0.w);
        const uint32_t flags = __float_as_uint(q1.w);
        V3 ray;
        float dist;
        if (flags & 1u) {  // isShadowed(sp, dir) (scene.cc:148-185)
            ray = normalize(l);
            dist = __int_as_float(0x7f800000);
        } else {           // isShadowed(sp, l) (scene.cc:107-146)
            ray = l - p;
            dist = length(ray);
            ray = normalize(ray);
        }
        uint32_t nodes = 0, tests = 0;
        occ[i] = scene_occluded(S, p, own, ray, dist, self_bias, stk, nodes, tests) ? 1 : 0;
    });
}

// one block per resident slot of every SM (queried once per device and kernel)
template <class K>
static int query_grid(K kernel, uint32_t n) {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int sms = 148, per = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kTraceBlock, 0) != cudaSuccess || per < 1)
            per = 1;
        cached[dev] = sms * per;
    }
    const uint64_t need = ((uint64_t)n + kTraceBlock - 1) / kTraceBlock;
    return (int)std::min<uint64_t>(std::max<uint64_t>(need, 1), (uint64_t)cached[dev]);
}

int grid_for(uint32_t n, int block) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t need = ((uint64_t)n + block - 1) / block;
    const uint64_t cap = (uint64_t)sms * 16;
    return (int)(need < cap ? (need ? need : 1) : cap);
}

}  // namespace yr

using namespace yr;

extern "C" {

YR_API yr_status yr_trace_closest(yr_scene *scene, const yr_ray *rays, uint32_t n, yr_hit *hits, int shadow_only,
                                  void *stream) {
    if (!scene || (n && (!rays || !hits))) return YR_ERR_INVALID_ARG;
    if (n == 0) return YR_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(scene->device);
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t *fetch = reinterpret_cast<uint32_t *>(scene->status + 1);
    cudaMemsetAsync(fetch, 0, sizeof(uint32_t), st);
    k_trace_closest<<<query_grid(k_trace_closest, n), kTraceBlock, 0, st>>>(scene->dev, rays, n, hits, shadow_only,
                                                                             fetch);
    yr_status r = cudaGetLastError() == cudaSuccess ? take_status(scene, st) : YR_ERR_CUDA;
    cudaSetDevice(prev);
    return r;
}

YR_API yr_status yr_trace_shadow(yr_scene *scene, const yr_shadow_ray *rays, uint32_t n, uint8_t *occluded,
                                 void *stream) {
    if (!scene || (n && (!rays || !occluded))) return YR_ERR_INVALID_ARG;
    if (n == 0) return YR_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(scene->device);
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t *fetch = reinterpret_cast<uint32_t *>(scene->status + 1);
    cudaMemsetAsync(fetch, 0, sizeof(uint32_t), st);
    k_trace_shadow<<<query_grid(k_trace_shadow, n), kTraceBlock, 0, st>>>(scene->dev, rays, n, occluded,
                                                                           scene->rdr.self_bias, fetch);
    yr_status r = cudaGetLastError() == cudaSuccess ? take_status(scene, st) : YR_ERR_CUDA;
    cudaSetDevice(prev);
    return r;
}

}  // extern "C"
