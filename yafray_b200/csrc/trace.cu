// yr_trace_closest / yr_trace_shadow: batched scene ray queries.
#include "dev_trace.cuh"
#include "scene.h"

namespace yr {

constexpr int kTraceBlock = 128;

__global__ void __launch_bounds__(kTraceBlock) k_trace_closest(DevScene S, const yr_ray *__restrict__ rays, uint32_t n,
                                                                yr_hit *__restrict__ hits, int shadow_only) {
    uint2 stk_nt[kKdStackCap];
    float stk_split[kKdStackCap];
    const KdStack stk{stk_nt, stk_split, kKdStackCap};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
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
    }
}

__global__ void __launch_bounds__(kTraceBlock) k_trace_shadow(DevScene S, const yr_shadow_ray *__restrict__ rays,
                                                               uint32_t n, uint8_t *__restrict__ occ, float self_bias) {
    uint2 stk_nt[kKdStackCap];
    float stk_split[kKdStackCap];
    const KdStack stk{stk_nt, stk_split, kKdStackCap};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
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
    }
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
    k_trace_closest<<<grid_for(n, kTraceBlock), kTraceBlock, 0, st>>>(scene->dev, rays, n, hits, shadow_only);
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
    k_trace_shadow<<<grid_for(n, kTraceBlock), kTraceBlock, 0, st>>>(scene->dev, rays, n, occluded,
                                                                     scene->rdr.self_bias);
    yr_status r = cudaGetLastError() == cudaSuccess ? take_status(scene, st) : YR_ERR_CUDA;
    cudaSetDevice(prev);
    return r;
}

}  // extern "C"
