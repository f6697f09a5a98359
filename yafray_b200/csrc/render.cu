// yr_render: the wavefront renderer.
//
// One wave = a block of whole pixels x spp camera samples.  Per wave:
//   k_primary        camera rays -> closest hit        (scene_t::raytrace)
//   k_shade<camera>  light samples -> shadow-ray queue (illuminate, per light)
//                    + the path light's first directions
//   k_trace_shadow_q dense shadow queue -> occlusion per slot (isShadowed)
//   k_gather<camera> per-light terms in the reference's summation order
//   per bounce j:
//     k_trace_bounce   bounce queue -> closest hit     (scene_t::firstHit)
//     k_shade<path>    light samples at the bounce vertex, next direction
//     k_trace_shadow_q
//     k_gather<path>   contribution of vertex j, re-queue live paths
//   k_finish         light sum, path term, AA average per pixel
// Shadow rays and bounce rays are appended to dense queues with one
// atomicAdd per warp (ballot + popc prefix); their results land in fixed
// per-vertex slots, so every sum is formed in the reference's order.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#define YR_WAVE_KERNELS 1
#include "dev_wave.cuh"

namespace yr {

int grid_for(uint32_t n, int block);

static yr_status scratch(yr_scene *s, int i, size_t bytes, void **p) {
    if ((int)s->scratch.size() <= i) s->scratch.resize(i + 1);
    DevBuf &b = s->scratch[i];
    if (b.bytes < bytes) {
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
        if (cudaMalloc(&b.p, bytes ? bytes : 16) != cudaSuccess) return YR_ERR_OUT_OF_MEMORY;
        b.bytes = bytes;
    }
    *p = b.p;
    return YR_OK;
}

// The launches of one render on `st`, without any synchronization;
// `timed(cls, launch)` wraps each kernel launch.  waves_begin() clears the
// render's counters and the image outside the region; wave_launch() runs
// the wave of camera samples [b, b + wcap); launch_waves() is all of it.
struct WaveGrids {
    int gq, gb;  // shadow queue, bounce queue
};

static WaveGrids waves_begin(yr_scene *scene, const Plan &P, uint32_t wcap, Wave &W, float *out, cudaStream_t st) {
    DevRender &R = scene->rdr;
    W.out = out;
    W.part = 1;  // the path shading takes the bounce walk's hits-first order
    cudaMemsetAsync(W.rays, 0, sizeof(unsigned long long) * 4, st);
    cudaMemsetAsync(W.kst, 0, sizeof(unsigned long long) * 3 * YR_K_COUNT, st);
    // pixels outside the region are written as 0 (scene.cc:773)
    if (P.rpix != P.npix) cudaMemsetAsync(out, 0, sizeof(float) * 4 * (size_t)P.npix, st);
    WaveGrids G{0, 0};
    if (R.raydepth <= 0) {
        // raytrace() returns black at the ray-level cap (scene.cc:204-209);
        // a tone map keeps black black except pow(0, 0) = 1 for gamma 0,
        // which is refused when the scene is created
        cudaMemsetAsync(out, 0, sizeof(float) * 4 * (size_t)P.npix, st);
        return G;
    }
    const uint32_t vcap = std::max(wcap, wcap * std::max(1u, P.npath));
#if YR_TRACE_GRID_PERSIST
    G.gq = std::min(grid_for(vcap * std::max(P.ns, 1u), kBlock), resident_grid(k_trace_shadow_q<false, true>));
    G.gb = std::min(grid_for(vcap, kBlock), resident_grid(k_trace_bounce<false>));
#else
    G.gq = grid_for(vcap * std::max(P.ns, 1u), kBlock);
    G.gb = G.gq;
#endif
    return G;
}

template <class Timed>
static void wave_launch(yr_scene *scene, const Plan &P, uint32_t wcap, Wave &W, const WaveGrids &G, uint64_t b,
                        cudaStream_t st, Timed &&timed) {
    DevRender &R = scene->rdr;
    const DevScene &D = scene->dev;
    const uint32_t npath = P.npath;
    const int gq = G.gq, gb = G.gb;
    // the traversal kernels with the reference-transforming loops only
    // for scenes that have references
    const bool inst = D.insts != nullptr;
    auto k_prim = inst ? k_primary<true> : k_primary<false>;
    // the shadow queue kernel with the casters' BVH walk alone when the
    // scene uses it (no shadow-ray tree, no exact order)
    const bool bvh = !D.use_sh_tree && !D.exact_order;
    auto k_shadow = inst ? (bvh ? k_trace_shadow_q<true, true> : k_trace_shadow_q<true, false>)
                         : (bvh ? k_trace_shadow_q<false, true> : k_trace_shadow_q<false, false>);
    auto k_bounce = inst ? k_trace_bounce<true> : k_trace_bounce<false>;
    W.base = (uint32_t)b;
    W.count = (uint32_t)std::min<uint64_t>(wcap, P.total - b);
    const int g = (int)((W.count + kBlock - 1) / kBlock);
    cudaMemsetAsync(W.counters, 0, sizeof(uint32_t) * 16, st);
    timed(YR_K_PRIMARY, [&] { k_prim<<<g, kBlock, 0, st>>>(D, R, W); });
    timed(YR_K_SHADE_CAMERA, [&] { k_shade_camera<<<g, kBlock, 0, st>>>(D, R, W); });
    timed(YR_K_OTHER, [&] { k_count<<<1, 1, 0, st>>>(W, 0); });
    cudaMemsetAsync(W.counters + 6, 0, sizeof(uint32_t), st);
    timed(YR_K_SHADOW, [&] { k_shadow<<<gq, kBlock, 0, st>>>(D, W, R.self_bias); });
    if (R.has_guess) {
        // the penumbra guess decided from its probes, then the sample rays
        // of the points in penumbra
        cudaMemsetAsync(W.counters, 0, sizeof(uint32_t), st);
        timed(YR_K_SHADE_CAMERA, [&] { k_guess_camera<<<g, kBlock, 0, st>>>(D, R, W); });
        timed(YR_K_OTHER, [&] { k_count<<<1, 1, 0, st>>>(W, 0); });
        cudaMemsetAsync(W.counters + 6, 0, sizeof(uint32_t), st);
        timed(YR_K_SHADOW, [&] { k_shadow<<<gq, kBlock, 0, st>>>(D, W, R.self_bias); });
    }
    timed(YR_K_GATHER, [&] { k_gather_camera<<<g, kBlock, 0, st>>>(R, W); });
    if (npath > 0) {
        const size_t nc = (size_t)W.count * npath * P.depth;
        timed(YR_K_OTHER, [&] {
            k_clear_contri<<<grid_for((uint32_t)std::min<size_t>(nc, 1u << 30), kBlock), kBlock, 0, st>>>(W, nc);
        });
        const int gp = (int)(((size_t)W.count * npath + kBlock - 1) / kBlock);
        auto bounces = [&] {
        for (int j = 0; j < R.path_depth; j++) {
            timed(YR_K_OTHER, [&] { k_count<<<1, 1, 0, st>>>(W, 1); });
            cudaMemsetAsync(W.counters + 7, 0, sizeof(uint32_t), st);
            cudaMemsetAsync(W.counters + 9, 0, 2 * sizeof(uint32_t), st);
            timed(YR_K_BOUNCE, [&] { k_bounce<<<gb, kBlock, 0, st>>>(D, W); });
            cudaMemsetAsync(W.counters, 0, sizeof(uint32_t), st);
            timed(YR_K_SHADE_PATH, [&] { k_shade_path<<<gp, kBlock, 0, st>>>(D, R, W, j); });
            timed(YR_K_OTHER, [&] { k_count<<<1, 1, 0, st>>>(W, 0); });
            cudaMemsetAsync(W.counters + 6, 0, sizeof(uint32_t), st);
            timed(YR_K_SHADOW, [&] { k_shadow<<<gq, kBlock, 0, st>>>(D, W, R.self_bias); });
            if (R.has_guess) {
                cudaMemsetAsync(W.counters, 0, sizeof(uint32_t), st);
                timed(YR_K_SHADE_PATH, [&] { k_guess_path<<<gp, kBlock, 0, st>>>(D, R, W, j); });
                timed(YR_K_OTHER, [&] { k_count<<<1, 1, 0, st>>>(W, 0); });
                cudaMemsetAsync(W.counters + 6, 0, sizeof(uint32_t), st);
                timed(YR_K_SHADOW, [&] { k_shadow<<<gq, kBlock, 0, st>>>(D, W, R.self_bias); });
            }
            timed(YR_K_GATHER, [&] { k_gather_path<<<gp, kBlock, 0, st>>>(R, W, j, R.background); });
            std::swap(W.bq, W.bq2);
            timed(YR_K_OTHER, [&] { k_swap_queues<<<1, 1, 0, st>>>(W); });
        }
        };
        bounces();
        if (R.path_threshold > 0.f) {
            // the adaptive rounds: round 0's sums and extra rounds, then up
            // to three more rounds of paths for the samples that take them
            W.rep = 0;
            timed(YR_K_OTHER, [&] { k_path_round<<<g, kBlock, 0, st>>>(R, W); });
            for (uint32_t r = 1; r <= 3; r++) {
                W.rep = r;
                timed(YR_K_OTHER, [&] {
                    k_clear_contri<<<grid_for((uint32_t)std::min<size_t>(nc, 1u << 30), kBlock), kBlock, 0, st>>>(W, nc);
                });
                cudaMemsetAsync(W.counters + 1, 0, sizeof(uint32_t), st);
                timed(YR_K_SHADE_CAMERA, [&] { k_path_restart<<<g, kBlock, 0, st>>>(D, R, W); });
                bounces();
                timed(YR_K_OTHER, [&] { k_path_round<<<g, kBlock, 0, st>>>(R, W); });
            }
            W.rep = 0;
        }
    }
    const int gf = (int)((W.count / R.spp + kBlock - 1) / kBlock);
    timed(YR_K_OTHER, [&] { k_finish<<<gf, kBlock, 0, st>>>(R, W); });
}

template <class Timed>
static void launch_waves(yr_scene *scene, const Plan &P, uint32_t wcap, Wave &W, float *out, cudaStream_t st,
                         Timed &&timed) {
    const WaveGrids G = waves_begin(scene, P, wcap, W, out, st);
    if (scene->rdr.raydepth <= 0) return;
    for (uint64_t b = 0; b < P.total; b += wcap) wave_launch(scene, P, wcap, W, G, b, st, timed);
}

yr_status enqueue_render(yr_scene *scene, const Plan &P, uint32_t wcap, Wave &W, float *out, cudaStream_t st) {
    launch_waves(scene, P, wcap, W, out, st, [](int, auto &&launch) { launch(); });
    return cudaGetLastError() == cudaSuccess ? YR_OK : YR_ERR_CUDA;
}

// All waves of one render on `st`.  `out` is the device RGBA image.
// With `events` false no CUDA event is created (stats->ms and the kernel
// times stay 0).
static yr_status run_waves(yr_scene *scene, const Plan &P, uint32_t wcap, Wave &W, float *out,
                           yr_render_stats *stats, cudaStream_t st, bool events) {
    DevRender &R = scene->rdr;
    W.out = out;
    const bool kstats = events && stats && stats->want_kernel_stats;
    double kms[YR_K_COUNT] = {0};
    uint32_t klaunch[YR_K_COUNT] = {0};
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> kev;
    auto timed = [&](int cls, auto &&launch) {
        klaunch[cls]++;
        if (!kstats) {
            launch();
            return;
        }
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, st);
        launch();
        cudaEventRecord(b, st);
        kev.push_back({cls, {a, b}});
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (events) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, st);
    }
    launch_waves(scene, P, wcap, W, out, st, timed);
    if (events) cudaEventRecord(e1, st);
    if (cudaGetLastError() != cudaSuccess) return YR_ERR_CUDA;
    yr_status ret = take_status(scene, st);
    if (stats) {
        unsigned long long r[4] = {0, 0, 0, 0}, k[3 * YR_K_COUNT];
        cudaMemcpyAsync(r, W.rays, sizeof(r), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(k, W.kst, sizeof(k), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        stats->rays_primary = (R.raydepth > 0) ? P.total : 0;
        stats->rays_shadow = r[1];
        stats->rays_bounce = r[2];
        float ms = 0.f;
        if (events) cudaEventElapsedTime(&ms, e0, e1);
        stats->ms = ms;
        for (auto &e : kev) {
            float m = 0.f;
            cudaEventElapsedTime(&m, e.second.first, e.second.second);
            kms[e.first] += m;
        }
        for (int c = 0; c < YR_K_COUNT; c++) {
            stats->kernel_ms[c] = kms[c];
            stats->kernel_launches[c] = klaunch[c];
            stats->kernel_rays[c] = k[3 * c];
            stats->kernel_nodes[c] = k[3 * c + 1];
            stats->kernel_tests[c] = k[3 * c + 2];
        }
    }
    for (auto &e : kev) {
        cudaEventDestroy(e.second.first);
        cudaEventDestroy(e.second.second);
    }
    if (events) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return ret;
}

// ------------------------------------------------- allocation-free render
// Scratch of yr_render_noalloc: one fixed block in the global memory of
// every GPU that loads this library, held until the process exits.  In host
// code the symbol only stands for the block; its device address comes from
// cudaGetSymbolAddress, taken once per device with that device current.
constexpr size_t kNoAllocScratchBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[kMaxDevices];

static yr_status noalloc_scratch(int device, void **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (device < 0 || device >= kMaxDevices) return YR_ERR_INVALID_ARG;
    if (!g_noalloc_addr[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return YR_ERR_CUDA;
        g_noalloc_addr[device] = p;
    }
    *out = g_noalloc_addr[device];
    return YR_OK;
}

}  // namespace yr

using namespace yr;

extern "C" YR_API yr_status yr_render_noalloc(yr_scene *scene, float *rgba, yr_render_stats *stats, void *stream) {
    if (!scene || !rgba) return YR_ERR_INVALID_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(scene->device) != cudaSuccess) return YR_ERR_CUDA;
    auto done = [&](yr_status e) {
        cudaSetDevice(prev);
        return e;
    };
    Plan P;
    yr_status ret = make_plan(scene, P);
    if (ret != YR_OK) return done(ret);
    // waves as large as the block allows; one pixel's samples must fit
    const uint32_t wcap = wave_for_budget(P, scene->rdr, kNoAllocScratchBytes);
    if (wcap < scene->rdr.spp) return done(YR_ERR_TOO_LARGE);
    void *block = nullptr;
    if ((ret = noalloc_scratch(scene->device, &block)) != YR_OK) return done(ret);
    Wave W;
    std::memset(&W, 0, sizeof(W));
    assign_wave(P, wcap, (char *)block, W);
    return done(run_waves(scene, P, wcap, W, rgba, stats, (cudaStream_t)stream, false));
}

extern "C" YR_API yr_status yr_render(yr_scene *scene, float *rgba, int rgba_on_host, yr_render_stats *stats,
                                      void *stream) {
    if (!scene || !rgba) return YR_ERR_INVALID_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(scene->device) != cudaSuccess) return YR_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    auto done = [&](yr_status e) {
        cudaSetDevice(prev);
        return e;
    };
    Plan P;
    yr_status ret = make_plan(scene, P);
    if (ret != YR_OK) return done(ret);
    // wave: whole pixels, scratch near 1.5 GB at most
    const uint32_t wcap = std::max(scene->rdr.spp, wave_for_budget(P, scene->rdr, render_budget(1)));
    PoolBlock blk(scene->device, st);  // given back (after a stream sync) when this call returns
    if ((ret = pool_acquire(scene->device, wave_bytes(P, wcap), blk.buf)) != YR_OK) return done(ret);
    Wave W;
    std::memset(&W, 0, sizeof(W));
    assign_wave(P, wcap, (char *)blk.buf.p, W);
    float *out = rgba;
    if (rgba_on_host) {
        void *ptr = nullptr;
        if ((ret = scratch(scene, 1, sizeof(float) * 4 * (size_t)P.npix, &ptr)) != YR_OK) return done(ret);
        out = (float *)ptr;
    }
    ret = run_waves(scene, P, wcap, W, out, stats, st, true);
    if (ret != YR_OK) return done(ret);
    if (rgba_on_host) {
        if (cudaMemcpyAsync(rgba, out, sizeof(float) * 4 * (size_t)P.npix, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return done(YR_ERR_CUDA);
        if (cudaStreamSynchronize(st) != cudaSuccess) return done(YR_ERR_CUDA);
    }
    return done(YR_OK);
}

extern "C" YR_API yr_status yr_render_progressive(yr_scene *scene, float *rgba, uint32_t wave_pixels,
                                                  yr_pixels_fn on_pixels, void *user, yr_render_stats *stats,
                                                  void *stream) {
    if (!scene || !rgba || !on_pixels) return YR_ERR_INVALID_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(scene->device) != cudaSuccess) return YR_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    auto done = [&](yr_status e) {
        cudaSetDevice(prev);
        return e;
    };
    Plan P;
    yr_status ret = make_plan(scene, P);
    if (ret != YR_OK) return done(ret);
    const DevRender &R = scene->rdr;
    uint32_t wcap = std::max(R.spp, wave_for_budget(P, R, render_budget(1)));
    if (wave_pixels) wcap = std::min(wcap, std::max(1u, wave_pixels) * R.spp);
    PoolBlock blk(scene->device, st);
    if ((ret = pool_acquire(scene->device, wave_bytes(P, wcap), blk.buf)) != YR_OK) return done(ret);
    Wave W;
    std::memset(&W, 0, sizeof(W));
    assign_wave(P, wcap, (char *)blk.buf.p, W);
    void *img = nullptr;
    if ((ret = scratch(scene, 1, sizeof(float) * 4 * (size_t)P.npix, &img)) != YR_OK) return done(ret);
    float *out = (float *)img;
    const WaveGrids G = waves_begin(scene, P, wcap, W, out, st);
    const size_t row = sizeof(float) * 4 * (size_t)R.cam.resx;
    auto no_timing = [](int, auto &&launch) { launch(); };
    uint64_t next = 0;  // first camera sample not yet delivered
    bool stop = false;
    if (R.raydepth <= 0 || P.rpix != P.npix) {
        // every pixel outside the region (or all, at ray depth 0) is 0 now
        if (cudaMemcpyAsync(rgba, out, row * R.cam.resy, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return done(YR_ERR_CUDA);
    }
    for (uint64_t b = 0; b < P.total && R.raydepth > 0 && !stop; b += wcap) {
        wave_launch(scene, P, wcap, W, G, b, st, no_timing);
        if (cudaGetLastError() != cudaSuccess) return done(YR_ERR_CUDA);
        // the wave's pixels, region pixels [b/spp, (b+count)/spp): copy
        // exactly those (row segments of the region), then hand them over
        const uint32_t p0 = (uint32_t)(b / R.spp);
        const uint32_t p1 = (uint32_t)(std::min<uint64_t>(P.total, b + wcap) / R.spp);
        for (uint32_t p = p0; p < p1;) {
            const uint32_t ry = p / (uint32_t)R.rw, rx = p % (uint32_t)R.rw;
            const uint32_t n = std::min<uint32_t>(p1 - p, (uint32_t)R.rw - rx);
            const size_t at = sizeof(float) * 4 * ((size_t)(R.ry0 + ry) * R.cam.resx + R.rx0 + rx);
            if (rx == 0 && n == (uint32_t)R.rw && p1 - p >= 2 * (uint32_t)R.rw) {
                // whole region rows: one strided copy
                const uint32_t rows = (p1 - p) / (uint32_t)R.rw;
                if (cudaMemcpy2DAsync((char *)rgba + at, row, (char *)out + at, row, sizeof(float) * 4 * R.rw, rows,
                                      cudaMemcpyDeviceToHost, st) != cudaSuccess)
                    return done(YR_ERR_CUDA);
                p += rows * (uint32_t)R.rw;
                continue;
            }
            if (cudaMemcpyAsync((char *)rgba + at, (char *)out + at, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost,
                                st) != cudaSuccess)
                return done(YR_ERR_CUDA);
            p += n;
        }
        if ((ret = take_status(scene, st)) != YR_OK) return done(ret);  // waits for the copy too
        next = (uint64_t)p1 * R.spp;
        stop = on_pixels(user, p0, p1 - p0) == 0;
    }
    if (R.raydepth <= 0 || P.rpix != P.npix) {
        if (cudaStreamSynchronize(st) != cudaSuccess) return done(YR_ERR_CUDA);
        if (R.raydepth <= 0) stop = on_pixels(user, 0, P.rpix) == 0;
    }
    if (stats) {
        unsigned long long r[4] = {0, 0, 0, 0};
        cudaMemcpyAsync(r, W.rays, sizeof(r), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return done(YR_ERR_CUDA);
        stats->ms = 0.f;
        stats->rays_primary = (R.raydepth > 0) ? next : 0;
        stats->rays_shadow = r[1];
        stats->rays_bounce = r[2];
    }
    return done(stop && next < P.total ? YR_ERR_CANCELLED : YR_OK);
}
