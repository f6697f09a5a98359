// yr_render_batch: many independent scenes in one persistent launch.
//
// Work items are (scene, tile of whole pixels).  A fixed grid of blocks
// (SMs x resident blocks) pulls items from one atomic counter; each block
// runs the wavefront stages of dev_wave.cuh over its tile with block-local
// ray queues (shadow queue, bounce queues and their counters live in the
// block's scratch and shared memory), so scenes of very different sizes
// share the GPU without one launch per scene and per wave.  The launch is
// captured once in a CUDA graph and replayed.  Block size, tile size and the
// kd stack capacity come from a small autotuner that times the candidates
// on a sample of the items the first time a batch is seen.
//
// Every camera sample, light sample and sum is computed by the same stage
// code as yr_render, so each image is identical to the per-scene render.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#include "dev_wave.cuh"

namespace yr {

struct BatchItem {
    uint32_t scene;
    uint32_t first_px;   // first pixel (region-local, row-major) of the tile
    uint32_t npx;
    uint32_t pad;
};

struct BatchArgs {
    const DevScene *scenes;
    const DevRender *renders;
    const uint32_t *ns;       // shadow slots per vertex, per scene
    const uint32_t *npath;    // path samples per camera sample, per scene
    const BatchItem *items;
    uint32_t nitems;
    uint32_t *next;           // item counter
    char *scratch;
    size_t cta_bytes;
    Plan pmax;                // layout maxima over the scenes
    uint32_t qmax;            // camera samples per tile at most
    float *const *outs;
    unsigned long long *rays; // primary, shadow, bounce
};

template <int STACK, bool INST>
__global__ void __launch_bounds__(256) k_batch(BatchArgs A) {
    __shared__ DevScene S;
    __shared__ DevRender R;
    __shared__ Wave W;
    __shared__ uint32_t cnt[16];
    __shared__ uint32_t item;
    uint2 stk_nt[STACK];
    float stk_split[STACK];
    const KdStack stk{stk_nt, stk_split, STACK};
    const uint32_t tid = threadIdx.x, lane = tid & 31u, nthr = blockDim.x;
    if (tid == 0) {
        W = Wave();
        assign_wave(A.pmax, A.qmax, A.scratch + (size_t)blockIdx.x * A.cta_bytes, W);
        W.counters = cnt;
    }
    uint32_t n_prim = 0, n_sh = 0, n_b = 0, nodes = 0, tests = 0;
    __syncthreads();
    for (;;) {
        if (tid == 0) item = atomicAdd(A.next, 1u);
        __syncthreads();
        const uint32_t it = item;
        if (it >= A.nitems) break;
        if (tid == 0) {
            const BatchItem bi = A.items[it];
            S = A.scenes[bi.scene];
            R = A.renders[bi.scene];
            W.base = bi.first_px * R.spp;
            W.count = bi.npx * R.spp;
            W.ns = A.ns[bi.scene];
            W.npath = A.npath[bi.scene];
            W.out = A.outs[bi.scene];
            for (int k = 0; k < 16; k++) cnt[k] = 0;
        }
        __syncthreads();
        const uint32_t count = W.count;
        for (uint32_t i = tid; i < count; i += nthr) {
            st_primary<INST>(S, R, W, i, stk, nodes, tests);
            n_prim++;
        }
        __syncthreads();
        for (uint32_t b0 = tid - lane; b0 < count; b0 += nthr) st_shade_camera(S, R, W, b0 + lane);
        __syncthreads();
        {
            const uint32_t n = cnt[0];
            for (uint32_t q = tid; q < n; q += nthr)
                if (st_trace_shadow<INST>(S, W, q, R.self_bias, stk, nodes, tests)) n_sh++;
        }
        __syncthreads();
        for (uint32_t i = tid; i < count; i += nthr) st_gather_camera(R, W, i);
        __syncthreads();
        if (W.npath > 0) {
            const uint32_t nc = count * W.npath * (uint32_t)R.path_depth;
            for (uint32_t q = tid; q < nc; q += nthr) W.p_contri[q] = make_float4(0.f, 0.f, 0.f, 0.f);
            __syncthreads();
            for (int j = 0; j < R.path_depth; j++) {
                const uint32_t nb = cnt[1];
                for (uint32_t q = tid; q < nb; q += nthr) {
                    st_trace_bounce<INST>(S, W, q, stk, nodes, tests);
                    n_b++;
                }
                __syncthreads();
                if (tid == 0) cnt[0] = 0;
                __syncthreads();
                for (uint32_t b0 = tid - lane; b0 < nb; b0 += nthr) st_shade_path(S, R, W, j, b0 + lane, nb);
                __syncthreads();
                {
                    const uint32_t n = cnt[0];
                    for (uint32_t q = tid; q < n; q += nthr)
                        if (st_trace_shadow<INST>(S, W, q, R.self_bias, stk, nodes, tests)) n_sh++;
                }
                __syncthreads();
                for (uint32_t b0 = tid - lane; b0 < nb; b0 += nthr)
                    st_gather_path(R, W, j, R.background, b0 + lane, nb);
                __syncthreads();
                if (tid == 0) {
                    uint32_t *t = W.bq;
                    W.bq = W.bq2;
                    W.bq2 = t;
                    cnt[1] = cnt[2];
                    cnt[2] = 0;
                }
                __syncthreads();
            }
        }
        const uint32_t npx = count / R.spp;
        for (uint32_t px = tid; px < npx; px += nthr) st_finish(R, W, px);
        __syncthreads();
    }
    const uint32_t a = __reduce_add_sync(0xffffffffu, n_prim), b = __reduce_add_sync(0xffffffffu, n_sh),
                   c = __reduce_add_sync(0xffffffffu, n_b);
    if (lane == 0) {
        atomicAdd(&A.rays[0], (unsigned long long)a);
        atomicAdd(&A.rays[1], (unsigned long long)b);
        atomicAdd(&A.rays[2], (unsigned long long)c);
    }
}

using BatchKernel = void (*)(BatchArgs);
static const int kStackOptions[3] = {32, 48, kKdStackCap};
// inst: some scene of the batch has references (instanced objects)
static BatchKernel batch_kernel(int stack, bool inst) {
    if (inst) {
        if (stack == 32) return k_batch<32, true>;
        if (stack == 48) return k_batch<48, true>;
        return k_batch<kKdStackCap, true>;
    }
    if (stack == 32) return k_batch<32, false>;
    if (stack == 48) return k_batch<48, false>;
    return k_batch<kKdStackCap, false>;
}

struct BatchConfig {
    int mode = 0;    // YR_BATCH_TILES / YR_BATCH_WAVES
    int block = 0;
    int tile = 0;    // camera samples per tile (cap)
    int stack = 0;
    int streams = 0;
    bool operator==(const BatchConfig &o) const {
        return mode == o.mode && block == o.block && tile == o.tile && stack == o.stack && streams == o.streams;
    }
};

// One stream of the waves schedule: its scenes run one after another
// through one scratch block.
struct WaveLane {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<uint32_t> scenes;
    char *scratch = nullptr;
    size_t bytes = 0;
};

// Device state of one batch (a list of scenes and output images), kept
// between calls so that repeated renders replay the captured graph.
struct BatchCtx {
    int device = -1;
    std::vector<yr_scene *> scenes;
    std::vector<float *> outs;
    std::vector<Plan> plans;
    std::vector<DevScene> h_scenes;     // the records uploaded, to spot changes
    std::vector<DevRender> h_renders;
    Plan pmax{};
    int max_depth = 0;
    uint64_t primary = 0;               // camera samples of all scenes
    DevScene *d_scenes = nullptr;
    DevRender *d_renders = nullptr;
    uint32_t *d_ns = nullptr, *d_npath = nullptr;
    float **d_outs = nullptr;
    BatchItem *d_items = nullptr;
    size_t items_cap = 0;
    uint32_t *d_next = nullptr;
    unsigned long long *d_rays = nullptr;   // tiles: 4; waves: 4 per scene
    unsigned long long *d_kst = nullptr;    // waves: shared kernel-class counters
    char *d_scratch = nullptr;
    size_t scratch_bytes = 0;
    BatchConfig tuned{};
    BatchConfig graph_cfg{};
    uint32_t graph_items = 0;
    char *graph_scratch = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<BatchItem> items;
    std::vector<WaveLane> lanes;
    int lanes_n = 0;
    size_t lane_budget = 1536ull << 20;
    cudaEvent_t fork = nullptr;

    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }
    void drop_lanes() {
        for (WaveLane &l : lanes) {
            if (l.stream) cudaStreamDestroy(l.stream);
            if (l.done) cudaEventDestroy(l.done);
            cudaFree(l.scratch);
        }
        lanes.clear();
        lanes_n = 0;
    }
    ~BatchCtx() {
        drop_graph();
        drop_lanes();
        if (fork) cudaEventDestroy(fork);
        cudaFree(d_scenes);
        cudaFree(d_renders);
        cudaFree(d_ns);
        cudaFree(d_npath);
        cudaFree(d_outs);
        cudaFree(d_items);
        cudaFree(d_next);
        cudaFree(d_rays);
        cudaFree(d_kst);
        cudaFree(d_scratch);
    }
};

static std::mutex g_batch_mu;
static std::map<std::vector<uintptr_t>, std::unique_ptr<BatchCtx>> g_batches;

void batch_forget(const yr_scene *s) {
    std::lock_guard<std::mutex> lock(g_batch_mu);
    for (auto it = g_batches.begin(); it != g_batches.end();) {
        if (std::find(it->second->scenes.begin(), it->second->scenes.end(), s) != it->second->scenes.end()) {
            int prev = 0;
            cudaGetDevice(&prev);
            cudaSetDevice(it->second->device);
            it = g_batches.erase(it);
            cudaSetDevice(prev);
        } else {
            ++it;
        }
    }
}

// relative work of one scene (camera samples x rays per sample)
static double scene_cost(const BatchCtx &C, uint32_t s) {
    const Plan &P = C.plans[s];
    return (double)P.total * (1.0 + P.ns) * (1.0 + P.npath * (double)P.depth * (1.0 + P.ns));
}

// Items for a tile cap: per scene, tiles of max(1, cap/spp) whole pixels;
// scenes with the most work per pixel first, so the long items start early.
static void make_items(const BatchCtx &C, int tile, std::vector<BatchItem> &items) {
    items.clear();
    std::vector<uint32_t> order(C.scenes.size());
    std::iota(order.begin(), order.end(), 0u);
    auto cost = [&](uint32_t s) { return scene_cost(C, s) / std::max<double>(1.0, (double)C.plans[s].rpix); };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost(a) > cost(b); });
    for (uint32_t s : order) {
        const DevRender &R = C.scenes[s]->rdr;
        const uint32_t tpx = std::max<uint32_t>(1u, (uint32_t)tile / R.spp);
        const uint32_t rpix = C.plans[s].rpix;
        for (uint32_t p0 = 0; p0 < rpix; p0 += tpx) items.push_back({s, p0, std::min(tpx, rpix - p0), 0u});
    }
}

static uint32_t tile_cap(const BatchCtx &C, int tile) {
    uint32_t q = 0;
    for (yr_scene *sc : C.scenes) {
        const uint32_t spp = sc->rdr.spp;
        q = std::max(q, std::max<uint32_t>(1u, (uint32_t)tile / spp) * spp);
    }
    return q;
}

static yr_status ensure(void **p, size_t &have, size_t need) {
    if (have >= need && *p) return YR_OK;
    cudaFree(*p);
    *p = nullptr;
    have = 0;
    if (cudaMalloc(p, need) != cudaSuccess) return YR_ERR_OUT_OF_MEMORY;
    have = need;
    return YR_OK;
}

// ------------------------------------------------------------ waves schedule


// Scenes to `n` streams, longest first onto the least loaded stream; one
// scratch block per stream, sized for its largest wave.
static yr_status make_lanes(BatchCtx &C, int n) {
    if (C.lanes_n == n) return YR_OK;
    C.lane_budget = render_budget(n);  // scratch per stream
    C.drop_graph();
    C.drop_lanes();
    C.lanes.resize(n);
    std::vector<uint32_t> order(C.scenes.size());
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return scene_cost(C, a) > scene_cost(C, b); });
    std::vector<double> load(n, 0.0);
    for (uint32_t s : order) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        C.lanes[k].scenes.push_back(s);
        load[k] += scene_cost(C, s);
    }
    for (WaveLane &l : C.lanes) {
        if (cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) != cudaSuccess)
            return YR_ERR_CUDA;
        size_t need = 0;
        for (uint32_t s : l.scenes) {
            const Plan &P = C.plans[s];
            const uint32_t spp = C.scenes[s]->rdr.spp;
            const uint32_t wcap = std::max(spp, wave_for_budget(P, C.scenes[s]->rdr, C.lane_budget));
            need = std::max(need, wave_bytes(P, wcap));
        }
        if (need && cudaMalloc(&l.scratch, need) != cudaSuccess) return YR_ERR_OUT_OF_MEMORY;
        l.bytes = need;
    }
    C.lanes_n = n;
    return YR_OK;
}

// Capture every scene's render on its stream, forked from and joined back
// into one capture stream, as one graph.
static yr_status capture_waves(BatchCtx &C) {
    C.drop_graph();
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return YR_ERR_CUDA;
    if (!C.fork && cudaEventCreateWithFlags(&C.fork, cudaEventDisableTiming) != cudaSuccess) return YR_ERR_CUDA;
    yr_status ret = YR_OK;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaStreamDestroy(cs);
        return YR_ERR_CUDA;
    }
    cudaMemsetAsync(C.d_rays, 0, sizeof(unsigned long long) * 4 * C.scenes.size(), cs);
    cudaEventRecord(C.fork, cs);
    for (WaveLane &l : C.lanes) {
        cudaStreamWaitEvent(l.stream, C.fork, 0);
        for (uint32_t s : l.scenes) {
            yr_scene *sc = C.scenes[s];
            const Plan &P = C.plans[s];
            const uint32_t wcap = std::max(sc->rdr.spp, wave_for_budget(P, sc->rdr, C.lane_budget));
            Wave W;
            std::memset(&W, 0, sizeof(W));
            assign_wave(P, wcap, l.scratch, W);
            W.rays = C.d_rays + 4 * (size_t)s;   // per-scene ray totals, outside the shared scratch
            W.kst = C.d_kst;
            if (ret == YR_OK) ret = enqueue_render(sc, P, wcap, W, C.outs[s], l.stream);
        }
        cudaEventRecord(l.done, l.stream);
        cudaStreamWaitEvent(cs, l.done, 0);
    }
    const cudaError_t ee = cudaStreamEndCapture(cs, &g);
    if (ret == YR_OK && ee != cudaSuccess) ret = YR_ERR_CUDA;
    if (ret == YR_OK && cudaGraphInstantiate(&C.graph, g, 0) != cudaSuccess) ret = YR_ERR_CUDA;
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    return ret;
}

// ------------------------------------------------------------ tiles schedule
// Upload items, size the scratch, launch (or replay the graph) on `st`.
static yr_status launch_tiles(BatchCtx &C, const BatchConfig &cfg, const std::vector<BatchItem> &items,
                              cudaStream_t st, bool use_graph) {
    const uint32_t qmax = tile_cap(C, cfg.tile);
    const size_t cta = (wave_bytes(C.pmax, qmax) + 255) / 256 * 256;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, C.device);
    bool inst = false;
    for (const yr_scene *sc : C.scenes) inst = inst || sc->dev.insts != nullptr;
    BatchKernel kern = batch_kernel(cfg.stack, inst);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, cfg.block, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int grid = std::max(1, std::min<int>(sms * per_sm, (int)items.size()));
    yr_status ret;
    if ((ret = ensure((void **)&C.d_scratch, C.scratch_bytes, cta * (size_t)sms * per_sm)) != YR_OK) return ret;
    if (items.size() > C.items_cap) {
        cudaFree(C.d_items);
        C.d_items = nullptr;
        if (cudaMalloc(&C.d_items, sizeof(BatchItem) * items.size()) != cudaSuccess) return YR_ERR_OUT_OF_MEMORY;
        C.items_cap = items.size();
        C.drop_graph();
    }
    if (cudaMemcpyAsync(C.d_items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
        return YR_ERR_CUDA;
    BatchArgs A;
    A.scenes = C.d_scenes;
    A.renders = C.d_renders;
    A.ns = C.d_ns;
    A.npath = C.d_npath;
    A.items = C.d_items;
    A.nitems = (uint32_t)items.size();
    A.next = C.d_next;
    A.scratch = C.d_scratch;
    A.cta_bytes = cta;
    A.pmax = C.pmax;
    A.qmax = qmax;
    A.outs = C.d_outs;
    A.rays = C.d_rays;
    auto record = [&](cudaStream_t s) {
        cudaMemsetAsync(C.d_next, 0, sizeof(uint32_t), s);
        cudaMemsetAsync(C.d_rays, 0, sizeof(unsigned long long) * 4, s);
        kern<<<grid, cfg.block, 0, s>>>(A);
    };
    if (use_graph) {
        if (!C.graph || !(C.graph_cfg == cfg) || C.graph_items != A.nitems || C.graph_scratch != C.d_scratch) {
            C.drop_graph();
            cudaStream_t cs;
            cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
            cudaGraph_t g;
            if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return YR_ERR_CUDA;
            record(cs);
            if (cudaStreamEndCapture(cs, &g) != cudaSuccess) return YR_ERR_CUDA;
            const cudaError_t ie = cudaGraphInstantiate(&C.graph, g, 0);
            cudaGraphDestroy(g);
            cudaStreamDestroy(cs);
            if (ie != cudaSuccess) return YR_ERR_CUDA;
            C.graph_cfg = cfg;
            C.graph_items = A.nitems;
            C.graph_scratch = C.d_scratch;
        }
        if (cudaGraphLaunch(C.graph, st) != cudaSuccess) return YR_ERR_CUDA;
    } else {
        record(st);
    }
    return cudaGetLastError() == cudaSuccess ? YR_OK : YR_ERR_CUDA;
}

// Run one configuration over all (or the given) items on `st`; device time
// of the launch in *ms_out when not null.
static yr_status run_config(BatchCtx &C, const BatchConfig &cfg, const std::vector<BatchItem> *items, cudaStream_t st,
                            bool use_graph, float *ms_out) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    yr_status ret = YR_OK;
    if (cfg.mode == YR_BATCH_WAVES) {
        if ((ret = make_lanes(C, cfg.streams)) == YR_OK && (!C.graph || !(C.graph_cfg == cfg))) {
            ret = capture_waves(C);
            C.graph_cfg = cfg;
        }
        if (ret == YR_OK && cudaGraphLaunch(C.graph, st) != cudaSuccess) ret = YR_ERR_CUDA;
    } else {
        if (C.lanes_n) {  // the graph of the other schedule is stale
            C.drop_graph();
            C.drop_lanes();
        }
        ret = launch_tiles(C, cfg, items ? *items : C.items, st, use_graph);
    }
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms_out) *ms_out = ms;
    return ret;
}

// Tiles: time every (stack, tile, block) candidate on every 8th item and keep
// the fastest, then time it on all items.  Waves: time 4 and 16 streams on
// the whole batch.  Keep the fastest schedule.
static yr_status autotune(BatchCtx &C, cudaStream_t st, int want_mode, BatchConfig &best) {
    yr_status r;
    float best_ms = 3.4e38f;
    if (want_mode != YR_BATCH_WAVES) {
        BatchConfig bt;
        float bt_ms = 3.4e38f;
        const int blocks[2] = {128, 256}, tiles[3] = {256, 512, 1024};
        for (int stack : kStackOptions) {
            if (C.max_depth + 2 > stack) continue;
            for (int tile : tiles)
                for (int block : blocks) {
                    BatchConfig cfg;
                    cfg.mode = YR_BATCH_TILES;
                    cfg.block = block;
                    cfg.tile = tile;
                    cfg.stack = stack;
                    std::vector<BatchItem> all, sample;
                    make_items(C, tile, all);
                    for (size_t i = 0; i < all.size(); i += 8) sample.push_back(all[i]);
                    float ms = 0.f;
                    if ((r = run_config(C, cfg, &sample, st, false, &ms)) != YR_OK) return r;
                    if (ms < bt_ms) {
                        bt_ms = ms;
                        bt = cfg;
                    }
                }
        }
        if (!bt.block) return YR_ERR_UNSUPPORTED;
        make_items(C, bt.tile, C.items);
        if ((r = run_config(C, bt, nullptr, st, false, &best_ms)) != YR_OK) return r;
        best = bt;
    }
    if (want_mode != YR_BATCH_TILES) {
        const int nmax = (int)std::min<size_t>(C.scenes.size(), 16);
        for (int n : {std::min(4, nmax), nmax}) {
            BatchConfig cfg;
            cfg.mode = YR_BATCH_WAVES;
            cfg.streams = n;
            float ms = 0.f;
            if ((r = run_config(C, cfg, nullptr, st, true, &ms)) != YR_OK) return r;  // capture + first replay
            if ((r = run_config(C, cfg, nullptr, st, true, &ms)) != YR_OK) return r;  // replay alone
            if (ms < best_ms) {
                best_ms = ms;
                best = cfg;
            }
            if (n == nmax) break;
        }
    }
    return best.mode ? YR_OK : YR_ERR_UNSUPPORTED;
}

}  // namespace yr

using namespace yr;

extern "C" YR_API yr_status yr_render_batch(yr_scene *const *scenes, uint32_t count, float *const *outs,
                                            yr_batch_params *params, yr_render_stats *stats, void *stream) {
    if (!scenes || !outs || count == 0) return YR_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < count; i++)
        if (!scenes[i] || !outs[i] || scenes[i]->device != scenes[0]->device) return YR_ERR_INVALID_ARG;
    const int want_mode = params ? params->mode : YR_BATCH_AUTO;
    if (want_mode < YR_BATCH_AUTO || want_mode > YR_BATCH_WAVES) return YR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_batch_mu);
    int prev = 0;
    cudaGetDevice(&prev);
    const int device = scenes[0]->device;
    cudaSetDevice(device);
    auto done = [&](yr_status e) {
        cudaSetDevice(prev);
        return e;
    };
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<uintptr_t> key;
    key.push_back((uintptr_t)device);
    for (uint32_t i = 0; i < count; i++) key.push_back((uintptr_t)scenes[i]);
    std::unique_ptr<BatchCtx> &slot = g_batches[key];
    yr_status ret;
    if (slot) {  // a scene whose parameters changed since the last call: start over
        for (uint32_t i = 0; i < count && slot; i++)
            if (std::memcmp(&slot->h_scenes[i], &scenes[i]->dev, sizeof(DevScene)) ||
                std::memcmp(&slot->h_renders[i], &scenes[i]->rdr, sizeof(DevRender)))
                slot.reset();
    }
    if (!slot) {
        std::unique_ptr<BatchCtx> C(new BatchCtx);
        C->device = device;
        C->scenes.assign(scenes, scenes + count);
        C->plans.resize(count);
        std::vector<DevScene> ds(count);
        std::vector<DevRender> dr(count);
        std::vector<uint32_t> ns(count), np(count);
        C->pmax = Plan{};
        for (uint32_t i = 0; i < count; i++) {
            if ((ret = make_plan(scenes[i], C->plans[i])) != YR_OK) return done(ret);
            if (scenes[i]->rdr.raydepth <= 0) return done(YR_ERR_UNSUPPORTED);
            const Plan &P = C->plans[i];
            C->pmax.ns = std::max(C->pmax.ns, P.ns);
            C->pmax.npath = std::max(C->pmax.npath, P.npath);
            C->pmax.nl = std::max(C->pmax.nl, P.nl);
            C->pmax.depth = std::max(C->pmax.depth, P.depth);
            C->max_depth = std::max(C->max_depth, scenes[i]->max_tree_depth);
            C->primary += P.total;
            std::memcpy(&ds[i], &scenes[i]->dev, sizeof(DevScene));
            std::memcpy(&dr[i], &scenes[i]->rdr, sizeof(DevRender));
            ns[i] = P.ns;
            np[i] = P.npath;
        }
        if (cudaMalloc(&C->d_scenes, sizeof(DevScene) * count) != cudaSuccess ||
            cudaMalloc(&C->d_renders, sizeof(DevRender) * count) != cudaSuccess ||
            cudaMalloc(&C->d_ns, 4 * count) != cudaSuccess || cudaMalloc(&C->d_npath, 4 * count) != cudaSuccess ||
            cudaMalloc(&C->d_outs, sizeof(float *) * count) != cudaSuccess ||
            cudaMalloc(&C->d_next, sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc(&C->d_rays, sizeof(unsigned long long) * 4 * count) != cudaSuccess ||
            cudaMalloc(&C->d_kst, sizeof(unsigned long long) * 3 * YR_K_COUNT) != cudaSuccess)
            return done(YR_ERR_OUT_OF_MEMORY);
        cudaMemcpy(C->d_scenes, ds.data(), sizeof(DevScene) * count, cudaMemcpyHostToDevice);
        cudaMemcpy(C->d_renders, dr.data(), sizeof(DevRender) * count, cudaMemcpyHostToDevice);
        cudaMemcpy(C->d_ns, ns.data(), 4 * count, cudaMemcpyHostToDevice);
        cudaMemcpy(C->d_npath, np.data(), 4 * count, cudaMemcpyHostToDevice);
        C->h_scenes = std::move(ds);
        C->h_renders = std::move(dr);
        slot = std::move(C);
    }
    BatchCtx &C = *slot;
    // output images may move between calls
    if (C.outs.size() != count || !std::equal(C.outs.begin(), C.outs.end(), outs)) {
        C.outs.assign(outs, outs + count);
        cudaMemcpy(C.d_outs, C.outs.data(), sizeof(float *) * count, cudaMemcpyHostToDevice);
        if (C.lanes_n) C.drop_graph();  // the waves graph holds the image pointers
    }
    // the tiles kernel runs each vertex's light sampling in one stage and
    // one round of paths: a scene whose area lights guess the penumbra
    // first, or whose path light takes adaptive rounds, takes the waves
    bool guess = false;
    for (uint32_t i = 0; i < count; i++)
        guess = guess || scenes[i]->rdr.has_guess || scenes[i]->rdr.path_threshold > 0.f;
    if (guess && want_mode == YR_BATCH_TILES) return done(YR_ERR_UNSUPPORTED);
    const int mode_wanted = guess ? YR_BATCH_WAVES : want_mode;
    BatchConfig cfg;
    const bool explicit_tiles = !guess && params && params->block_size > 0 && params->queue_tile > 0 &&
                                want_mode != YR_BATCH_WAVES;
    const bool explicit_waves = params && want_mode == YR_BATCH_WAVES && params->streams > 0;
    if (explicit_tiles) {
        cfg.mode = YR_BATCH_TILES;
        cfg.block = params->block_size;
        cfg.tile = params->queue_tile;
        if (cfg.block % 32 || cfg.block < 32 || cfg.block > 1024 || cfg.tile < 1) return done(YR_ERR_INVALID_ARG);
        cfg.stack = kKdStackCap;
        for (int s : kStackOptions)
            if (C.max_depth + 2 <= s) {
                cfg.stack = s;
                break;
            }
    } else if (explicit_waves) {
        cfg.mode = YR_BATCH_WAVES;
        cfg.streams = std::min<int>(params->streams, (int)count);
    } else {
        if (!C.tuned.mode || (mode_wanted && C.tuned.mode != mode_wanted)) {
            BatchConfig t;
            if ((ret = autotune(C, st, mode_wanted, t)) != YR_OK) return done(ret);
            C.tuned = t;
        }
        cfg = C.tuned;
    }
    if (cfg.mode == YR_BATCH_TILES) make_items(C, cfg.tile, C.items);
    float ms = 0.f;
    const bool use_graph = !params || params->use_graph || cfg.mode == YR_BATCH_WAVES;
    if ((ret = run_config(C, cfg, nullptr, st, use_graph, &ms)) != YR_OK) return done(ret);
    // device status words of every scene
    for (yr_scene *sc : C.scenes)
        if ((ret = take_status(sc, st)) != YR_OK) return done(ret);
    if (stats) {
        const size_t nr = cfg.mode == YR_BATCH_WAVES ? 4 * (size_t)count : 4;
        std::vector<unsigned long long> r(nr, 0ull);
        cudaMemcpy(r.data(), C.d_rays, sizeof(unsigned long long) * nr, cudaMemcpyDeviceToHost);
        std::memset(stats, 0, sizeof(*stats));
        for (size_t i = 0; i < nr; i += 4) {
            stats->rays_primary += r[i];
            stats->rays_shadow += r[i + 1];
            stats->rays_bounce += r[i + 2];
        }
        if (cfg.mode == YR_BATCH_WAVES) stats->rays_primary = C.primary;
        stats->ms = ms;
        stats->kernel_ms[YR_K_OTHER] = ms;
        stats->kernel_launches[YR_K_OTHER] = 1;
    }
    if (params) {  // report the configuration used
        params->mode = cfg.mode;
        params->block_size = cfg.block;
        params->queue_tile = cfg.tile;
        params->stack_entries = cfg.mode == YR_BATCH_WAVES ? kKdStackCap : cfg.stack;
        params->streams = cfg.streams;
    }
    return done(YR_OK);
}
