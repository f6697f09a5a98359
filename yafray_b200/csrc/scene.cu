// yr_scene_create / yr_scene_destroy: host flattening and device upload.
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstring>
#include <new>

#include "dev_trace.cuh"
#include "scene.h"

namespace yr {
namespace {

V3 hv(const float *p) { return V3{p[0], p[1], p[2]}; }

// vector3d_t::normalize on the host (1/sqrt in double, vector3d.h:207-217)
V3 h_normalize(V3 a) {
    float l = a.x * a.x + a.y * a.y + a.z * a.z;
    if (l != 0.f) {
        float k = (float)(1.0 / std::sqrt((double)l));
        a.x *= k;
        a.y *= k;
        a.z *= k;
    }
    return a;
}
float h_length(const V3 &a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
V3 h_div(const V3 &a, float f) { return V3{a.x / f, a.y / f, a.z / f}; }

template <class T>
yr_status dev_upload(yr_scene *s, const T *host, size_t count, T **out) {
    *out = nullptr;
    if (count == 0) return YR_OK;
    DevBuf b;
    b.bytes = sizeof(T) * count;
    if (cudaMalloc(&b.p, b.bytes) != cudaSuccess) return YR_ERR_OUT_OF_MEMORY;
    s->bufs.push_back(b);
    if (cudaMemcpy(b.p, host, b.bytes, cudaMemcpyHostToDevice) != cudaSuccess) return YR_ERR_CUDA;
    *out = (T *)b.p;
    return YR_OK;
}

// Child links, leaf triangles and prim-list ranges of a flattened tree.
bool valid_tree(const std::vector<uint2> &nodes, const std::vector<uint32_t> &prims, size_t ntris) {
    const size_t n = nodes.size();
    for (size_t i = 0; i < n; i++) {
        const uint32_t f = nodes[i].y, w = nodes[i].x;
        if ((f & 3u) != 3u) {
            // the right child follows the left subtree, so every descent
            // moves to a higher index and ends
            if (i + 1 >= n || (f >> 2) >= n || (f >> 2) < i + 2) return false;
        } else {
            const uint32_t np = f >> 2;
            if (np == 1 && w >= ntris) return false;
            if (np > 1 && ((size_t)w + np > prims.size())) return false;
        }
    }
    for (uint32_t p : prims)
        if (p >= ntris) return false;
    return true;
}

}  // namespace

// ------------------------------------------------------------ scratch pool
static std::mutex g_pool_mu;
static std::map<int, std::vector<DevBuf>> g_pool_free;
static std::map<int, int> g_live_scenes;

yr_status pool_acquire(int device, size_t bytes, DevBuf &out) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    std::vector<DevBuf> &fl = g_pool_free[device];
    int best = -1;
    for (int i = 0; i < (int)fl.size(); i++)
        if (fl[i].bytes >= bytes && (best < 0 || fl[i].bytes < fl[best].bytes)) best = i;
    if (best >= 0) {
        out = fl[best];
        fl.erase(fl.begin() + best);
        return YR_OK;
    }
    if (!fl.empty()) {  // replace the largest free block by a larger one
        auto it = std::max_element(fl.begin(), fl.end(),
                                   [](const DevBuf &a, const DevBuf &b) { return a.bytes < b.bytes; });
        cudaFree(it->p);
        fl.erase(it);
    }
    out.bytes = bytes ? bytes : 16;
    if (cudaMalloc(&out.p, out.bytes) != cudaSuccess) {
        out = DevBuf{};
        return YR_ERR_OUT_OF_MEMORY;
    }
    return YR_OK;
}

void pool_release(int device, const DevBuf &b) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (g_live_scenes[device] > 0) {
        g_pool_free[device].push_back(b);
    } else {
        cudaFree(b.p);
    }
}

static void pool_scene_count(int device, int delta) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    int &n = g_live_scenes[device];
    n += delta;
    if (n <= 0) {
        n = 0;
        for (DevBuf &b : g_pool_free[device]) cudaFree(b.p);
        g_pool_free[device].clear();
    }
}

void make_shader(const yr_shader_desc &d, DevShader &o) {
    o.color = c3(d.color[0], d.color[1], d.color[2]);
    o.specular = c3(d.specular[0], d.specular[1], d.specular[2]);
    o.hard = d.hard;
    o.tex_type = (int)d.tex_type;
    o.tc1 = c3(d.tex_color1[0], d.tex_color1[1], d.tex_color1[2]);
    o.tc2 = c3(d.tex_color2[0], d.tex_color2[1], d.tex_color2[2]);
    o.H = d.tex_H;
    o.lacunarity = d.tex_lacunarity;
    o.octaves = d.tex_octaves;
    o.tsize = d.tex_size;
    o.intensity = d.tex_intensity;
    o.mod_color = d.mod_color;
    o.mod_spec = d.mod_specular;
    o.mod_hard = d.mod_hard;
    for (int k = 0; k < 3; k++) {
        o.msize[k] = d.mod_size[k];
        o.mofs[k] = d.mod_ofs[k];
    }
    o.tdepth = d.tex_depth;
    o.thard = (int)d.tex_hard;
    o.texco = (int)(d.tex_map & 0xffu);
    for (int k = 0; k < 3; k++) {
        const uint32_t p = (d.tex_map >> (8 * (k + 1))) & 0xffu;
        o.proj[k] = p == YR_PROJ_DEFAULT ? k : (p >= YR_PROJ_X && p <= YR_PROJ_Z ? (int)p - 1 : -1);
    }
    o.mod_mode = (int)d.mod_mode;
    o.noise = (int)d.tex_noise;
    o.noise2 = (int)d.tex_noise2;
    o.tshape = (int)d.tex_shape;
    o.tvariant = (int)d.tex_variant;
    o.turb = d.tex_turbulence;
    // textureMarble_t ctor (basictex.cc:113-115)
    o.sharp = d.tex_sharpness > 1 ? (float)(1.0 / (double)d.tex_sharpness) : 1.0f;
    o.offset = d.tex_offset;
    o.gain = d.tex_gain;
    o.distort = d.tex_distort;
    for (int k = 0; k < 4; k++) o.weights[k] = d.tex_weights[k];
    o.mk_exp = d.tex_mk_exponent;
    o.metric = (int)d.tex_metric;
    // textureVoronoi_t ctor (basictex.cc:585-589): iscale = intensity / sum |w|
    const float sw = ((std::fabs(d.tex_weights[0]) + std::fabs(d.tex_weights[1])) + std::fabs(d.tex_weights[2])) +
                     std::fabs(d.tex_weights[3]);
    o.viscale = sw != 0.f ? d.tex_intensity / sw : 0.f;
    o.vinvw = sw != 0.f ? 1.0f / sw : 0.f;
}

// Enumerations of a shader record in range (texture type, noise bases,
// modulator mode, shape / type / metric fields of the texture used).
bool valid_shader(const yr_shader_desc &d) {
    if (d.tex_type > YR_TEX_GRADIENT || d.mod_mode > YR_MOD_SUB) return false;
    if ((d.tex_map & 0xffu) > YR_TEXCO_UV) return false;
    for (int k = 1; k < 4; k++)
        if (((d.tex_map >> (8 * k)) & 0xffu) > YR_PROJ_NONE) return false;
    if (d.tex_type == YR_TEX_NONE) return true;
    if (d.tex_noise > YR_NOISE_CELLNOISE || d.tex_noise2 > YR_NOISE_CELLNOISE) return false;
    switch (d.tex_type) {
    case YR_TEX_MARBLE:
    case YR_TEX_WOOD: return d.tex_shape <= YR_WAVE_TRI && d.tex_depth >= 0 && d.tex_depth < 30;
    case YR_TEX_CLOUDS: return d.tex_variant <= 2 && d.tex_depth >= 0 && d.tex_depth < 30;
    case YR_TEX_VORONOI: return d.tex_shape <= 3 && d.tex_metric <= YR_DIST_MINKOVSKY;
    case YR_TEX_GRADIENT: return d.tex_shape <= YR_GRAD_HALO;
    default: return true;
    }
}

// areaLight_t::fillQuad (arealight.cc:31-73): sample grid and jitter axes.
static yr_status fill_quad(const yr_light_desc &d, DevLight &L, std::vector<float> &pts) {
    const V3 a = hv(d.p[0]), b = hv(d.p[1]), c = hv(d.p[2]), dd = hv(d.p[3]);
    const int nsam = d.samples;
    if (nsam < 1) return YR_ERR_INVALID_ARG;
    const float ab = h_length(b - a), bc = h_length(c - b), cd = h_length(dd - c), da = h_length(a - dd);
    const float max_v = (bc > da) ? bc : da;
    const float max_h = (ab > cd) ? ab : cd;
    const int v_samp = (int)((max_v / (max_v + max_h)) * 2.0 * (double)std::sqrt((float)nsam));
    const int h_samp = (int)((max_h / (max_v + max_h)) * 2.0 * (double)std::sqrt((float)nsam));
    L.pt_base = (int)(pts.size() / 9);
    if (nsam == 1) {
        // fillQuad returns 1 without filling; illuminate() then samples the
        // whole quad (arealight.cc:115-130)
        L.samples = 1;
        return YR_OK;
    }
    if (v_samp * h_samp > nsam) return YR_ERR_UNSUPPORTED;  // the reference would write past its array
    const V3 inc_v_a = h_div(dd - a, (float)v_samp), inc_v_b = h_div(c - b, (float)v_samp);
    V3 line_a = a + 0.5f * inc_v_a, line_b = b + 0.5f * inc_v_b;
    int index = 0;
    for (int i = 0; i < v_samp; ++i) {
        const V3 inc_h = h_div(line_b - line_a, (float)h_samp);
        V3 point = line_a + 0.5f * inc_h;
        for (int j = 0; j < h_samp; ++j) {
            const float vf = ((float)j) / ((float)h_samp);
            const V3 inc_v = inc_v_a * (float)(1.0 - vf) + inc_v_b * vf;
            const float rec[9] = {point.x, point.y, point.z, inc_h.x, inc_h.y, inc_h.z, inc_v.x, inc_v.y, inc_v.z};
            pts.insert(pts.end(), rec, rec + 9);
            index++;
            point = point + inc_h;
        }
        line_a = line_a + inc_v_a;
        line_b = line_b + inc_v_b;
    }
    L.samples = index;
    return YR_OK;
}

yr_status make_lights(const std::vector<yr_light_desc> &in, std::vector<DevLight> &out, std::vector<float> &pts) {
    out.clear();
    pts.clear();
    for (const yr_light_desc &d : in) {
        DevLight L;
        std::memset(&L, 0, sizeof(L));
        L.type = (int)d.type;
        L.color = c3(d.color[0], d.color[1], d.color[2]);
        L.rawc = L.color;
        L.power = d.power;
        L.samples = d.samples;
        L.depth = d.depth;
        L.cast = d.cast_shadows ? 1 : 0;
        L.maxdist = d.maxdist;
        switch (d.type) {
        case YR_LIGHT_POINT:
            L.from = hv(d.p[0]);
            L.color = L.color * d.power;  // pointLight_t ctor: color = c*inte
            break;
        case YR_LIGHT_AREA: {
            yr_status st = fill_quad(d, L, pts);
            if (st != YR_OK) return st;
            if (d.psamples < 0 || d.psamples > 64) return YR_ERR_INVALID_ARG;
            // the guess runs only with more than one sample (arealight.cc:115-134)
            L.psamples = L.samples > 1 ? d.psamples : 0;
            const V3 a = hv(d.p[0]), b = hv(d.p[1]), c = hv(d.p[2]), dd = hv(d.p[3]);
            L.direction = h_normalize(cross(b - a, dd - a));
            L.from = (((a + b) + c) + dd) * 0.25f;
            L.corner = a;
            L.tox = b - a;
            L.toy = dd - a;
            break;
        }
        case YR_LIGHT_HEMI:
            if (d.samples < 1) return YR_ERR_INVALID_ARG;
            L.sampdiv = d.power / (float)d.samples;
            break;
        case YR_LIGHT_PATH:
            if (d.samples < 1 || d.depth < 0) return YR_ERR_INVALID_ARG;
            break;
        default:
            return YR_ERR_UNSUPPORTED;
        }
        out.push_back(L);
    }
    // probe slots of a vertex follow its sample slots
    int ns = 0;
    for (const DevLight &L : out)
        ns += L.type == YR_LIGHT_POINT ? 1 : (L.type == YR_LIGHT_AREA || L.type == YR_LIGHT_HEMI ? L.samples : 0);
    for (DevLight &L : out)
        if (L.psamples > 0) {
            L.probe_off = ns;
            ns += L.psamples;
        }
    return YR_OK;
}

// camera_t ctor for CM_PERSPECTIVE (camera.cc:27-87)
// camera_t ctor (camera.cc:27-87), perspective, in the shipped build's
// (-O3 -ffast-math) evaluation: vto.normLen() as a float division 1/|vto|,
// and the divisions by resx and resy as products with their reciprocals
// (vup scaled by (resy*aspect) * (1/resx), then by 1/resy; vright by 1/resx).
void make_camera(const yr_camera_desc &c, DevCamera &o) {
    const V3 pos = hv(c.pos);
    V3 vup = hv(c.up) - pos;
    V3 vto = hv(c.look) - pos;
    V3 vright = cross(vup, vto);
    vup = cross(vright, vto);
    vup = h_normalize(vup);
    vright = h_normalize(vright);
    vright = vright * -1.0f;
    // fdist = vto.normLen()
    {
        float vl = vto.x * vto.x + vto.y * vto.y + vto.z * vto.z;
        if (vl != 0.f) {
            vl = std::sqrt(vl);
            const float dv = 1.0f / vl;
            vto.x *= dv;
            vto.y *= dv;
            vto.z *= dv;
        }
    }
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

yr_status upload_params(yr_scene *s) {
    if (!s->shaders.empty() &&
        cudaMemcpy(s->d_shaders, s->shaders.data(), sizeof(DevShader) * s->shaders.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess)
        return YR_ERR_CUDA;
    if (!s->lights.empty() &&
        cudaMemcpy(s->d_lights, s->lights.data(), sizeof(DevLight) * s->lights.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess)
        return YR_ERR_CUDA;
    return YR_OK;
}

yr_status take_status(yr_scene *s, cudaStream_t stream) {
    if (cudaMemcpyAsync(s->status_host, s->status, sizeof(int), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        return YR_ERR_CUDA;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return YR_ERR_CUDA;
    const int code = *s->status_host;
    if (code != 0) {
        if (cudaMemsetAsync(s->status, 0, sizeof(int), stream) != cudaSuccess) return YR_ERR_CUDA;
        if (cudaStreamSynchronize(stream) != cudaSuccess) return YR_ERR_CUDA;
        return (yr_status)code;
    }
    return YR_OK;
}

}  // namespace yr

using namespace yr;

static void destroy_scene(yr_scene *s) {
    if (!s) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    for (DevBuf &b : s->bufs) cudaFree(b.p);
    for (DevBuf &b : s->scratch) cudaFree(b.p);
    if (s->pooled) pool_scene_count(s->device, -1);
    if (s->status) cudaFree(s->status);
    if (s->status_host) cudaFreeHost(s->status_host);
    cudaSetDevice(prev);
    delete s;
}

extern "C" {

YR_API yr_status yr_scene_create(const yr_scene_desc *desc, int device, yr_scene **out) {
    if (!desc || !out) return YR_ERR_INVALID_ARG;
    *out = nullptr;
    if (desc->nobjects == 0 || !desc->objects) return YR_ERR_EMPTY_SCENE;
    if (desc->nshaders == 0 || !desc->shaders) return YR_ERR_INVALID_ARG;
    if (desc->nlights && !desc->lights) return YR_ERR_INVALID_ARG;
    if (desc->camera.resx <= 0 || desc->camera.resy <= 0) return YR_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return YR_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return YR_ERR_INVALID_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return YR_ERR_CUDA;

    yr_scene *s = new (std::nothrow) yr_scene;
    if (!s) return YR_ERR_OUT_OF_MEMORY;
    s->device = device;
    yr_status st = YR_OK;
    auto fail = [&](yr_status e) {
        destroy_scene(s);
        cudaSetDevice(prev);
        return e;
    };
    const auto t0 = std::chrono::steady_clock::now();

    // ---- geometry: per-object trees flattened into global arrays
    std::vector<float4> tris;
    std::vector<uint2> nodes;
    std::vector<uint32_t> prims, tri_shader;
    std::vector<float> tri_nrm;  // 9 per triangle (corner normals) up to the last smoothed object
    std::vector<float> tri_uv;   // 6 per triangle (texture coordinates) up to the last object with them
    std::vector<float4> orco_m;  // 3 rows per mesh with an orco matrix
    std::vector<DevObject> objects;
    std::vector<Box> obounds;
    size_t total_tris = 0;
    std::vector<DevInst> insts;
    auto is_inst = [&](uint32_t o) { return desc->objects[o].instance_matrix != nullptr; };
    for (uint32_t o = 0; o < desc->nobjects; o++)
        if (!is_inst(o)) total_tris += desc->objects[o].ntris;
    if (total_tris == 0) return fail(YR_ERR_EMPTY_SCENE);
    if (total_tris >= (1u << 30)) return fail(YR_ERR_TOO_LARGE);
    tris.reserve(3 * total_tris);
    tri_shader.reserve(total_tris);
    for (uint32_t o = 0; o < desc->nobjects; o++) {
        const yr_object_desc &od = desc->objects[o];
        if (is_inst(o)) {  // a reference to a mesh (not to another reference)
            if (od.instance_of >= desc->nobjects || is_inst(od.instance_of)) return fail(YR_ERR_INVALID_ARG);
            for (int k = 0; k < 16; k++)
                if (!std::isfinite(od.instance_matrix[k])) return fail(YR_ERR_INVALID_ARG);
            if (desc->render.flags & YR_RENDER_SHADOW_TREE) return fail(YR_ERR_UNSUPPORTED);
            continue;
        }
        if (od.ntris == 0 || !od.verts || !od.tris) return fail(YR_ERR_EMPTY_SCENE);
        if (od.shader != YR_PER_TRIANGLE && od.shader >= desc->nshaders) return fail(YR_ERR_INVALID_ARG);
        if (od.shader == YR_PER_TRIANGLE && !od.tri_shaders) return fail(YR_ERR_INVALID_ARG);
    }
    // kd-trees of different objects are independent: build them on all host
    // cores (each tree is the same as a sequential build)
    std::vector<KdTree> trees(desc->nobjects);
    std::vector<yr_status> tree_st(desc->nobjects, YR_OK);
    std::vector<char> built(desc->nobjects, 0);
    if (desc->render.flags & YR_RENDER_GPU_KD_BUILD) {  // all meshes' trees in one GPU build
        std::vector<KdMesh> ms;
        std::vector<uint32_t> which;
        for (uint32_t o = 0; o < desc->nobjects; o++) {
            const yr_object_desc &od = desc->objects[o];
            if (is_inst(o) || od.tree) continue;
            ms.push_back(KdMesh{od.verts, od.nverts, od.tris, od.ntris});
            which.push_back(o);
        }
        if (!ms.empty()) {
            std::vector<KdTree> gt;
            yr_status gs;
            try {
                gs = build_kdtrees_gpu(ms, KdParams(), device, gt);
            } catch (const std::bad_alloc &) {
                gs = YR_ERR_OUT_OF_MEMORY;
            }
            if (gs != YR_OK) return fail(gs);
            for (size_t i = 0; i < which.size(); i++) {
                trees[which[i]] = std::move(gt[i]);
                built[which[i]] = 1;
            }
        }
    }
    {
        std::atomic<uint32_t> next{0};
        auto worker = [&] {
            for (;;) {
                const uint32_t o = next.fetch_add(1);
                if (o >= desc->nobjects) return;
                if (is_inst(o)) continue;  // shares its original's tree
                if (built[o]) continue;
                const yr_object_desc &od = desc->objects[o];
                KdTree &tree = trees[o];
                try {
                    if (od.tree) {
                        tree.nodes.assign(od.tree->nodes, od.tree->nodes + od.tree->nnodes);
                        tree.prims.assign(od.tree->prims, od.tree->prims + od.tree->nprims);
                        std::memcpy(tree.bound.a, od.tree->bound, 12);
                        std::memcpy(tree.bound.g, od.tree->bound + 3, 12);
                        tree.max_depth = od.tree->max_depth;
                    } else {
                        tree_st[o] = build_kdtree(od.verts, od.nverts, od.tris, od.ntris, tree);
                    }
                } catch (const std::bad_alloc &) {
                    tree_st[o] = YR_ERR_OUT_OF_MEMORY;
                }
            }
        };
        unsigned nth = std::thread::hardware_concurrency();
        nth = std::max(1u, std::min(nth ? nth : 1u, desc->nobjects));
        std::vector<std::thread> pool;
        for (unsigned t = 1; t < nth; t++) pool.emplace_back(worker);
        worker();
        for (std::thread &t : pool) t.join();
    }
    for (uint32_t o = 0; o < desc->nobjects; o++) {
        const yr_object_desc &od = desc->objects[o];
        if (is_inst(o)) {  // filled in below, once every mesh is placed
            objects.push_back(DevObject{});
            obounds.push_back(Box{});
            continue;
        }
        if (tree_st[o] != YR_OK) return fail(tree_st[o]);
        KdTree tree = std::move(trees[o]);
        if (tree.max_depth > s->max_tree_depth) s->max_tree_depth = tree.max_depth;
        const uint32_t tri_base = (uint32_t)(tris.size() / 3);
        const uint32_t node_base = (uint32_t)nodes.size();
        const uint32_t prim_base = (uint32_t)prims.size();
        for (uint32_t t = 0; t < od.ntris; t++) {
            uint32_t vi[3];
            for (int k = 0; k < 3; k++) {
                vi[k] = od.tris[3 * (size_t)t + k];
                if (vi[k] >= od.nverts) return fail(YR_ERR_INVALID_ARG);
            }
            const V3 a = hv(od.verts + 3 * (size_t)vi[0]);
            const V3 b = hv(od.verts + 3 * (size_t)vi[1]);
            const V3 c = hv(od.verts + 3 * (size_t)vi[2]);
            // triangle_t ctor: normal = normalize((b-a)^(c-a)) (triangle.cc:30-43)
            const V3 n = h_normalize(cross(b - a, c - a));
            tris.push_back(make_float4(a.x, a.y, a.z, n.x));
            tris.push_back(make_float4(b.x, b.y, b.z, n.y));
            tris.push_back(make_float4(c.x, c.y, c.z, n.z));
            const uint32_t sh = od.shader == YR_PER_TRIANGLE ? od.tri_shaders[t] : od.shader;
            if (sh >= desc->nshaders) return fail(YR_ERR_INVALID_ARG);
            tri_shader.push_back(sh);
        }
        // smoothed objects: the corner normals of meshObject_t::autoSmooth
        const bool smooth = od.smooth_angle >= 1.f;
        if (smooth) {
            std::vector<float> cn;
            smooth_normals(od.verts, od.tris, od.nverts, od.ntris, od.smooth_angle, cn);
            if (tri_nrm.size() < 9 * (size_t)tri_base) tri_nrm.resize(9 * (size_t)tri_base, 0.f);
            tri_nrm.insert(tri_nrm.end(), cn.begin(), cn.end());
        }
        // texture coordinates (the mesh's facesuv), 6 per triangle
        if (od.uvs) {
            for (size_t k = 0; k < 6 * (size_t)od.ntris; k++)
                if (!std::isfinite(od.uvs[k])) return fail(YR_ERR_INVALID_ARG);
            if (tri_uv.size() < 6 * (size_t)tri_base) tri_uv.resize(6 * (size_t)tri_base, 0.f);
            tri_uv.insert(tri_uv.end(), od.uvs, od.uvs + 6 * (size_t)od.ntris);
        }
        for (const yr_kd_node &nd : tree.nodes) {
            uint2 g;
            g.y = nd.flags;
            g.x = nd.word;
            if ((nd.flags & 3u) != 3u) {
                const uint32_t right = (nd.flags >> 2) + node_base;
                if ((nd.flags >> 2) >= tree.nodes.size() || right >= (1u << 30)) return fail(YR_ERR_BAD_TREE);
                g.y = (nd.flags & 3u) | (right << 2);
            } else {
                const uint32_t np = nd.flags >> 2;
                if (np == 1) {
                    if (nd.word >= od.ntris) return fail(YR_ERR_BAD_TREE);
                    g.x = nd.word + tri_base;
                } else if (np > 1) {
                    if ((size_t)nd.word + np > tree.prims.size()) return fail(YR_ERR_BAD_TREE);
                    g.x = nd.word + prim_base;
                }
            }
            nodes.push_back(g);
        }
        for (uint32_t p : tree.prims) {
            if (p >= od.ntris) return fail(YR_ERR_BAD_TREE);
            prims.push_back(p + tri_base);
        }
        DevObject dob;
        std::memcpy(dob.tb, tree.bound.a, 12);
        std::memcpy(dob.tb + 3, tree.bound.g, 12);
        dob.root = node_base;
        dob.tri_base = tri_base;
        dob.ntris = od.ntris;
        dob.flags = (od.cast_shadows ? 1u : 0u) | (smooth ? 2u : 0u) | (od.uvs ? 4u : 0u);
        const Box obb = mesh_bound(od.verts, od.tris, od.ntris);
        std::memcpy(dob.ob, obb.a, 12);
        std::memcpy(dob.ob + 3, obb.g, 12);
        dob.inst = -1;
        dob.orco = -1;
        if (od.orco_matrix) {  // toObjectOrco of a transformed mesh: rows 0-2 of backOrco
            for (int k = 0; k < 12; k++)
                if (!std::isfinite(od.orco_matrix[k])) return fail(YR_ERR_INVALID_ARG);
            dob.orco = (int)(orco_m.size() / 3);
            for (int r = 0; r < 3; r++)
                orco_m.push_back(make_float4(od.orco_matrix[4 * r], od.orco_matrix[4 * r + 1], od.orco_matrix[4 * r + 2],
                                             od.orco_matrix[4 * r + 3]));
        }
        objects.push_back(dob);
        obounds.push_back(obb);
    }
    // references (referenceObject_t): the original's tree, triangles,
    // shading flags and shadow flag (reference.cc:38-44), its own matrices
    // and the placed box of the original's bound
    for (uint32_t o = 0; o < desc->nobjects; o++) {
        if (!is_inst(o)) continue;
        const yr_object_desc &od = desc->objects[o];
        InstanceXf xf;
        if (!instance_xf(od.instance_matrix, xf)) return fail(YR_ERR_INVALID_ARG);  // singular matrix
        if (od.instance_inverse)  // the caller's M^-1 (e.g. referenceObject_t::back)
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 4; j++) xf.back[4 * i + j] = od.instance_inverse[4 * i + j];
        DevInst di{};
        std::memcpy(di.m, xf.m, sizeof(xf.m));
        std::memcpy(di.back, xf.back, sizeof(xf.back));
        std::memcpy(di.rot, xf.rot, sizeof(xf.rot));
        DevObject dob = objects[od.instance_of];
        const Box ob = instance_bound(obounds[od.instance_of], od.instance_matrix);
        std::memcpy(dob.ob, ob.a, 12);
        std::memcpy(dob.ob + 3, ob.g, 12);
        dob.inst = (int)insts.size();
        insts.push_back(di);
        objects[o] = dob;
        obounds[o] = ob;
    }
    // shadow-ray tree over the triangles of every shadow-casting object
    std::vector<uint2> sh_nodes;
    std::vector<uint32_t> sh_prims, tri_obj(total_tris);
    float sh_tb[6] = {0, 0, 0, 0, 0, 0};
    {
        std::vector<float> mv;
        std::vector<uint32_t> mt, remap;
        for (uint32_t o = 0; o < desc->nobjects; o++) {
            if (is_inst(o)) continue;  // (no shadow-ray tree with references)
            const yr_object_desc &od = desc->objects[o];
            for (uint32_t t = 0; t < od.ntris; t++) tri_obj[objects[o].tri_base + t] = o;
            if (!od.cast_shadows) continue;
            const uint32_t vbase = (uint32_t)(mv.size() / 3);
            mv.insert(mv.end(), od.verts, od.verts + 3 * (size_t)od.nverts);
            for (size_t k = 0; k < 3 * (size_t)od.ntris; k++) mt.push_back(od.tris[k] + vbase);
            for (uint32_t t = 0; t < od.ntris; t++) remap.push_back(objects[o].tri_base + t);
        }
        if (!remap.empty() && (desc->render.flags & YR_RENDER_SHADOW_TREE)) {
            KdTree st_tree;
            KdParams kp;
            kp.max_leaf = 1;                   // deeper tree, fewer triangle tests
            kp.large_scene_penalty = false;
            unsigned nth = std::thread::hardware_concurrency();
            st = build_kdtree(mv.data(), (uint32_t)(mv.size() / 3), mt.data(), (uint32_t)remap.size(), st_tree, kp,
                              (int)std::max(1u, nth));
            if (st != YR_OK) return fail(st);
            if (st_tree.nodes.size() >= kNodeMask) return fail(YR_ERR_TOO_LARGE);
            if (st_tree.max_depth + 2 > kKdStackCap) return fail(YR_ERR_TOO_LARGE);
            sh_nodes.reserve(st_tree.nodes.size());
            for (const yr_kd_node &nd : st_tree.nodes) {
                uint2 g;
                g.x = nd.word;
                g.y = nd.flags;
                if ((nd.flags & 3u) == 3u && (nd.flags >> 2) == 1) g.x = remap[nd.word];
                sh_nodes.push_back(g);
            }
            sh_prims.reserve(st_tree.prims.size());
            for (uint32_t p : st_tree.prims) sh_prims.push_back(remap[p]);
            std::memcpy(sh_tb, st_tree.bound.a, 12);
            std::memcpy(sh_tb + 3, st_tree.bound.g, 12);
        }
    }
    std::vector<ObjNode> otree;
    build_object_tree(obounds, otree);
    // traversal state is sized for these limits (kd stack: depth + 2 exits)
    if (nodes.size() >= kNodeMask) return fail(YR_ERR_TOO_LARGE);
    // every index the device walk follows stays inside its array (the walk
    // itself only checks the stack and an iteration cap)
    if (!valid_tree(nodes, prims, total_tris) || !valid_tree(sh_nodes, sh_prims, total_tris))
        return fail(YR_ERR_BAD_TREE);
    for (const DevObject &o : objects)
        if (o.ntris && o.root >= nodes.size()) return fail(YR_ERR_BAD_TREE);
    if (s->max_tree_depth + 2 > kKdStackCap) return fail(YR_ERR_TOO_LARGE);
    {
        int depth = 0;
        std::vector<std::pair<int, int>> st{{0, 0}};
        while (!st.empty()) {
            auto [n, d] = st.back();
            st.pop_back();
            depth = std::max(depth, d);
            if (otree[n].left >= 0) {
                st.push_back({otree[n].left, d + 1});
                st.push_back({otree[n].right, d + 1});
            }
        }
        if (depth > kMaxObjStack) return fail(YR_ERR_UNSUPPORTED);
    }
    const auto t1 = std::chrono::steady_clock::now();

    // ---- upload
    const float4 *d_tris;
    const uint2 *d_nodes;
    const uint32_t *d_prims, *d_tri_shader;
    const DevObject *d_objects;
    // object trees for the device: one 64-byte record per interior node
    // holding both children's boxes and codes (>= 0: interior record,
    // < 0: ~object), so that a step of the walk is one dependent load
    auto flatten_objtree = [](const std::vector<ObjNode> &t, std::vector<float4> &recs, int &root) {
        recs.clear();
        root = -1;
        if (t.empty()) return;
        std::vector<int> rec(t.size(), -1);
        int nrec = 0;
        for (size_t n = 0; n < t.size(); n++)
            if (t[n].left >= 0) rec[n] = nrec++;
        auto code = [&](int n) { return t[n].left >= 0 ? rec[n] : ~t[n].right; };
        recs.resize(4 * (size_t)nrec);
        for (size_t n = 0; n < t.size(); n++) {
            if (t[n].left < 0) continue;
            const ObjNode &L = t[t[n].left], &R = t[t[n].right];
            float4 *o = &recs[4 * (size_t)rec[n]];
            o[0] = make_float4(L.bmin[0], L.bmin[1], L.bmin[2], L.bmax[0]);
            o[1] = make_float4(L.bmax[1], L.bmax[2], R.bmin[0], R.bmin[1]);
            o[2] = make_float4(R.bmin[2], R.bmax[0], R.bmax[1], R.bmax[2]);
            const int lc = code(t[n].left), rc = code(t[n].right);
            float lf, rf;
            std::memcpy(&lf, &lc, 4);
            std::memcpy(&rf, &rc, 4);
            o[3] = make_float4(lf, rf, 0.f, 0.f);
        }
        root = code(0);
    };
    std::vector<float4> onodes, sonodes;
    int oroot = -1, soroot = -1;
    flatten_objtree(otree, onodes, oroot);
    // shadow rays: an SAH BVH over the objects that cast shadows
    std::vector<ObjNode> sotree;
    {
        std::vector<int> casters;
        for (uint32_t o = 0; o < desc->nobjects; o++)
            if (objects[o].flags & 1u) casters.push_back((int)o);
        build_sah_object_bvh(obounds, casters, sotree);
        int depth = 0;
        std::vector<std::pair<int, int>> stk;
        if (!sotree.empty()) stk.push_back({0, 0});
        while (!stk.empty()) {
            auto [n, d] = stk.back();
            stk.pop_back();
            depth = std::max(depth, d);
            if (sotree[n].left >= 0) {
                stk.push_back({sotree[n].left, d + 1});
                stk.push_back({sotree[n].right, d + 1});
            }
        }
        if (depth > kMaxObjStack) return fail(YR_ERR_UNSUPPORTED);
        flatten_objtree(sotree, sonodes, soroot);
    }
    const float4 *d_onodes = nullptr;
    if ((st = dev_upload(s, tris.data(), tris.size(), (float4 **)&d_tris)) != YR_OK) return fail(st);
    if ((st = dev_upload(s, nodes.data(), nodes.size(), (uint2 **)&d_nodes)) != YR_OK) return fail(st);
    if (!prims.empty() && (st = dev_upload(s, prims.data(), prims.size(), (uint32_t **)&d_prims)) != YR_OK)
        return fail(st);
    if (prims.empty()) d_prims = nullptr;
    if ((st = dev_upload(s, tri_shader.data(), tri_shader.size(), (uint32_t **)&d_tri_shader)) != YR_OK)
        return fail(st);
    const float *d_tri_nrm = nullptr, *d_tri_uv = nullptr;
    if ((st = dev_upload(s, tri_nrm.data(), tri_nrm.size(), (float **)&d_tri_nrm)) != YR_OK) return fail(st);
    if ((st = dev_upload(s, tri_uv.data(), tri_uv.size(), (float **)&d_tri_uv)) != YR_OK) return fail(st);
    const float4 *d_orco_m = nullptr;
    if ((st = dev_upload(s, orco_m.data(), orco_m.size(), (float4 **)&d_orco_m)) != YR_OK) return fail(st);
    if ((st = dev_upload(s, objects.data(), objects.size(), (DevObject **)&d_objects)) != YR_OK) return fail(st);
    const DevInst *d_insts = nullptr;
    if (!insts.empty() && (st = dev_upload(s, insts.data(), insts.size(), (DevInst **)&d_insts)) != YR_OK)
        return fail(st);
    if ((st = dev_upload(s, onodes.data(), onodes.size(), (float4 **)&d_onodes)) != YR_OK) return fail(st);
    const float4 *d_sonodes = nullptr;
    if ((st = dev_upload(s, sonodes.data(), sonodes.size(), (float4 **)&d_sonodes)) != YR_OK) return fail(st);
    const uint2 *d_sh_nodes = nullptr;
    const uint32_t *d_sh_prims = nullptr, *d_tri_obj = nullptr;
    if ((st = dev_upload(s, sh_nodes.data(), sh_nodes.size(), (uint2 **)&d_sh_nodes)) != YR_OK) return fail(st);
    if ((st = dev_upload(s, sh_prims.data(), sh_prims.size(), (uint32_t **)&d_sh_prims)) != YR_OK) return fail(st);
    if ((st = dev_upload(s, tri_obj.data(), tri_obj.size(), (uint32_t **)&d_tri_obj)) != YR_OK) return fail(st);
    // [0] status word, [1] work counter of the ray-query kernels
    if (cudaMalloc(&s->status, 2 * sizeof(int)) != cudaSuccess) return fail(YR_ERR_OUT_OF_MEMORY);
    if (cudaMemset(s->status, 0, 2 * sizeof(int)) != cudaSuccess) return fail(YR_ERR_CUDA);
    if (cudaMallocHost(&s->status_host, sizeof(int)) != cudaSuccess) return fail(YR_ERR_OUT_OF_MEMORY);

    DevScene &D = s->dev;
    D.tris = d_tris;
    D.nodes = d_nodes;
    D.prims = d_prims;
    D.objects = d_objects;
    D.insts = d_insts;
    D.tri_nrm = d_tri_nrm;
    D.tri_uv = d_tri_uv;
    D.orco_m = d_orco_m;
    D.onodes = d_onodes;
    D.oroot = oroot;
    D.sonodes = d_sonodes;
    D.soroot = soroot;
    D.nsotree = (uint32_t)sotree.size();
    if (!sotree.empty()) {
        std::memcpy(D.sotb, sotree[0].bmin, 12);
        std::memcpy(D.sotb + 3, sotree[0].bmax, 12);
    }
    if (!otree.empty()) {
        std::memcpy(D.otb, otree[0].bmin, 12);
        std::memcpy(D.otb + 3, otree[0].bmax, 12);
    }
    D.nobjects = desc->nobjects;
    D.ntris = (uint32_t)total_tris;
    D.nnodes = (uint32_t)nodes.size();
    D.nprims = (uint32_t)prims.size();
    D.notree = (uint32_t)otree.size();
    D.sh_nodes = d_sh_nodes;
    D.sh_prims = d_sh_prims;
    D.tri_obj = d_tri_obj;
    D.sh_nnodes = (uint32_t)sh_nodes.size();
    D.sh_nprims = (uint32_t)sh_prims.size();
    std::memcpy(D.sh_tb, sh_tb, sizeof(sh_tb));
    D.use_sh_tree = (desc->render.flags & YR_RENDER_SHADOW_TREE) ? 1 : 0;
    D.exact_order = (desc->render.flags & YR_RENDER_EXACT_ORDER) ? 1 : 0;
    D.coord_max = 0.f;
    if (!otree.empty())
        for (int k = 0; k < 3; k++)
            D.coord_max = std::max(D.coord_max, std::max(std::fabs(otree[0].bmin[k]), std::fabs(otree[0].bmax[k])));
    D.status = s->status;

    // ---- shading records
    s->shader_desc.assign(desc->shaders, desc->shaders + desc->nshaders);
    s->light_desc.assign(desc->lights, desc->lights + desc->nlights);
    s->shaders.resize(desc->nshaders);
    for (uint32_t i = 0; i < desc->nshaders; i++) {
        if (!valid_shader(desc->shaders[i])) return fail(YR_ERR_INVALID_ARG);
        make_shader(desc->shaders[i], s->shaders[i]);
    }
    if ((st = make_lights(s->light_desc, s->lights, s->area_pts)) != YR_OK) return fail(st);
    if ((st = dev_upload(s, s->shaders.data(), s->shaders.size(), &s->d_shaders)) != YR_OK) return fail(st);
    if (!s->lights.empty() && (st = dev_upload(s, s->lights.data(), s->lights.size(), &s->d_lights)) != YR_OK)
        return fail(st);
    const float *d_pts = nullptr;
    if (!s->area_pts.empty() && (st = dev_upload(s, s->area_pts.data(), s->area_pts.size(), (float **)&d_pts)) != YR_OK)
        return fail(st);
    s->camera = desc->camera;
    s->render = desc->render;
    DevRender &R = s->rdr;
    make_camera(desc->camera, R.cam);
    R.shaders = s->d_shaders;
    R.lights = s->d_lights;
    R.area_pts = d_pts;
    R.tri_shader = d_tri_shader;
    R.nlights = (int)s->lights.size();
    R.nshaders = (int)s->shaders.size();
    R.has_guess = 0;
    for (const DevLight &L : s->lights)
        if (L.psamples > 0) R.has_guess = 1;
    R.spp = desc->render.spp ? desc->render.spp : 1;
    R.pw = desc->render.aa_pixelwidth;
    R.totsamdiv = R.spp > 1 ? (float)(1.0 / (float)(R.spp - 1)) : 0.f;
    R.seed = desc->render.seed;
    R.self_bias = desc->render.self_bias;
    // scene_t::setExposure / setGamma (scene.h:162-163), tonemap, clampRGB,
    // alphaPremultiply
    R.tonemap = (desc->render.flags & YR_RENDER_TONEMAP) ? 1 : 0;
    R.clamp_rgb = (desc->render.flags & YR_RENDER_CLAMP_RGB) ? 1 : 0;
    R.premultiply = (desc->render.flags & YR_RENDER_ALPHA_PREMULTIPLY) ? 1 : 0;
    R.exposure = -desc->render.exposure;
    // gamma 0 makes every sample pow(x, 0) = 1 (white); not supported
    if (R.tonemap && desc->render.gamma == 0.0f) return fail(YR_ERR_UNSUPPORTED);
    R.gamma_r = desc->render.gamma != 0.0f ? (float)(1.0 / (double)desc->render.gamma) : 0.0f;
    R.raydepth = desc->render.raydepth;
    R.background = c3(desc->render.background[0], desc->render.background[1], desc->render.background[2]);
    {
        const int32_t *rg = desc->render.region;
        if (rg[0] == 0 && rg[1] == 0 && rg[2] == 0 && rg[3] == 0) {
            R.rx0 = 0;
            R.ry0 = 0;
            R.rw = desc->camera.resx;
            R.rh = desc->camera.resy;
        } else {
            if (rg[0] < 0 || rg[1] > desc->camera.resx || rg[0] >= rg[1] || rg[2] < 0 || rg[3] > desc->camera.resy ||
                rg[2] >= rg[3])
                return fail(YR_ERR_INVALID_ARG);
            R.rx0 = rg[0];
            R.ry0 = rg[2];
            R.rw = rg[1] - rg[0];
            R.rh = rg[3] - rg[2];
        }
    }
    R.path_light = -1;
    for (int i = 0; i < R.nlights; i++)
        if (s->lights[i].type == YR_LIGHT_PATH) {
            if (R.path_light >= 0) return fail(YR_ERR_UNSUPPORTED);  // one path light per scene
            R.path_light = i;
            R.path_samples = s->lights[i].samples;
            R.path_depth = s->lights[i].depth;
        }
    R.path_threshold = 0.f;
    if (R.path_light >= 0) {
        const float t = s->light_desc[R.path_light].threshold;
        if (!(t <= 0.f) && !std::isfinite(t)) return fail(YR_ERR_INVALID_ARG);
        R.path_threshold = t > 0.f ? t : 0.f;
    }

    // ---- adjoint parameter vector (yr_param_count): per shader color[3] and
    // specular weight, plus amplitude and base colour for textured shaders;
    // per light its power
    {
        uint32_t n = 0;
        s->sh_pbase.resize(s->shaders.size());
        s->spec_dir.assign(4 * s->shaders.size(), 0.f);
        for (size_t i = 0; i < s->shaders.size(); i++) {
            s->sh_pbase[i] = (int)n;
            n += 4 + (s->shader_desc[i].tex_type != YR_TEX_NONE ? 4 : 0);
            const float *ks = s->shader_desc[i].specular;
            const float w = std::max(ks[0], std::max(ks[1], ks[2]));
            for (int k = 0; k < 3; k++) s->spec_dir[4 * i + k] = w > 0.f ? ks[k] / w : 1.f;
        }
        s->li_pidx.resize(s->lights.size());
        for (size_t i = 0; i < s->lights.size(); i++) s->li_pidx[i] = (int)n++;
        s->nparams = n;
        if ((st = dev_upload(s, s->sh_pbase.data(), s->sh_pbase.size(), &s->d_sh_pbase)) != YR_OK) return fail(st);
        if (!s->li_pidx.empty() && (st = dev_upload(s, s->li_pidx.data(), s->li_pidx.size(), &s->d_li_pidx)) != YR_OK)
            return fail(st);
        if ((st = dev_upload(s, (const float4 *)s->spec_dir.data(), s->shaders.size(), &s->d_spec_dir)) != YR_OK)
            return fail(st);
    }

    yr_scene_info &I = s->info;
    I.nobjects = desc->nobjects;
    I.ntriangles = (uint32_t)total_tris;
    I.nnodes = (uint32_t)nodes.size();
    I.nprims = (uint32_t)prims.size();
    I.nlights = desc->nlights;
    I.device_bytes = 0;
    for (const DevBuf &b : s->bufs) I.device_bytes += b.bytes;
    I.build_seconds = std::chrono::duration<double>(t1 - t0).count();
    pool_scene_count(s->device, +1);
    s->pooled = true;
    cudaSetDevice(prev);
    *out = s;
    return YR_OK;
}

YR_API yr_status yr_scene_destroy(yr_scene *scene) {
    if (!scene) return YR_ERR_INVALID_ARG;
    batch_forget(scene);
    adj_batch_forget(scene);
    destroy_scene(scene);
    return YR_OK;
}

YR_API yr_status yr_scene_info_get(const yr_scene *scene, yr_scene_info *info) {
    if (!scene || !info) return YR_ERR_INVALID_ARG;
    *info = scene->info;
    return YR_OK;
}

YR_API yr_status yr_scene_set_camera_vectors(yr_scene *scene, const float *pos, const float *vto, const float *vup,
                                             const float *vright) {
    if (!scene || !pos || !vto || !vup || !vright) return YR_ERR_INVALID_ARG;
    for (int k = 0; k < 3; k++)
        if (!std::isfinite(pos[k]) || !std::isfinite(vto[k]) || !std::isfinite(vup[k]) || !std::isfinite(vright[k]))
            return YR_ERR_INVALID_ARG;
    DevCamera &c = scene->rdr.cam;
    c.pos = v3(pos[0], pos[1], pos[2]);
    c.vto = v3(vto[0], vto[1], vto[2]);
    c.vup = v3(vup[0], vup[1], vup[2]);
    c.vright = v3(vright[0], vright[1], vright[2]);
    // batched renders and adjoint steps captured before keep kernel
    // arguments with the old camera: drop them so they are captured again
    batch_forget(scene);
    adj_batch_forget(scene);
    return YR_OK;
}

YR_API yr_status yr_scene_set_params(yr_scene *scene, const yr_shader_desc *shaders, const yr_light_desc *lights) {
    if (!scene) return YR_ERR_INVALID_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(scene->device);
    if (shaders) {
        for (size_t i = 0; i < scene->shader_desc.size(); i++)
            if (!valid_shader(shaders[i])) {
                cudaSetDevice(prev);
                return YR_ERR_INVALID_ARG;
            }
        scene->shader_desc.assign(shaders, shaders + scene->shader_desc.size());
        for (size_t i = 0; i < scene->shaders.size(); i++) make_shader(shaders[i], scene->shaders[i]);
    }
    if (lights) {
        // geometry of the lights must not change (sample grids are fixed)
        std::vector<yr_light_desc> ld(lights, lights + scene->light_desc.size());
        std::vector<DevLight> nl;
        std::vector<float> pts;
        yr_status st = make_lights(ld, nl, pts);
        if (st != YR_OK) {
            cudaSetDevice(prev);
            return st;
        }
        if (pts != scene->area_pts) {
            cudaSetDevice(prev);
            return YR_ERR_INVALID_ARG;
        }
        scene->light_desc = ld;
        scene->lights = nl;
        if (scene->rdr.path_light >= 0) {
            const float t = ld[scene->rdr.path_light].threshold;
            scene->rdr.path_threshold = (t > 0.f && std::isfinite(t)) ? t : 0.f;
        }
    }
    yr_status st = upload_params(scene);
    cudaSetDevice(prev);
    return st;
}

}  // extern "C"
