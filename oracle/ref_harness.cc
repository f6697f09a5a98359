// Test harness around the UNMODIFIED YafRay 0.0.9 reference (linked from
// objects built from the reference sources by oracle/Makefile).  Test
// infrastructure only: it generates golden vectors for tests/golden/ and is
// the reference arm of bench.py; the product never links or runs it.
//
// Written in C++98 because the reference objects are built with -std=gnu++98.
//
//   yr_ref_harness tree    SCENE OUT           kd-trees + object tree
//   yr_ref_harness rays    SCENE RAYS OUT      kd / scene ray queries
//   yr_ref_harness camera  SCENE OUT           primary ray directions
//   yr_ref_harness instmat SCENE OUT           each reference's M^-1 (back)
//   yr_ref_harness orcomat SCENE OUT           each transformed mesh's orco matrix
//   yr_ref_cudascene iface SCENE OUT ARM [pathcache]
//                                              the scene through a yafrayInterface_t,
//                                              call by call: ARM ref = interfaceImpl_t,
//                                              cuda = cudaInterface_t (the library)
//   yr_ref_cudascene cudarender SCENE OUT [x0 x1 y0 y1 [STOP_AFTER]]
//                                              the scene through cudascene_t (the
//                                              library), a build of this file
//                                              with YR_HARNESS_CUDASCENE
//   yr_ref_harness render_blocks SCENE OUT THREADS BLOCKS [REPEATS]
//                                              listed 64x64 blocks of the frame,
//                                              threadedscene_t's worker loop
//   yr_ref_harness render  SCENE OUT THREADS [x0 x1 y0 y1 [REPEATS]]
//                                              stock scene_t::render, float sink,
//                                              ray counts, one JSON line per render
//   yr_ref_harness illum   SCENE QUERIES OUT   one light's illuminate() with the
//                                              sample stream set from outside
//   yr_ref_harness noise   POINTS OUT          newPerlin / fBm / turbulence
//   yr_ref_harness halton  OUT                 Halton setStart+getNext values
//   yr_ref_harness imgout  KIND IN OUT         float RGBA image through outTga_t /
//                                              outHDR_t (KIND tga, tga_alpha, hdr)
//   yr_ref_harness noisegen POINTS OUT         every noise basis, turbulence,
//                                              voronoi distances per metric
//   yr_ref_harness texeval SCENE POINTS OUT    each shader's texture getColor /
//                                              getFloat
//
// Private members (kdTree_t::nodes, meshObject_t::triangles, scene_t::BTree)
// are read by compiling the reference headers with private/protected
// mapped to public; no reference source is changed.
#define private public
#define protected public
#include "scene.h"
#include "threadedscene.h"
#include "mesh.h"
#include "reference.h"
#include "kdtree.h"
#include "camera.h"
#include "noise.h"
#include "mcqmc.h"
#include "texture.h"
#include "geometree.h"
#include "pointlight.h"
#include "arealight.h"
#include "hemilight.h"
#include "pathlight.h"
#include "basicshaders.h"
#include "basictex.h"
#include "targaIO.h"
#include "HDR_io.h"
#ifdef YR_HARNESS_CUDASCENE
#include "cudascene.h"
#include "cudainterface.h"
#include "sunsky.h"
#endif
#undef private
#undef protected

#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <algorithm>
#include <map>
#include <new>
#include <string>
#include <vector>

extern "C" {
#include "../include/yr.h"
}

using namespace yafray;

namespace yafray {
// basictex.cc references the JPEG loader (jpeg.cc needs jpeglib.h, absent);
// image textures are not on the path.
cBuffer_t *load_jpeg(const char *name) { return NULL; }
geomeTree_t<object3d_t> *buildObjectTree(std::list<object3d_t *> &obj_list);
noiseGenerator_t *newNoise(const std::string &ntype);
}

// Ray counters: the reference has none (mesh.cc:409-412 are unused), so
// the calls that plugins make into scene_t::isShadowed / firstHit are
// counted through link-time wrappers (-Wl,--wrap in oracle/Makefile).
// Each thread counts in its own counter record (registered on its first
// count, one cache line each), so the timed render shares no counter cache
// line between threads; a render's totals are the sum over the records
// once its threads are done.
struct RayCounter {
    long shadow, bounce;
    char pad[64 - 2 * sizeof(long)];
} __attribute__((aligned(64)));
static __thread RayCounter *t_ctr = NULL;
static std::vector<RayCounter *> g_ctrs;
static pthread_mutex_t g_ctr_mu = PTHREAD_MUTEX_INITIALIZER;
static RayCounter *my_counter() {
    if (!t_ctr) {
        void *mem = NULL;
        if (posix_memalign(&mem, 64, sizeof(RayCounter)) != 0) abort();
        t_ctr = new (mem) RayCounter();
        t_ctr->shadow = t_ctr->bounce = 0;
        pthread_mutex_lock(&g_ctr_mu);
        g_ctrs.push_back(t_ctr);
        pthread_mutex_unlock(&g_ctr_mu);
    }
    return t_ctr;
}
static void counts_reset() {
    pthread_mutex_lock(&g_ctr_mu);
    for (size_t i = 0; i < g_ctrs.size(); i++) g_ctrs[i]->shadow = g_ctrs[i]->bounce = 0;
    pthread_mutex_unlock(&g_ctr_mu);
}
static void counts_sum(long &shadow, long &bounce) {
    shadow = bounce = 0;
    pthread_mutex_lock(&g_ctr_mu);
    for (size_t i = 0; i < g_ctrs.size(); i++) {
        shadow += g_ctrs[i]->shadow;
        bounce += g_ctrs[i]->bounce;
    }
    pthread_mutex_unlock(&g_ctr_mu);
}
extern "C" {
bool __real__ZNK6yafray7scene_t10isShadowedERNS_13renderState_tERKNS_14surfacePoint_tERKNS_9point3d_tE(
    const scene_t *, renderState_t &, const surfacePoint_t &, const point3d_t &);
bool __wrap__ZNK6yafray7scene_t10isShadowedERNS_13renderState_tERKNS_14surfacePoint_tERKNS_9point3d_tE(
    const scene_t *s, renderState_t &st, const surfacePoint_t &sp, const point3d_t &l) {
    ++my_counter()->shadow;
    return __real__ZNK6yafray7scene_t10isShadowedERNS_13renderState_tERKNS_14surfacePoint_tERKNS_9point3d_tE(s, st, sp,
                                                                                                           l);
}
bool __real__ZNK6yafray7scene_t10isShadowedERNS_13renderState_tERKNS_14surfacePoint_tERKNS_10vector3d_tE(
    const scene_t *, renderState_t &, const surfacePoint_t &, const vector3d_t &);
bool __wrap__ZNK6yafray7scene_t10isShadowedERNS_13renderState_tERKNS_14surfacePoint_tERKNS_10vector3d_tE(
    const scene_t *s, renderState_t &st, const surfacePoint_t &sp, const vector3d_t &d) {
    ++my_counter()->shadow;
    return __real__ZNK6yafray7scene_t10isShadowedERNS_13renderState_tERKNS_14surfacePoint_tERKNS_10vector3d_tE(s, st,
                                                                                                            sp, d);
}
bool __real__ZNK6yafray7scene_t8firstHitERNS_13renderState_tERNS_14surfacePoint_tERKNS_9point3d_tERKNS_10vector3d_tEb(
    const scene_t *, renderState_t &, surfacePoint_t &, const point3d_t &, const vector3d_t &, bool);
bool __wrap__ZNK6yafray7scene_t8firstHitERNS_13renderState_tERNS_14surfacePoint_tERKNS_9point3d_tERKNS_10vector3d_tEb(
    const scene_t *s, renderState_t &st, surfacePoint_t &sp, const point3d_t &p, const vector3d_t &r, bool sh) {
    ++my_counter()->bounce;
    return __real__ZNK6yafray7scene_t8firstHitERNS_13renderState_tERNS_14surfacePoint_tERKNS_9point3d_tERKNS_10vector3d_tEb(
        s, st, sp, p, r, sh);
}
}

static double now_s() {
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + tv.tv_usec * 1e-6;
}

static void die(const char *msg) {
    fprintf(stderr, "yr_ref_harness: %s\n", msg);
    exit(2);
}

// ---------------------------------------------------------------- scene file
struct SceneFile {
    yr_camera_desc cam;
    yr_render_params rp;
    std::vector<yr_shader_desc> shaders;
    std::vector<yr_light_desc> lights;
    struct Obj {
        uint32_t nv, nt, shader, cast;
        float smooth;
        int32_t inst;  // >= 0: a reference to that object, placed by M
        float M[16];
        std::vector<float> v;
        std::vector<uint32_t> t;
        std::vector<uint32_t> tri_shader;  // when shader == YR_PER_TRIANGLE
        std::vector<float> uv;             // 6 per triangle (record version 6), or none
        bool transformed;                  // record version 7: made as the loader makes meshes
                                           // (through meshObject_t::transform), for its orco
    };
    std::vector<Obj> objs;
};

static void rd(FILE *f, void *p, size_t n) {
    if (n && fread(p, 1, n, f) != n) die("short read");
}

static void load_scene(const char *path, SceneFile &s) {
    FILE *f = fopen(path, "rb");
    if (!f) die("cannot open scene");
    char magic[4];
    rd(f, magic, 4);
    if (memcmp(magic, "YRS1", 4)) die("bad scene magic");
    uint32_t hdr[4];
    rd(f, hdr, 16);
    rd(f, &s.cam, sizeof(s.cam));
    // render parameters before record version 3 end at exposure (gamma then 1)
    memset(&s.rp, 0, sizeof(s.rp));
    s.rp.gamma = 1.f;
    rd(f, &s.rp, hdr[3] >= 3 ? sizeof(s.rp) : offsetof(yr_render_params, exposure));
    s.shaders.resize(hdr[1]);
    memset(s.shaders.data(), 0, sizeof(yr_shader_desc) * hdr[1]);
    // shader records before version 2 end at mod_mode, before version 5 at mod_specular
    const size_t shsize = hdr[3] >= 5   ? sizeof(yr_shader_desc)
                          : hdr[3] >= 2 ? offsetof(yr_shader_desc, mod_specular)
                                        : offsetof(yr_shader_desc, mod_mode);
    for (uint32_t i = 0; i < hdr[1]; i++) rd(f, &s.shaders[i], shsize);
    s.lights.resize(hdr[2]);
    if (hdr[2]) rd(f, &s.lights[0], sizeof(yr_light_desc) * hdr[2]);
    s.objs.resize(hdr[0]);
    for (uint32_t i = 0; i < hdr[0]; i++) {
        uint32_t oh[4];
        rd(f, oh, 16);
        SceneFile::Obj &o = s.objs[i];
        o.smooth = 0.f;
        if (hdr[3] >= 1) rd(f, &o.smooth, 4);  // record version 1: smoothing angle
        o.inst = -1;
        if (hdr[3] >= 4) rd(f, &o.inst, 4);    // record version 4: reference index (+ matrix)
        if (o.inst >= 0) {
            rd(f, o.M, 64);
            int32_t has_inv = 0;
            float inv[16];
            rd(f, &has_inv, 4);  // a given M^-1 is the library's input; the reference computes its own
            if (has_inv) rd(f, inv, 64);
            o.nv = o.nt = 0;
            o.shader = oh[2];
            o.cast = oh[3];
            if (hdr[3] >= 6) {  // record version 6: texture coordinates flag (none on a reference)
                int32_t has_uv = 0;
                rd(f, &has_uv, 4);
            }
            o.transformed = false;
            if (hdr[3] >= 7) {  // record version 7: orco matrix flag (none on a reference)
                int32_t has_orco = 0;
                rd(f, &has_orco, 4);
                if (has_orco) die("orco matrix on a reference");
            }
            continue;
        }
        o.nv = oh[0];
        o.nt = oh[1];
        o.shader = oh[2];
        o.cast = oh[3];
        o.v.resize(3 * o.nv);
        o.t.resize(3 * o.nt);
        rd(f, &o.v[0], 4 * o.v.size());
        rd(f, &o.t[0], 4 * o.t.size());
        if (o.shader == YR_PER_TRIANGLE) {
            o.tri_shader.resize(o.nt);
            rd(f, &o.tri_shader[0], 4 * o.nt);
        }
        if (hdr[3] >= 6) {  // record version 6: texture coordinates, 6 per triangle
            int32_t has_uv = 0;
            rd(f, &has_uv, 4);
            if (has_uv) {
                o.uv.resize(6 * (size_t)o.nt);
                rd(f, &o.uv[0], 4 * o.uv.size());
            }
        }
        // record version 7: a flag and the orco matrix, the library's input;
        // the reference makes that mesh through meshObject_t::transform and
        // computes its own
        o.transformed = false;
        if (hdr[3] >= 7) {
            int32_t has_orco = 0;
            rd(f, &has_orco, 4);
            if (has_orco) {
                float om[16];
                rd(f, om, 64);
                o.transformed = true;
            }
        }
    }
    fclose(f);
}

// ------------------------------------------------------- reference objects
struct RefScene {
    scene_t *scene;
    camera_t *camera;
    std::vector<meshObject_t *> meshes;   // per object; NULL for references
    std::vector<object3d_t *> objs;       // per object
    std::vector<shader_t *> shaders;
    std::vector<texture_t *> textures;
    std::vector<light_t *> lights;
    std::map<const object3d_t *, int> objindex;
};

static point3d_t P3(const float *p) { return point3d_t(p[0], p[1], p[2]); }
static color_t C3(const float *p) { return color_t(p[0], p[1], p[2]); }

static const char *noise_name(uint32_t t) {
    static const char *n[10] = {"newperlin",  "stdperlin",  "blender",    "voronoi_f1",      "voronoi_f2",
                                "voronoi_f3", "voronoi_f4", "voronoi_f2f1", "voronoi_crackle", "cellnoise"};
    return t < 10 ? n[t] : "newperlin";
}

// the texture of a shader record, through the plugin's own constructors
static texture_t *make_texture(const yr_shader_desc &d) {
    const color_t c1 = C3(d.tex_color1), c2 = C3(d.tex_color2);
    static const char *shapes[3] = {"sin", "saw", "tri"};
    const char *shape = shapes[d.tex_shape < 3 ? d.tex_shape : 0];
    switch (d.tex_type) {
    case YR_TEX_MUSGRAVE_FBM:
    case YR_TEX_MUSGRAVE_MULTIFRACTAL:
    case YR_TEX_MUSGRAVE_HETEROTERRAIN:
    case YR_TEX_MUSGRAVE_HYBRIDMF:
    case YR_TEX_MUSGRAVE_RIDGEDMF: {
        static const char *mt[5] = {"fBm", "multifractal", "heteroterrain", "hybridmf", "ridgedmf"};
        const int k = d.tex_type == YR_TEX_MUSGRAVE_FBM ? 0 : (int)d.tex_type - YR_TEX_MUSGRAVE_MULTIFRACTAL + 1;
        return new textureMusgrave_t(c1, c2, d.tex_H, d.tex_lacunarity, d.tex_octaves, d.tex_offset, d.tex_gain,
                                     d.tex_size, d.tex_intensity, noise_name(d.tex_noise), mt[k]);
    }
    case YR_TEX_CLOUDS:
        return new textureClouds_t(d.tex_depth, d.tex_size, d.tex_hard != 0, c1, c2, noise_name(d.tex_noise),
                                   d.tex_variant == 1 ? "positive" : (d.tex_variant == 2 ? "negative" : ""));
    case YR_TEX_MARBLE:
        return new textureMarble_t(d.tex_depth, d.tex_size, c1, c2, d.tex_turbulence, d.tex_sharpness,
                                   d.tex_hard != 0, noise_name(d.tex_noise), shape);
    case YR_TEX_WOOD:
        return new textureWood_t(d.tex_depth, d.tex_size, c1, c2, d.tex_turbulence, d.tex_hard != 0,
                                 noise_name(d.tex_noise), d.tex_variant ? "rings" : "bands", shape);
    case YR_TEX_VORONOI: {
        static const char *dm[7] = {"real",           "squared",        "manhattan", "chebychev",
                                    "minkovsky_half", "minkovsky_four", "minkovsky"};
        return new textureVoronoi_t(c1, c2, (int)d.tex_shape, d.tex_weights[0], d.tex_weights[1], d.tex_weights[2],
                                    d.tex_weights[3], d.tex_mk_exponent, d.tex_size, d.tex_intensity,
                                    dm[d.tex_metric < 7 ? d.tex_metric : 0]);
    }
    case YR_TEX_DISTORTED_NOISE:
        return new textureDistortedNoise_t(c1, c2, d.tex_distort, d.tex_size, noise_name(d.tex_noise),
                                           noise_name(d.tex_noise2));
    case YR_TEX_GRADIENT: {
        static const char *gt[6] = {"linear", "quadratic", "cubic", "diagonal", "sphere", "halo"};
        return new textureGradient_t(c1, c2, gt[d.tex_shape < 6 ? d.tex_shape : 0], d.tex_variant != 0);
    }
    }
    die("bad texture type");
    return NULL;
}

static shader_t *make_shader(const yr_shader_desc &d, std::vector<texture_t *> &textures) {
    // genericShader_t::factory defaults (basicshaders.cc:217-262)
    genericShader_t *sh = new genericShader_t(C3(d.color), d.hard, (CFLOAT)1.0, color_t(0.0), color_t(0.0),
                                              C3(d.specular), color_t(0.0), color_t(0.0), NULL, 0.0, (CFLOAT)1.0,
                                              1.0, false, false, 0, 0, false, color_t(0.0));
    if (d.tex_type != YR_TEX_NONE) {
        texture_t *tex = make_texture(d);
        textures.push_back(tex);
        modulator_t modu(tex);
        modu.sizeX(d.mod_size[0]);
        modu.sizeY(d.mod_size[1]);
        modu.sizeZ(d.mod_size[2]);
        modu.ofsX(d.mod_ofs[0]);
        modu.ofsY(d.mod_ofs[1]);
        modu.ofsZ(d.mod_ofs[2]);
        static const char *modes[4] = {"mix", "mul", "add", "sub"};
        modu.string2modetype(modes[d.mod_mode < 4 ? d.mod_mode : 0]);
        modu.color(d.mod_color);
        modu.specular(d.mod_specular);
        modu.hard(d.mod_hard);
        modu.transmision(0);
        modu.reflection(0);
        modu.displace(0);
        modu.string2maptype("flat");
        static const char *texco[6] = {"global", "orco", "normal", "window", "reflect", "uv"};
        modu.string2texcotype(texco[(d.tex_map & 0xffu) < 6 ? (d.tex_map & 0xffu) : 0]);
        modu.string2cliptype("extend");
        std::string proj[3];
        for (int k = 0; k < 3; k++) {
            const uint32_t pc = (d.tex_map >> (8 * (k + 1))) & 0xffu;
            proj[k] = pc == YR_PROJ_DEFAULT ? std::string(1, "xyz"[k]) : std::string(1, "nxyzn"[pc < 5 ? pc : 4]);
        }
        modu.string2texprojection(proj[0], proj[1], proj[2]);
        sh->addModulator(modu);
    }
    return sh;
}

static light_t *make_light(const yr_light_desc &d) {
    switch (d.type) {
    case YR_LIGHT_POINT:
        return new pointLight_t(P3(d.p[0]), C3(d.color), d.power, d.cast_shadows != 0);
    case YR_LIGHT_AREA:
        return new areaLight_t(P3(d.p[0]), P3(d.p[1]), P3(d.p[2]), P3(d.p[3]), d.samples, C3(d.color), d.power,
                               d.psamples, false);
    case YR_LIGHT_HEMI:
        return new hemiLight_t(d.samples, C3(d.color), d.power, d.maxdist, false, true);
    case YR_LIGHT_PATH:
        // use_QMC, no cache; adaptive repetitions at the record's threshold
        // (off, as a huge threshold, when it is not above 0)
        return new pathLight_t(d.samples, d.power, d.depth, 0, true, false, 1.0, d.threshold > 0 ? d.threshold : 1e9f);
    }
    die("bad light type");
    return NULL;
}

// the "constant" background plugin (constBackground_t, sunsky.h:12-21): a
// fixed colour for every direction
class constBg_t : public background_t {
  public:
    constBg_t(const color_t &c) : color(c) {}
    virtual color_t operator()(const vector3d_t &dir, renderState_t &state, bool filtered = false) const {
        return color;
    }
    color_t color;
};

// `scene`: the scene object to fill (a derived scene class); NULL = a new
// plain scene_t
static void build_ref(const SceneFile &s, RefScene &r, bool with_lights = true, scene_t *scene = NULL) {
    r.scene = scene ? scene : scene_t::factory();
    for (size_t i = 0; i < s.shaders.size(); i++) r.shaders.push_back(make_shader(s.shaders[i], r.textures));
    for (size_t i = 0; i < s.objs.size(); i++) {
        const SceneFile::Obj &o = s.objs[i];
        if (o.inst >= 0) {  // made below, once the meshes exist
            r.meshes.push_back(NULL);
            r.objs.push_back(NULL);
            continue;
        }
        std::vector<point3d_t> ver(o.nv);
        for (uint32_t k = 0; k < o.nv; k++) ver[k] = P3(&o.v[3 * k]);
        std::vector<triangle_t> ts(o.nt);
        for (uint32_t k = 0; k < o.nt; k++)
            ts[k] = triangle_t(&ver[o.t[3 * k]], &ver[o.t[3 * k + 1]], &ver[o.t[3 * k + 2]]);
        if (o.shader == YR_PER_TRIANGLE)  // triangle_t::setShader, used by getSurface
            for (uint32_t k = 0; k < o.nt; k++) ts[k].setShader(r.shaders.at(o.tri_shader[k]));
        std::vector<vector3d_t> nor;
        std::vector<GFLOAT> fuv(o.uv.begin(), o.uv.end());
        std::vector<CFLOAT> fvcol;
        if (!fuv.empty())  // each triangle's six coordinates, as the loader sets them
            for (uint32_t k = 0; k < o.nt; k++) ts[k].setUV(fuv.begin() + 6 * (size_t)k);
        // a "transformed" mesh is made as the loader and yafrayInterface_t
        // make every mesh: with the current transform, here the identity
        // (interface_impl.cc:242, render.cc:757), which sets its orco matrix
        meshObject_t *m = o.transformed ? meshObject_t::factory(false, matrix4x4_t(1), ver, nor, ts, fuv, fvcol)
                                        : meshObject_t::factory(ver, nor, ts, fuv, fvcol);
        m->setShader(r.shaders.at(o.shader == YR_PER_TRIANGLE ? o.tri_shader[0] : o.shader));
        m->castShadows(o.cast != 0);
        if (o.smooth >= 1.f) m->autoSmooth(o.smooth);  // as the loader does (render.cc:764)
        m->tangentsFromUV();                           // render.cc:765 (nothing without uv or orco)
        r.meshes.push_back(m);
        r.objs.push_back(m);
        r.objindex[m] = (int)i;
    }
    // references (the loader's objects with an "original", render.cc:672-680)
    for (size_t i = 0; i < s.objs.size(); i++) {
        const SceneFile::Obj &o = s.objs[i];
        if (o.inst < 0) continue;
        if ((size_t)o.inst >= r.meshes.size() || !r.meshes[o.inst]) die("reference to a missing mesh");
        matrix4x4_t M(1);
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) M[a][b] = o.M[4 * a + b];
        referenceObject_t *ro = referenceObject_t::factory(M, r.meshes[o.inst]);
        r.objs[i] = ro;
        r.objindex[ro] = (int)i;
    }
    for (size_t i = 0; i < r.objs.size(); i++) r.scene->addObject(r.objs[i]);
    const yr_camera_desc &c = s.cam;
    r.camera = new camera_t(P3(c.pos), P3(c.look), P3(c.up), c.resx, c.resy, c.aspect, c.focal, 0, 0, false,
                            camera_t::CM_PERSPECTIVE, camera_t::BK_DISK1, camera_t::BB_NONE, 0);
    r.scene->setCamera(r.camera);
    r.scene->setBias(s.rp.self_bias);
    r.scene->setMaxRayDepth(s.rp.raydepth);
    r.scene->tonemap((s.rp.flags & YR_RENDER_TONEMAP) != 0);
    r.scene->clampRGB((s.rp.flags & YR_RENDER_CLAMP_RGB) != 0);
    r.scene->alphaPremultiply((s.rp.flags & YR_RENDER_ALPHA_PREMULTIPLY) != 0);
    r.scene->setExposure(s.rp.exposure);
    r.scene->setGamma(s.rp.gamma);
    if (s.rp.background[0] != 0.f || s.rp.background[1] != 0.f || s.rp.background[2] != 0.f)
        r.scene->setBackground(new constBg_t(C3(s.rp.background)));
    r.scene->alphaMaskBackground(false);
    r.scene->setFog(0, color_t(0.0));
    if (with_lights)
        for (size_t i = 0; i < s.lights.size(); i++) {
            light_t *l = make_light(s.lights[i]);
            r.lights.push_back(l);
            r.scene->addLight(l);
        }
}

static void wr(FILE *f, const void *p, size_t n) {
    if (n && fwrite(p, 1, n, f) != n) die("short write");
}

// ------------------------------------------------------------------- tree
static void cmd_tree(const SceneFile &s, const char *out) {
    RefScene r;
    build_ref(s, r, false);
    FILE *f = fopen(out, "wb");
    if (!f) die("cannot open output");
    uint32_t n = 0;  // trees of the meshes (references share their original's)
    for (size_t i = 0; i < r.meshes.size(); i++) n += r.meshes[i] ? 1 : 0;
    wr(f, &n, 4);
    for (size_t i = 0; i < r.meshes.size(); i++) {
        meshObject_t *m = r.meshes[i];
        if (!m) continue;
        kdTree_t *t = m->n_tree;
        const triangle_t *base = &m->triangles[0];
        std::vector<uint32_t> nodes, prims;
        for (uint32_t k = 0; k < t->nextFreeNode; k++) {
            const kdTreeNode &nd = t->nodes[k];
            uint32_t word = 0;
            if (nd.IsLeaf()) {
                int np = nd.nPrimitives();
                if (np == 1) word = (uint32_t)(nd.onePrimitive - base);
                else if (np > 1) {
                    word = (uint32_t)prims.size();
                    for (int q = 0; q < np; q++) prims.push_back((uint32_t)(nd.primitives[q] - base));
                }
            } else {
                float sp = nd.division;
                memcpy(&word, &sp, 4);
            }
            nodes.push_back(word);
            nodes.push_back(nd.flags);
        }
        uint32_t hdr[2] = {t->nextFreeNode, (uint32_t)prims.size()};
        wr(f, hdr, 8);
        float tb[6] = {t->treeBound.a.x, t->treeBound.a.y, t->treeBound.a.z,
                       t->treeBound.g.x, t->treeBound.g.y, t->treeBound.g.z};
        wr(f, tb, 24);
        int32_t ip[2] = {t->maxDepth, t->maxLeafSize};
        wr(f, ip, 8);
        float fp[2] = {t->costRatio, t->eBonus};
        wr(f, fp, 8);
        bound_t ob = m->getBound();
        float obf[6] = {ob.a.x, ob.a.y, ob.a.z, ob.g.x, ob.g.y, ob.g.z};
        wr(f, obf, 24);
        wr(f, &nodes[0], 4 * nodes.size());
        if (!prims.empty()) wr(f, &prims[0], 4 * prims.size());
    }
    // object tree, depth-first preorder, left before right
    geomeTree_t<object3d_t> *root = buildObjectTree(r.scene->obj_list);
    std::vector<const geomeTree_t<object3d_t> *> stack, order;
    stack.push_back(root);
    while (!stack.empty()) {
        const geomeTree_t<object3d_t> *nd = stack.back();
        stack.pop_back();
        order.push_back(nd);
        if (!nd->isLeaf()) {
            stack.push_back(nd->goRight());
            stack.push_back(nd->goLeft());
        }
    }
    std::map<const geomeTree_t<object3d_t> *, int> idx;
    for (size_t i = 0; i < order.size(); i++) idx[order[i]] = (int)i;
    uint32_t nn = (uint32_t)order.size();
    wr(f, &nn, 4);
    for (size_t i = 0; i < order.size(); i++) {
        const geomeTree_t<object3d_t> *nd = order[i];
        const bound_t &b = nd->getBound();
        float bb[6] = {b.a.x, b.a.y, b.a.z, b.g.x, b.g.y, b.g.z};
        int32_t lr[2];
        if (nd->isLeaf()) {
            lr[0] = -1;
            lr[1] = r.objindex[nd->getElement()];
        } else {
            lr[0] = idx[nd->goLeft()];
            lr[1] = idx[nd->goRight()];
        }
        wr(f, bb, 24);
        wr(f, lr, 8);
    }
    fclose(f);
}

// ------------------------------------------------------------------- rays
// Ray record: u32 mode, u32 object, f32 from[3], f32 dir[3], f32 dist, f32 l[3]
//   mode 0: kdTree_t::Intersect on `object`  -> u32 hit, u32 tri, f32 Z
//   mode 1: kdTree_t::IntersectS on `object` -> u32 hit, u32 tri, f32 0
//   mode 2: scene_t::firstHit(from, dir, shadow=false) -> u32 hit, u32 obj, u32 tri, f32 Z
//   mode 3: scene_t::isShadowed(sp{P=from, object}, l) -> u32 occluded
//   mode 4: scene_t::firstHit(from, dir, shadow=true)  (as mode 2)
struct RayRec {
    uint32_t mode, object;
    float from[3], dir[3], dist, l[3];
};

static void cmd_rays(const SceneFile &s, const char *rays_path, const char *out) {
    RefScene r;
    build_ref(s, r, false);
    r.scene->BTree = buildObjectTree(r.scene->obj_list);
    FILE *fi = fopen(rays_path, "rb");
    if (!fi) die("cannot open rays");
    uint32_t n;
    rd(fi, &n, 4);
    std::vector<RayRec> rays(n);
    if (n) rd(fi, &rays[0], sizeof(RayRec) * n);
    fclose(fi);
    FILE *f = fopen(out, "wb");
    if (!f) die("cannot open output");
    renderState_t state;
    for (uint32_t i = 0; i < n; i++) {
        const RayRec &q = rays[i];
        point3d_t from = P3(q.from);
        vector3d_t dir(q.dir[0], q.dir[1], q.dir[2]);
        uint32_t o[4] = {0, 0xffffffffu, 0xffffffffu, 0};
        if (q.mode == 0 || q.mode == 1) {
            meshObject_t *m = r.meshes.at(q.object);
            const triangle_t *base = &m->triangles[0];
            triangle_t *hitt = NULL;
            PFLOAT dis = q.dist;
            if (dis < 0) dis = std::numeric_limits<PFLOAT>::infinity();
            PFLOAT Z = dis;
            bool h = q.mode == 0 ? m->n_tree->Intersect(from, dir, dis, &hitt, Z)
                                 : m->n_tree->IntersectS(from, dir, dis, &hitt);
            o[0] = h;
            if (h && hitt) o[2] = (uint32_t)(hitt - base);
            float zf = q.mode == 0 && h ? Z : 0.f;
            memcpy(&o[3], &zf, 4);
            o[1] = q.object;
        } else if (q.mode == 2 || q.mode == 4) {
            surfacePoint_t sp;
            bool h = r.scene->firstHit(state, sp, from, dir, q.mode == 4);
            o[0] = h;
            if (h) {
                o[1] = r.objindex[sp.getObject()];
                meshObject_t *m = r.meshes.at(o[1]);
                if (!m) m = r.meshes.at(s.objs[o[1]].inst);  // a reference: the original's triangle
                o[2] = (uint32_t)((const triangle_t *)sp.getOrigin() - &m->triangles[0]);
                float zf = sp.Z();
                memcpy(&o[3], &zf, 4);
            }
        } else if (q.mode == 3) {
            surfacePoint_t sp(r.objs.at(q.object), from, from, vector3d_t(0, 0, 1), vector3d_t(0, 0, 1), 0, 0,
                              color_t(0.0), 0);
            o[0] = r.scene->isShadowed(state, sp, P3(q.l));
        }
        wr(f, o, 16);
    }
    fclose(f);
}

// -------------------------------------------------------------- references
// Each reference's M^-1 as referenceObject_t computes it (back,
// reference.cc:13-14): u32 count, then per reference u32 object index and
// 16 floats.
static void cmd_instmat(const SceneFile &s, const char *out) {
    RefScene r;
    build_ref(s, r, false);
    std::vector<uint32_t> idx;
    for (size_t i = 0; i < r.objs.size(); i++)
        if (!r.meshes[i]) idx.push_back((uint32_t)i);
    FILE *f = fopen(out, "wb");
    if (!f) die("cannot open output");
    uint32_t n = (uint32_t)idx.size();
    wr(f, &n, 4);
    for (size_t k = 0; k < idx.size(); k++) {
        const referenceObject_t *ro = (const referenceObject_t *)r.objs[idx[k]];
        wr(f, &idx[k], 4);
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                const float v = ro->back[a][b];
                wr(f, &v, 4);
            }
    }
    fclose(f);
}

// Each transformed mesh's orco matrix as meshObject_t::transform computes
// it (backOrco, mesh.cc:452-481): u32 count, then per mesh u32 object index
// and 16 floats.
static void cmd_orcomat(const SceneFile &s, const char *out) {
    RefScene r;
    build_ref(s, r, false);
    std::vector<uint32_t> idx;
    for (size_t i = 0; i < s.objs.size(); i++)
        if (s.objs[i].inst < 0 && s.objs[i].transformed) idx.push_back((uint32_t)i);
    FILE *f = fopen(out, "wb");
    if (!f) die("cannot open output");
    uint32_t n = (uint32_t)idx.size();
    wr(f, &n, 4);
    for (size_t k = 0; k < idx.size(); k++) {
        const meshObject_t *m = r.meshes[idx[k]];
        wr(f, &idx[k], 4);
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                const float v = m->backOrco[a][b];
                wr(f, &v, 4);
            }
    }
    fclose(f);
}

// ----------------------------------------------------------------- camera
static void cmd_camera(const SceneFile &s, const char *out) {
    RefScene r;
    build_ref(s, r, false);
    FILE *f = fopen(out, "wb");
    for (int i = 0; i < s.cam.resy; i++)
        for (int j = 0; j < s.cam.resx; j++) {
            PFLOAT wt;
            vector3d_t d = r.camera->shootRay((PFLOAT)j + 0.5f, (PFLOAT)i + 0.5f, wt);
            float v[3] = {d.x, d.y, d.z};
            wr(f, v, 12);
        }
    fclose(f);
}

// ----------------------------------------------------------------- render
class floatSink_t : public colorOutput_t {
  public:
    floatSink_t(int w, int h) : W(w), H(h), img(4 * (size_t)w * h, 0.f) {}
    virtual bool putPixel(int x, int y, const color_t &c, CFLOAT alpha, PFLOAT depth) {
        float *p = &img[4 * ((size_t)y * W + x)];
        p[0] = c.getR();
        p[1] = c.getG();
        p[2] = c.getB();
        p[3] = alpha;
        return true;
    }
    virtual void flush() {}
    int W, H;
    std::vector<float> img;
};

static void cmd_render(const SceneFile &s, const char *out, int threads, const int *crop, int reps) {
    RefScene r;
    build_ref(s, r, true);
    scene_t *sc = r.scene;
    threadedscene_t *tsc = NULL;
    if (threads > 1) {
        // threadedscene_t holds its own copy of the scene state; rebuild through it
        tsc = (threadedscene_t *)threadedscene_t::factory();
        tsc->setCPUs(threads);
        for (size_t i = 0; i < r.objs.size(); i++) tsc->addObject(r.objs[i]);
        for (size_t i = 0; i < r.lights.size(); i++) tsc->addLight(r.lights[i]);
        tsc->setCamera(r.camera);
        tsc->setBias(s.rp.self_bias);
        tsc->setMaxRayDepth(s.rp.raydepth);
        tsc->tonemap((s.rp.flags & YR_RENDER_TONEMAP) != 0);
        tsc->clampRGB((s.rp.flags & YR_RENDER_CLAMP_RGB) != 0);
        tsc->alphaPremultiply((s.rp.flags & YR_RENDER_ALPHA_PREMULTIPLY) != 0);
        tsc->setExposure(s.rp.exposure);
        tsc->setGamma(s.rp.gamma);
        tsc->setBackground(r.scene->background);
        tsc->alphaMaskBackground(false);
        tsc->setFog(0, color_t(0.0));
        sc = tsc;
    }
    const uint32_t spp = s.rp.spp ? s.rp.spp : 1;
    // every pixel resampled: AA_threshold 0 (renderblock.cc:22-66 uses >=)
    sc->setAASamples(spp > 1 ? 1 : 0, spp > 1 ? (int)spp - 1 : 1, s.rp.aa_pixelwidth, 0.0, false);
    long region_px = (long)s.cam.resx * s.cam.resy;
    if (crop) {
        // screen-space region in [-1,1] (scene.cc:745-747), from pixel bounds
        // (pixel centres, so a pixel is inside exactly when x0 <= x < x1)
        PFLOAT rx = (PFLOAT)s.cam.resx, ry = (PFLOAT)s.cam.resy;
        sc->setRegion(2.0 * crop[0] / rx - 1.0, 2.0 * crop[1] / rx - 1.0, 1.0 - 2.0 * crop[3] / ry,
                      1.0 - 2.0 * crop[2] / ry);
        region_px = (long)(crop[1] - crop[0]) * (crop[3] - crop[2]);
    }
    floatSink_t sink(s.cam.resx, s.cam.resy);
    // repeated renders share one scene (and one kd-tree build); each prints a line
    for (int rep = 0; rep < reps; rep++) {
        counts_reset();
        double t0 = now_s();
        sc->render(sink);
        double t1 = now_s();
        long nsh = 0, nbo = 0;
        counts_sum(nsh, nbo);
        printf("{\"render_s\": %.6f, \"threads\": %d, \"primary\": %ld, \"shadow\": %ld, \"bounce\": %ld}\n",
               t1 - t0, threads, region_px * (long)spp, nsh, nbo);
        fflush(stdout);
    }
    FILE *f = fopen(out, "wb");
    wr(f, &sink.img[0], 4 * sink.img.size());
    fclose(f);
}

// ---------------------------------------------------------- render blocks
// CPU timing on a stratified sample of the frame.  threadedscene_t renders
// a frame as 64x64 blocks (blockSpliter_t, renderblock.cc:71-101: each
// block's area carries a one-pixel border on its inner sides) that worker
// threads take one at a time and pass to the scene's own per-area render,
// scene_t::render(renderArea_t&) (threadedscene.cc:77-95).  This command
// runs that worker loop over a chosen list of those blocks instead of all of
// them, so that a sample spread over the whole frame can be timed on every
// host core (threadedscene_t refuses more threads than blocks of its region).
class blockScene_t : public scene_t {
  public:
    blockScene_t() {}
    // what scene_t::render(colorOutput_t&) and threadedscene_t::render do
    // before the first block (scene.cc:555; threadedscene.cc:110-116)
    void prepare() {
        BTree = buildObjectTree(obj_list);
        setupLights();
    }
    void release() {
        delete BTree;
        BTree = NULL;
    }
};

struct BlockRun {
    const blockScene_t *scene;
    std::vector<renderArea_t> *areas;
    colorOutput_t *out;
    long next;
};

static void *block_worker(void *arg) {
    BlockRun *R = (BlockRun *)arg;
    for (;;) {
        const long k = __sync_fetch_and_add(&R->next, 1L);
        if (k >= (long)R->areas->size()) break;
        renderArea_t &a = (*R->areas)[k];
        R->scene->render(a);
        a.out(*R->out);  // blocks write disjoint real regions
    }
    return NULL;
}

// blocks: "bx.by,bx.by,..." in 64-pixel block units
static void cmd_render_blocks(const SceneFile &s, const char *out, int threads, const char *blocks, int reps) {
    RefScene r;
    blockScene_t *bs = new blockScene_t();
    build_ref(s, r, true, bs);
    const uint32_t spp = s.rp.spp ? s.rp.spp : 1;
    bs->setAASamples(spp > 1 ? 1 : 0, spp > 1 ? (int)spp - 1 : 1, s.rp.aa_pixelwidth, 0.0, false);
    const int W = s.cam.resx, H = s.cam.resy, B = 64;
    std::vector<renderArea_t> areas;
    long traced_px = 0;
    for (const char *q = blocks; *q;) {
        int bx = 0, by = 0, used = 0;
        if (sscanf(q, "%d.%d%n", &bx, &by, &used) != 2) die("bad block list");
        q += used;
        if (*q == ',') q++;
        const int rx = bx * B, ry = by * B;
        if (rx < 0 || ry < 0 || rx >= W || ry >= H) die("block outside the frame");
        // blockSpliter_t's area of this block (renderblock.cc:84-97)
        int x = rx, y = ry, w = std::min(B, W - rx), h = std::min(B, H - ry);
        const int rw = w, rh = h;
        if (x > 0) { x--; w++; }
        if (y > 0) { y--; h++; }
        if (x + w < W - 1) w++;
        if (y + h < H - 1) h++;
        renderArea_t a;
        a.set(x, y, w, h);
        a.setReal(rx, ry, rw, rh);
        areas.push_back(a);
        traced_px += (long)w * h;
    }
    if (threads < 1) threads = 1;
    floatSink_t sink(W, H);
    bs->prepare();
    for (int rep = 0; rep < reps; rep++) {
        counts_reset();
        BlockRun R = {bs, &areas, &sink, 0};
        std::vector<pthread_t> th(threads);
        double t0 = now_s();
        for (int i = 0; i < threads; i++) pthread_create(&th[i], NULL, block_worker, &R);
        for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
        double t1 = now_s();
        long nsh = 0, nbo = 0;
        counts_sum(nsh, nbo);
        printf("{\"render_s\": %.6f, \"threads\": %d, \"blocks\": %d, \"primary\": %ld, \"shadow\": %ld, "
               "\"bounce\": %ld}\n",
               t1 - t0, threads, (int)areas.size(), traced_px * (long)spp, nsh, nbo);
        fflush(stdout);
    }
    bs->release();
    FILE *f = fopen(out, "wb");
    wr(f, &sink.img[0], 4 * sink.img.size());
    fclose(f);
}

#ifdef YR_HARNESS_CUDASCENE
// ------------------------------------------------------------ cudarender
// The drop-in: the same scene built from the reference's own objects
// (meshObject_t, genericShader_t, pointLight_t, camera_t) into a
// cudascene_t, rendered by cudascene_t::render - the library, through
// yr_render - into the float sink.  One JSON line: the library's status
// and the render time.
// a float sink that asks the render to stop after `limit` pixels
class stoppingSink_t : public floatSink_t {
  public:
    stoppingSink_t(int w, int h, long lim) : floatSink_t(w, h), limit(lim), taken(0) {}
    virtual bool putPixel(int x, int y, const color_t &c, CFLOAT alpha, PFLOAT depth) {
        if (limit >= 0 && taken >= limit) return false;
        taken++;
        return floatSink_t::putPixel(x, y, c, alpha, depth);
    }
    long limit, taken;
};

static void cmd_cudarender(const SceneFile &s, const char *out, const int *crop, long stop_after) {
    RefScene r;
    cudascene_t *cs = new cudascene_t(0);
    build_ref(s, r, true, cs);
    const uint32_t spp = s.rp.spp ? s.rp.spp : 1;
    cs->setAASamples(spp > 1 ? 1 : 0, spp > 1 ? (int)spp - 1 : 1, s.rp.aa_pixelwidth, 0.0, false);
    if (crop) {
        PFLOAT rx = (PFLOAT)s.cam.resx, ry = (PFLOAT)s.cam.resy;
        cs->setRegion(2.0 * crop[0] / rx - 1.0, 2.0 * crop[1] / rx - 1.0, 1.0 - 2.0 * crop[3] / ry,
                      1.0 - 2.0 * crop[2] / ry);
    }
    stoppingSink_t sink(s.cam.resx, s.cam.resy, stop_after);
    double t0 = now_s();
    cs->render(sink);
    double t1 = now_s();
    printf("{\"status\": %d, \"render_s\": %.6f, \"pixels\": %ld}\n", (int)cs->lastStatus(), t1 - t0,
           sink.taken);
    fflush(stdout);
    FILE *f = fopen(out, "wb");
    wr(f, &sink.img[0], 4 * sink.img.size());
    fclose(f);
    delete cs;
}
#endif

#ifdef YR_HARNESS_CUDASCENE
// ------------------------------------------------------------------ iface
// The host API: the scene handed to a yafrayInterface_t call by call, as a
// front end does (shaders with their texture and modulator parameter maps,
// meshes through addObject_trimesh with the identity transform,
// references through transformPush + addObject_reference, lights and the
// camera as parameter maps, a "constant" background), then
// render(params, sink).  ARM "ref" is the reference's interfaceImpl_t
// (threadedscene_t, the CPU); "cuda" is cudaInterface_t (the library).
// The plugins are registered by hand, as their registerPlugin functions
// and bbreg.cc do.  One JSON line: the status (cuda arm) and the time.
extern "C" {
void registerPlugin_pointlight(renderEnvironment_t &);
void registerPlugin_arealight(renderEnvironment_t &);
void registerPlugin_hemilight(renderEnvironment_t &);
void registerPlugin_pathlight(renderEnvironment_t &);
void registerPlugin_basicshaders(renderEnvironment_t &);
void registerPlugin_sunsky(renderEnvironment_t &);
}

static void iface_register(yafrayInterface_t &y) {
    registerPlugin_pointlight(y);
    registerPlugin_arealight(y);
    registerPlugin_hemilight(y);
    registerPlugin_pathlight(y);
    registerPlugin_basicshaders(y);
    registerPlugin_sunsky(y);
    y.registerFactory("clouds", textureClouds_t::factory);
    y.registerFactory("marble", textureMarble_t::factory);
    y.registerFactory("wood", textureWood_t::factory);
    y.registerFactory("voronoi", textureVoronoi_t::factory);
    y.registerFactory("musgrave", textureMusgrave_t::factory);
    y.registerFactory("distorted_noise", textureDistortedNoise_t::factory);
    y.registerFactory("gradient", textureGradient_t::factory);
}

static parameter_t P_col(const float *c) { return parameter_t(c[0], c[1], c[2]); }
static parameter_t P_pt(const float *c) { return parameter_t(point3d_t(c[0], c[1], c[2])); }
static parameter_t P_on(bool b) { return parameter_t(std::string(b ? "on" : "off")); }
static parameter_t P_str(const char *v) { return parameter_t(std::string(v)); }

// yr_shader_desc -> the generic shader's, its texture's and its
// modulator's parameter maps (the names of basicshaders.cc / basictex.cc)
static void iface_shader(yafrayInterface_t &y, const yr_shader_desc &d, int k) {
    char name[32], tname[32];
    snprintf(name, sizeof(name), "sh%04d", k);
    snprintf(tname, sizeof(tname), "tex%04d", k);
    std::list<paramMap_t> mods;
    if (d.tex_type != YR_TEX_NONE) {
        paramMap_t t;
        t["name"] = P_str(tname);
        t["color1"] = P_col(d.tex_color1);
        t["color2"] = P_col(d.tex_color2);
        static const char *noise[10] = {"newperlin",  "stdperlin",  "blender",      "voronoi_f1",      "voronoi_f2",
                                        "voronoi_f3", "voronoi_f4", "voronoi_f2f1", "voronoi_crackle", "cellnoise"};
        static const char *shapes[3] = {"sin", "saw", "tri"};
        const char *nt = noise[d.tex_noise < 10 ? d.tex_noise : 0];
        switch (d.tex_type) {
        case YR_TEX_MUSGRAVE_FBM:
        case YR_TEX_MUSGRAVE_MULTIFRACTAL:
        case YR_TEX_MUSGRAVE_HETEROTERRAIN:
        case YR_TEX_MUSGRAVE_HYBRIDMF:
        case YR_TEX_MUSGRAVE_RIDGEDMF:
            // the musgrave factory reads its kind from "type", which through
            // addTexture is the texture type itself ("musgrave"): every
            // musgrave texture made this way is fBm (basictex.cc:694,
            // interface_impl.cc:133)
            t["type"] = P_str("musgrave");
            t["noise_type"] = P_str(nt);
            t["H"] = parameter_t(d.tex_H);
            t["lacunarity"] = parameter_t(d.tex_lacunarity);
            t["octaves"] = parameter_t(d.tex_octaves);
            t["offset"] = parameter_t(d.tex_offset);
            t["gain"] = parameter_t(d.tex_gain);
            t["size"] = parameter_t(d.tex_size);
            t["intensity"] = parameter_t(d.tex_intensity);
            break;
        case YR_TEX_CLOUDS:
            t["type"] = P_str("clouds");
            t["noise_type"] = P_str(nt);
            t["depth"] = parameter_t((float)d.tex_depth);
            t["size"] = parameter_t(d.tex_size);
            t["hard"] = P_on(d.tex_hard != 0);
            t["bias"] = P_str(d.tex_variant == 1 ? "positive" : (d.tex_variant == 2 ? "negative" : ""));
            break;
        case YR_TEX_MARBLE:
        case YR_TEX_WOOD:
            t["type"] = P_str(d.tex_type == YR_TEX_MARBLE ? "marble" : "wood");
            t["noise_type"] = P_str(nt);
            t["depth"] = parameter_t((float)d.tex_depth);
            t["turbulence"] = parameter_t(d.tex_turbulence);
            t["size"] = parameter_t(d.tex_size);
            t["hard"] = P_on(d.tex_hard != 0);
            t["shape"] = P_str(shapes[d.tex_shape < 3 ? d.tex_shape : 0]);
            if (d.tex_type == YR_TEX_MARBLE) t["sharpness"] = parameter_t(d.tex_sharpness);
            else t["wood_type"] = P_str(d.tex_variant ? "rings" : "bands");
            break;
        case YR_TEX_VORONOI: {
            static const char *ct[4] = {"int", "col1", "col2", "col3"};
            static const char *dm[7] = {"real",           "squared",        "manhattan", "chebychev",
                                        "minkovsky_half", "minkovsky_four", "minkovsky"};
            t["type"] = P_str("voronoi");
            t["color_type"] = P_str(ct[d.tex_shape < 4 ? d.tex_shape : 0]);
            t["weight1"] = parameter_t(d.tex_weights[0]);
            t["weight2"] = parameter_t(d.tex_weights[1]);
            t["weight3"] = parameter_t(d.tex_weights[2]);
            t["weight4"] = parameter_t(d.tex_weights[3]);
            t["mk_exponent"] = parameter_t(d.tex_mk_exponent);
            t["intensity"] = parameter_t(d.tex_intensity);
            t["size"] = parameter_t(d.tex_size);
            t["distance_metric"] = P_str(dm[d.tex_metric < 7 ? d.tex_metric : 0]);
            break;
        }
        case YR_TEX_DISTORTED_NOISE:
            t["type"] = P_str("distorted_noise");
            t["noise_type1"] = P_str(nt);
            t["noise_type2"] = P_str(noise[d.tex_noise2 < 10 ? d.tex_noise2 : 0]);
            t["distort"] = parameter_t(d.tex_distort);
            t["size"] = parameter_t(d.tex_size);
            break;
        case YR_TEX_GRADIENT: {
            static const char *gt[6] = {"linear", "quadratic", "cubic", "diagonal", "sphere", "halo"};
            t["type"] = P_str("gradient");
            t["gradient_type"] = P_str(gt[d.tex_shape < 6 ? d.tex_shape : 0]);
            t["flip_xy"] = P_on(d.tex_variant != 0);
            break;
        }
        default:
            die("iface: texture type without a parameter map here");
        }
        y.addTexture(t);
        paramMap_t m;
        static const char *modes[4] = {"mix", "mul", "add", "sub"};
        static const char *texco[6] = {"global", "orco", "normal", "window", "reflect", "uv"};
        m["texname"] = P_str(tname);
        m["mode"] = P_str(modes[d.mod_mode < 4 ? d.mod_mode : 0]);
        m["color"] = parameter_t(d.mod_color);
        m["specular"] = parameter_t(d.mod_specular);
        m["hard"] = parameter_t(d.mod_hard);
        m["sizex"] = parameter_t(d.mod_size[0]);
        m["sizey"] = parameter_t(d.mod_size[1]);
        m["sizez"] = parameter_t(d.mod_size[2]);
        m["ofsx"] = parameter_t(d.mod_ofs[0]);
        m["ofsy"] = parameter_t(d.mod_ofs[1]);
        m["ofsz"] = parameter_t(d.mod_ofs[2]);
        m["texco"] = P_str(texco[(d.tex_map & 0xffu) < 6 ? (d.tex_map & 0xffu) : 0]);
        const char *pnames[3] = {"proj_x", "proj_y", "proj_z"};
        for (int a = 0; a < 3; a++) {
            const uint32_t pc = (d.tex_map >> (8 * (a + 1))) & 0xffu;
            static const char *ax[5] = {"", "x", "y", "z", "n"};
            m[pnames[a]] = P_str(pc == YR_PROJ_DEFAULT ? (a == 0 ? "x" : (a == 1 ? "y" : "z")) : ax[pc < 5 ? pc : 4]);
        }
        mods.push_back(m);
    }
    paramMap_t p;
    p["name"] = P_str(name);
    p["type"] = P_str("generic");
    p["color"] = P_col(d.color);
    p["specular"] = P_col(d.specular);
    p["hard"] = parameter_t(d.hard);
    y.addShader(p, mods);
}

static void iface_light(yafrayInterface_t &y, const yr_light_desc &d, int k, bool path_cache) {
    char name[32];
    snprintf(name, sizeof(name), "light%04d", k);
    paramMap_t p;
    p["name"] = P_str(name);
    p["power"] = parameter_t(d.power);
    switch (d.type) {
    case YR_LIGHT_POINT:
        p["type"] = P_str("pointlight");
        p["from"] = P_pt(d.p[0]);
        p["color"] = P_col(d.color);
        p["cast_shadows"] = P_on(d.cast_shadows != 0);
        break;
    case YR_LIGHT_AREA:
        p["type"] = P_str("arealight");
        p["a"] = P_pt(d.p[0]);
        p["b"] = P_pt(d.p[1]);
        p["c"] = P_pt(d.p[2]);
        p["d"] = P_pt(d.p[3]);
        p["color"] = P_col(d.color);
        p["samples"] = parameter_t((float)d.samples);
        p["psamples"] = parameter_t((float)d.psamples);
        break;
    case YR_LIGHT_HEMI:
        p["type"] = P_str("hemilight");
        p["color"] = P_col(d.color);
        p["samples"] = parameter_t((float)d.samples);
        p["maxdistance"] = parameter_t(d.maxdist);
        p["use_QMC"] = P_on(true);
        break;
    case YR_LIGHT_PATH:
        p["type"] = P_str("pathlight");
        p["samples"] = parameter_t((float)d.samples);
        p["depth"] = parameter_t((float)d.depth);
        p["use_QMC"] = P_on(true);
        p["threshold"] = parameter_t(d.threshold > 0 ? d.threshold : 1e9f);
        if (path_cache) p["cache"] = P_on(true);  // the irradiance cache (not modelled by the library)
        break;
    }
    y.addLight(p);
}

static void cmd_iface(const std::string &arm, const SceneFile &s, const char *out, const std::string &extra) {
    yafrayInterface_t *y = arm == "cuda" ? (yafrayInterface_t *)new cudaInterface_t(0, "")
                                         : (yafrayInterface_t *)new interfaceImpl_t(1, "");
    iface_register(*y);
    for (size_t k = 0; k < s.shaders.size(); k++) iface_shader(*y, s.shaders[k], (int)k);
    std::vector<std::string> shader_names;
    for (size_t k = 0; k < s.shaders.size(); k++) {
        char name[32];
        snprintf(name, sizeof(name), "sh%04d", (int)k);
        shader_names.push_back(name);
    }
    // object names keep the file's order (the interface's tables are
    // ordered by name, and so are the scene's object and light lists)
    for (size_t i = 0; i < s.objs.size(); i++) {
        const SceneFile::Obj &o = s.objs[i];
        char name[32];
        snprintf(name, sizeof(name), "obj%04d", (int)i);
        if (o.inst >= 0) continue;
        std::vector<point3d_t> verts(o.nv);
        for (uint32_t k = 0; k < o.nv; k++) verts[k] = P3(&o.v[3 * k]);
        std::vector<int> faces(o.t.begin(), o.t.end());
        std::vector<GFLOAT> uv(o.uv.begin(), o.uv.end());
        std::vector<CFLOAT> vcol;
        std::vector<std::string> shaders;
        std::vector<int> faceshader;
        if (o.shader == YR_PER_TRIANGLE) {
            shaders = shader_names;
            std::swap(shaders[0], shaders[o.tri_shader[0]]);  // the object's own shader first
            std::vector<int> slot(shader_names.size());
            for (size_t k = 0; k < shaders.size(); k++) slot[atoi(shaders[k].c_str() + 2)] = (int)k;
            for (uint32_t k = 0; k < o.nt; k++) faceshader.push_back(slot[o.tri_shader[k]]);
        } else {
            shaders.push_back(shader_names.at(o.shader));
        }
        y->addObject_trimesh(name, verts, faces, uv, vcol, shaders, faceshader, o.smooth >= 1.f ? o.smooth : 0.f,
                             o.cast != 0, true, true, false, false, color_t(0.0), color_t(0.0), 1.0);
    }
    for (size_t i = 0; i < s.objs.size(); i++) {
        const SceneFile::Obj &o = s.objs[i];
        if (o.inst < 0) continue;
        char name[32], orig[32];
        snprintf(name, sizeof(name), "obj%04d", (int)i);
        snprintf(orig, sizeof(orig), "obj%04d", o.inst);
        float M[16];
        memcpy(M, o.M, sizeof(M));
        y->transformPush(M);
        y->addObject_reference(name, orig);
        y->transformPop();
    }
    for (size_t k = 0; k < s.lights.size(); k++) iface_light(*y, s.lights[k], (int)k, extra == "pathcache");
    paramMap_t cam;
    cam["name"] = P_str("cam");
    cam["from"] = P_pt(s.cam.pos);
    cam["to"] = P_pt(s.cam.look);
    cam["up"] = P_pt(s.cam.up);
    cam["resx"] = parameter_t((float)s.cam.resx);
    cam["resy"] = parameter_t((float)s.cam.resy);
    cam["focal"] = parameter_t(s.cam.focal);
    cam["aspect_ratio"] = parameter_t(s.cam.aspect);
    y->addCamera(cam);
    paramMap_t rp;
    rp["camera_name"] = P_str("cam");
    rp["raydepth"] = parameter_t((float)s.rp.raydepth);
    rp["bias"] = parameter_t(s.rp.self_bias);
    const uint32_t spp = s.rp.spp ? s.rp.spp : 1;
    rp["AA_passes"] = parameter_t(spp > 1 ? 1.f : 0.f);
    rp["AA_minsamples"] = parameter_t(spp > 1 ? (float)(spp - 1) : 1.f);
    rp["AA_pixelwidth"] = parameter_t(s.rp.aa_pixelwidth);
    rp["AA_threshold"] = parameter_t(0.f);
    rp["exposure"] = parameter_t(s.rp.exposure);
    rp["gamma"] = parameter_t(s.rp.gamma);
    rp["clamp_rgb"] = P_on((s.rp.flags & YR_RENDER_CLAMP_RGB) != 0);
    rp["alpha_premultiply"] = P_str((s.rp.flags & YR_RENDER_ALPHA_PREMULTIPLY) ? "on" : "off");
    if (s.rp.background[0] != 0.f || s.rp.background[1] != 0.f || s.rp.background[2] != 0.f) {
        paramMap_t bg;
        bg["name"] = P_str("bg");
        bg["type"] = P_str("constant");
        bg["color"] = P_col(s.rp.background);
        y->addBackground(bg);
        rp["background_name"] = P_str("bg");
    }
    floatSink_t sink(s.cam.resx, s.cam.resy);
    double t0 = now_s();
    y->render(rp, sink);
    double t1 = now_s();
    const int status = arm == "cuda" ? (int)((cudaInterface_t *)y)->lastStatus() : 0;
    printf("{\"status\": %d, \"render_s\": %.6f}\n", status, t1 - t0);
    fflush(stdout);
    FILE *f = fopen(out, "wb");
    wr(f, &sink.img[0], 4 * sink.img.size());
    fclose(f);
    delete y;
}
#endif

// ------------------------------------------------------------- illuminate
// One light's illuminate() at the first hit of a ray, with the light's
// sample stream set from outside, so that the oracle can be given the same
// samples:
//   hemi (hemilight.cc:57-115): HSEQ[0], HSEQ[1] setStart(m0 * samples);
//   path (pathlight.cc:223-403, pathtools.cc:8-43): every level's Halton
//        stream of the state's sampler setStart(m0 * samples); `synced` says
//        whether each level 0..depth-1 was then advanced exactly `samples`
//        times (true when no path stops early);
//   area (arealight.cc:93-198): the global LCG (vector3d.h:262-285) seeded
//        with `lcg`; the values it hands out are returned in vals[], then
//        the grid points of the penumbra guess's probes (rand() seeded with
//        `lcg`, arealight.cc:186).
// Query: u32 light, u32 m0, i32 lcg, f32 eye[3], f32 from[3], f32 dir[3]
// Output: u32 hit, u32 synced, f32 rgb[3], u32 nvals, f32 vals[64]
struct IllumRec {
    uint32_t light, m0;
    int32_t lcg;
    float eye[3], from[3], dir[3];
};

static void cmd_illum(const SceneFile &s, const char *q_path, const char *out) {
    RefScene r;
    build_ref(s, r, true);
    r.scene->BTree = buildObjectTree(r.scene->obj_list);
    r.scene->setupLights();  // as scene_t::render does (scene.cc:555)
    FILE *fi = fopen(q_path, "rb");
    if (!fi) die("cannot open queries");
    uint32_t n;
    rd(fi, &n, 4);
    std::vector<IllumRec> qs(n);
    if (n) rd(fi, &qs[0], sizeof(IllumRec) * n);
    fclose(fi);
    FILE *f = fopen(out, "wb");
    if (!f) die("cannot open output");
    for (uint32_t i = 0; i < n; i++) {
        const IllumRec &q = qs[i];
        uint32_t head[2] = {0, 1};
        float rgb[3] = {0, 0, 0};
        uint32_t nvals = 0;
        float vals[64];
        memset(vals, 0, sizeof(vals));
        renderState_t state;
        surfacePoint_t sp;
        if (q.light >= r.lights.size()) die("bad light index");
        if (r.scene->firstHit(state, sp, P3(q.from), vector3d_t(q.dir[0], q.dir[1], q.dir[2]), false)) {
            head[0] = 1;
            light_t *l = r.lights[q.light];
            const vector3d_t eye = P3(q.eye) - sp.P();
            haltonSampler_t *hs = NULL;
            pathLight_t *pl = NULL;
            switch (s.lights[q.light].type) {
            case YR_LIGHT_HEMI: {
                hemiLight_t *hl = (hemiLight_t *)l;
                hl->HSEQ[0].setStart(q.m0 * (unsigned)hl->samples);
                hl->HSEQ[1].setStart(q.m0 * (unsigned)hl->samples);
                break;
            }
            case YR_LIGHT_PATH: {
                pl = (pathLight_t *)l;
                hs = (haltonSampler_t *)pl->getSampler(state, *r.scene);
                for (int k = 0; k < 2 * (pl->maxdepth + 1); k++) hs->HSEQ[k].setStart(q.m0 * (unsigned)pl->samples);
                break;
            }
            case YR_LIGHT_AREA: {
                areaLight_t *al = (areaLight_t *)l;
                nvals = 2u * (uint32_t)al->samples;
                if (nvals + (uint32_t)al->fsamples > 64) die("area light with more than 64 values");
                myseed = q.lcg;
                for (uint32_t k = 0; k < nvals; k++) vals[k] = ourRandom();
                myseed = q.lcg;
                // the penumbra guess draws its grid points with rand()
                // (arealight.cc:186): the same seed, the same draws
                srand((unsigned)q.lcg);
                for (int k = 0; k < al->fsamples; k++) vals[nvals + k] = (float)(rand() % al->samples);
                srand((unsigned)q.lcg);
                nvals += (uint32_t)al->fsamples;
                break;
            }
            }
            const color_t c = l->illuminate(state, *r.scene, sp, eye);
            rgb[0] = c.getR();
            rgb[1] = c.getG();
            rgb[2] = c.getB();
            if (hs) {
                // how many rounds of paths ran: every level's stream must
                // have advanced the same whole number of rounds of `samples`
                // values (true when no path stops early); head[1] = rounds
                int rounds = -1;
                for (int lev = 0; lev < pl->maxdepth; lev++)
                    for (int k = 2 * lev; k < 2 * lev + 2; k++) {
                        Halton ref(hs->HSEQ[k]._base);
                        ref.setStart(q.m0 * (unsigned)pl->samples);
                        int found = 0;
                        for (int rr = 1; rr <= 4 && !found; rr++) {
                            for (int m = 0; m < pl->samples; m++) ref.getNext();
                            if (ref.value == hs->HSEQ[k].value) found = rr;
                        }
                        if (!found || (rounds >= 0 && rounds != found)) rounds = 0;
                        else if (rounds < 0) rounds = found;
                    }
                head[1] = rounds > 0 ? (uint32_t)rounds : 0;
            }
        }
        wr(f, head, 8);
        wr(f, rgb, 12);
        wr(f, &nvals, 4);
        wr(f, vals, sizeof(vals));
    }
    fclose(f);
}

// ------------------------------------------------------------------- noise
static void cmd_noise(const char *pts_path, const char *out) {
    FILE *fi = fopen(pts_path, "rb");
    if (!fi) die("cannot open points");
    uint32_t n;
    rd(fi, &n, 4);
    std::vector<float> pts(3 * n);
    rd(fi, &pts[0], 12 * n);
    fclose(fi);
    newPerlin_t perlin;
    fBm_t fbm6(1.0, 2.0, 6.0, &perlin);
    fBm_t fbm25(0.8, 2.5, 3.5, &perlin);
    FILE *f = fopen(out, "wb");
    for (uint32_t i = 0; i < n; i++) {
        point3d_t p(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        float v[5] = {perlin(p), fbm6(p), fbm25(p), turbulence(&perlin, p, 2, 1.0, false),
                      turbulence(&perlin, p, 3, 2.5, true)};
        wr(f, v, 20);
    }
    fclose(f);
}

// ---------------------------------------------------------- noise bases
// Every noise basis of newNoise (basictex.cc:34-60) and turbulence
// (noise.cc:808-819) over it, plus the voronoi texture's own metrics.
// Output per point: 10 bases, then turbulence(basis, p, 3, 1.5, hard) for
// hard = 0 / 1 per basis (20 values), then voronoi_t::getFeatures distances
// da[0..3] for the 7 metrics (mk_exponent 2.5): 58 floats.
static void cmd_noisegen(const char *pts_path, const char *out) {
    FILE *fi = fopen(pts_path, "rb");
    if (!fi) die("cannot open points");
    uint32_t n;
    rd(fi, &n, 4);
    std::vector<float> pts(3 * (size_t)n);
    if (n) rd(fi, &pts[0], 12 * (size_t)n);
    fclose(fi);
    noiseGenerator_t *gens[10];
    for (int k = 0; k < 10; k++) gens[k] = newNoise(noise_name(k));
    voronoi_t vor[7];
    for (int k = 0; k < 7; k++) {
        vor[k].setDistM((voronoi_t::dMetricType)k);
        vor[k].setMinkovskyExponent(2.5);
    }
    FILE *f = fopen(out, "wb");
    for (uint32_t i = 0; i < n; i++) {
        const point3d_t p(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        float v[58];
        for (int k = 0; k < 10; k++) {
            v[k] = (*gens[k])(p);
            v[10 + 2 * k] = turbulence(gens[k], p, 3, 1.5, false);
            v[11 + 2 * k] = turbulence(gens[k], p, 3, 1.5, true);
        }
        for (int k = 0; k < 7; k++) {
            vor[k].getFeatures(p);
            for (int j = 0; j < 4; j++) v[30 + 4 * k + j] = vor[k].getDistance(j);
        }
        wr(f, v, sizeof(v));
    }
    fclose(f);
}

// -------------------------------------------------------------- textures
// Each textured shader's texture_t::getColor (rgb) and getFloat at the
// given texture-space points: per shader, per point, 4 floats.
static void cmd_texeval(const SceneFile &s, const char *pts_path, const char *out) {
    FILE *fi = fopen(pts_path, "rb");
    if (!fi) die("cannot open points");
    uint32_t n;
    rd(fi, &n, 4);
    std::vector<float> pts(3 * (size_t)n);
    if (n) rd(fi, &pts[0], 12 * (size_t)n);
    fclose(fi);
    FILE *f = fopen(out, "wb");
    for (size_t k = 0; k < s.shaders.size(); k++) {
        if (s.shaders[k].tex_type == YR_TEX_NONE) continue;
        texture_t *tex = make_texture(s.shaders[k]);
        for (uint32_t i = 0; i < n; i++) {
            const point3d_t p(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
            const colorA_t c = tex->getColor(p);
            const float v[4] = {c.getR(), c.getG(), c.getB(), tex->getFloat(p)};
            wr(f, v, 16);
        }
        delete tex;
    }
    fclose(f);
}

// ------------------------------------------------------------ image outputs
// A float RGBA image (u32 w, u32 h, then w*h*4 floats, top row first)
// written by the reference's own outTga_t (with or without alpha) or
// outHDR_t, pixel by pixel through putPixel as renderArea_t::out does
// (renderblock.cc:8-20).
static void cmd_imgout(const char *kind, const char *in, const char *out) {
    FILE *fi = fopen(in, "rb");
    if (!fi) die("cannot open image");
    uint32_t wh[2];
    rd(fi, wh, 8);
    std::vector<float> px(4 * (size_t)wh[0] * wh[1]);
    if (!px.empty()) rd(fi, &px[0], 4 * px.size());
    fclose(fi);
    const std::string k = kind;
    colorOutput_t *o;
    if (k == "hdr") o = new outHDR_t(wh[0], wh[1], out);
    else if (k == "tga" || k == "tga_alpha") o = new outTga_t(wh[0], wh[1], out, k == "tga_alpha");
    else die("image kind: tga, tga_alpha or hdr");
    for (uint32_t y = 0; y < wh[1]; y++)
        for (uint32_t x = 0; x < wh[0]; x++) {
            const float *p = &px[4 * ((size_t)y * wh[0] + x)];
            o->putPixel(x, y, color_t(p[0], p[1], p[2]), p[3], 0);
        }
    o->flush();
    delete o;
}

// ------------------------------------------------------------------ halton
static void cmd_halton(const char *out) {
    FILE *f = fopen(out, "wb");
    int base = 2;
    for (int b = 0; b < 12; b++) {
        for (unsigned int i = 0; i < 4096; i++) {
            Halton h(base);
            h.setStart(i);
            float v = h.getNext();
            wr(f, &v, 4);
        }
        base = nextPrime(base);
    }
    // RI_vdC / RI_S / RI_LP
    for (unsigned int i = 0; i < 4096; i++) {
        float v[3] = {RI_vdC(i * 2654435761u), RI_S(i * 40503u), RI_LP(i * 7919u)};
        wr(f, v, 12);
    }
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc < 3) die("usage: yr_ref_harness CMD ARGS...");
    std::string cmd = argv[1];
    std::cout.setstate(std::ios::failbit);  // silence the reference's progress output
    if (cmd == "noise") {
        if (argc < 4) die("noise POINTS OUT");
        cmd_noise(argv[2], argv[3]);
        return 0;
    }
    if (cmd == "halton") {
        cmd_halton(argv[2]);
        return 0;
    }
    if (cmd == "imgout") {
        if (argc < 5) die("imgout KIND IN OUT");
        cmd_imgout(argv[2], argv[3], argv[4]);
        return 0;
    }
    if (cmd == "noisegen") {
        if (argc < 4) die("noisegen POINTS OUT");
        cmd_noisegen(argv[2], argv[3]);
        return 0;
    }
    SceneFile s;
    load_scene(argv[2], s);
    if (cmd == "tree") {
        cmd_tree(s, argv[3]);
    } else if (cmd == "rays") {
        if (argc < 5) die("rays SCENE RAYS OUT");
        cmd_rays(s, argv[3], argv[4]);
    } else if (cmd == "instmat") {
        cmd_instmat(s, argv[3]);
    } else if (cmd == "orcomat") {
        cmd_orcomat(s, argv[3]);
    } else if (cmd == "texeval") {
        if (argc < 5) die("texeval SCENE POINTS OUT");
        cmd_texeval(s, argv[3], argv[4]);
    } else if (cmd == "illum") {
        if (argc < 5) die("illum SCENE QUERIES OUT");
        cmd_illum(s, argv[3], argv[4]);
    } else if (cmd == "camera") {
        cmd_camera(s, argv[3]);
    } else if (cmd == "render") {
        if (argc < 5) die("render SCENE OUT THREADS [x0 x1 y0 y1 [REPEATS]]");
        int crop[4];
        bool has_crop = argc >= 9;
        if (has_crop)
            for (int k = 0; k < 4; k++) crop[k] = atoi(argv[5 + k]);
        const int reps = argc >= 10 ? atoi(argv[9]) : 1;
        cmd_render(s, argv[3], atoi(argv[4]), has_crop ? crop : NULL, reps < 1 ? 1 : reps);
#ifdef YR_HARNESS_CUDASCENE
    } else if (cmd == "cudarender") {
        if (argc < 4) die("cudarender SCENE OUT [x0 x1 y0 y1 [STOP_AFTER]]");
        int crop[4];
        const bool has_crop = argc >= 8;
        if (has_crop)
            for (int k = 0; k < 4; k++) crop[k] = atoi(argv[4 + k]);
        cmd_cudarender(s, argv[3], has_crop ? crop : NULL, argc >= 9 ? atol(argv[8]) : -1L);
    } else if (cmd == "iface") {
        if (argc < 5) die("iface SCENE OUT ARM [pathcache]");
        cmd_iface(argv[4], s, argv[3], argc >= 6 ? argv[5] : "");
#endif
    } else if (cmd == "render_blocks") {
        if (argc < 6) die("render_blocks SCENE OUT THREADS BLOCKS [REPEATS]");
        const int reps = argc >= 7 ? atoi(argv[6]) : 1;
        cmd_render_blocks(s, argv[3], atoi(argv[4]), argv[5], reps < 1 ? 1 : reps);
    } else {
        die("unknown command");
    }
    return 0;
}
