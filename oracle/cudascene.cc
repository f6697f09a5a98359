// cudascene_t (cudascene.h): YafRay's scene rendered through the B200
// library.  The scene's own lists are read once and handed to
// yr_scene_create (the library builds the same kd-trees and object tree);
// every render is then one yr_render call.
//
// What it takes: meshObject_t objects (flat, or smoothed with the angle
// given in the hints; one shader per object or per triangle; texture
// coordinates; the orco matrix of a transformed mesh), referenceObject_t
// placements of them, genericShader_t shaders without modulators (or with
// the record given in the hints), point lights (other lights through the
// hints), the pinhole camera, a constant background (through the hints),
// and the render settings the library models (ray depth, bias, one AA pass
// resampling every pixel, tone map, alpha premultiply, region).  Anything
// else is refused with YR_ERR_UNSUPPORTED before any device work;
// lastStatus() says so.
#include "cudascene.h"

#include <cmath>
#include <iostream>
#include <map>
#include <vector>

#include "basicshaders.h"
#include "camera.h"
#include "mesh.h"
#include "pointlight.h"
#include "reference.h"

__BEGIN_YAFRAY

// The plugin classes keep their parameters in protected members.  A
// pointer to such a member may be formed inside a class derived from its
// owner (naming the derived class); reading an object through it is then
// ordinary member access.  These accessors are the only use of the
// derived classes, which are never instantiated.
struct meshFields : meshObject_t {
    static std::vector<point3d_t> meshObject_t::*m_vertices() { return &meshFields::vertices; }
    static std::vector<triangle_t> meshObject_t::*m_triangles() { return &meshFields::triangles; }
    static std::vector<vector3d_t> meshObject_t::*m_normals() { return &meshFields::normals; }
    static std::vector<GFLOAT> meshObject_t::*m_facesuv() { return &meshFields::facesuv; }
    static bool meshObject_t::*m_unt() { return &meshFields::unt; }
    static bool meshObject_t::*m_hasorco() { return &meshFields::hasorco; }
    static matrix4x4_t meshObject_t::*m_backOrco() { return &meshFields::backOrco; }
};
struct refFields : referenceObject_t {
    static object3d_t *referenceObject_t::*m_original() { return &refFields::original; }
    static matrix4x4_t referenceObject_t::*m_M() { return &refFields::M; }
    static matrix4x4_t referenceObject_t::*m_back() { return &refFields::back; }
};
struct shaderFields : genericShader_t {
    static color_t genericShader_t::*m_scolor() { return &shaderFields::scolor; }
    static color_t genericShader_t::*m_ks() { return &shaderFields::ks; }
    static CFLOAT genericShader_t::*m_hard() { return &shaderFields::hard; }
    static std::vector<modulator_t> genericShader_t::*m_mods() { return &shaderFields::mods; }
};
struct pointFields : pointLight_t {
    static point3d_t pointLight_t::*m_from() { return &pointFields::from; }
    static color_t pointLight_t::*m_color() { return &pointFields::color; }
    static bool pointLight_t::*m_cast() { return &pointFields::cast_shadows; }
    static CFLOAT pointLight_t::*m_glow() { return &pointFields::glow_int; }
};
struct cameraFields : camera_t {
    static vector3d_t camera_t::*m_vto() { return &cameraFields::vto; }
    static vector3d_t camera_t::*m_vup() { return &cameraFields::vup; }
    static vector3d_t camera_t::*m_vright() { return &cameraFields::vright; }
    static camera_t::cameraType camera_t::*m_type() { return &cameraFields::camtype; }
    static PFLOAT camera_t::*m_aperture() { return &cameraFields::aperture; }
};

static void put3(float *d, const point3d_t &p) { d[0] = p.x; d[1] = p.y; d[2] = p.z; }
static void put3(float *d, const vector3d_t &v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; }
static void put3(float *d, const color_t &c) { d[0] = c.getR(); d[1] = c.getG(); d[2] = c.getB(); }
static void put16(float *d, const matrix4x4_t &m) {
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) d[4 * a + b] = m[a][b];
}

cudascene_t::~cudascene_t() {
    if (handle) yr_scene_destroy(handle);
}

yr_status cudascene_t::capture() {
    // shaders: one record per distinct genericShader_t, in order of first use
    std::map<const shader_t *, uint32_t> shader_index;
    std::vector<yr_shader_desc> shaders;
    struct add_shader {
        static yr_status run(const shader_t *s, const cudaHints_t *h, std::map<const shader_t *, uint32_t> &idx,
                             std::vector<yr_shader_desc> &out, uint32_t &k) {
            std::map<const shader_t *, uint32_t>::iterator it = idx.find(s);
            if (it != idx.end()) {
                k = it->second;
                return YR_OK;
            }
            yr_shader_desc d;
            memset(&d, 0, sizeof(d));
            std::map<const shader_t *, yr_shader_desc>::const_iterator hs;
            if (h && h->refused.count(s)) return YR_ERR_UNSUPPORTED;
            if (h && (hs = h->shaders.find(s)) != h->shaders.end()) {
                d = hs->second;
            } else {
                const genericShader_t *g = dynamic_cast<const genericShader_t *>(s);
                if (!g || !(g->*shaderFields::m_mods()).empty()) return YR_ERR_UNSUPPORTED;
                put3(d.color, g->*shaderFields::m_scolor());
                put3(d.specular, g->*shaderFields::m_ks());
                d.hard = g->*shaderFields::m_hard();
            }
            k = (uint32_t)out.size();
            idx[s] = k;
            out.push_back(d);
            return YR_OK;
        }
    };

    // objects, in obj_list order (the order buildObjectTree sees them)
    std::vector<yr_object_desc> objs;
    std::vector<std::vector<float> > verts, mats;
    std::vector<std::vector<uint32_t> > tris, tri_shaders;
    std::map<const object3d_t *, uint32_t> obj_index;
    for (std::list<object3d_t *>::const_iterator o = obj_list.begin(); o != obj_list.end(); ++o)
        obj_index[*o] = (uint32_t)obj_index.size();
    for (std::list<object3d_t *>::const_iterator o = obj_list.begin(); o != obj_list.end(); ++o) {
        if (hints && hints->refused.count(*o)) return YR_ERR_UNSUPPORTED;
        if ((*o)->caustics()) return YR_ERR_UNSUPPORTED;  // pathlight.cc:198: caustic paths are not modelled
        verts.push_back(std::vector<float>());
        tris.push_back(std::vector<uint32_t>());
        tri_shaders.push_back(std::vector<uint32_t>());
        mats.push_back(std::vector<float>());
        const referenceObject_t *ro = dynamic_cast<const referenceObject_t *>(*o);
        if (ro) {  // a placement of a mesh of this scene: its M and M^-1 as the reference holds them
            std::map<const object3d_t *, uint32_t>::const_iterator org = obj_index.find(ro->*refFields::m_original());
            if (org == obj_index.end() || !dynamic_cast<const meshObject_t *>(org->first)) return YR_ERR_UNSUPPORTED;
            mats.back().resize(32);
            put16(&mats.back()[0], ro->*refFields::m_M());
            put16(&mats.back()[16], ro->*refFields::m_back());
            yr_object_desc d;
            memset(&d, 0, sizeof(d));
            d.instance_of = org->second;
            objs.push_back(d);
            continue;
        }
        const meshObject_t *m = dynamic_cast<const meshObject_t *>(*o);
        if (!m) return YR_ERR_UNSUPPORTED;  // spheres: not taken here
        if (m->*meshFields::m_hasorco()) return YR_ERR_UNSUPPORTED;  // explicit orco points
        const std::vector<point3d_t> &V = m->*meshFields::m_vertices();
        const std::vector<triangle_t> &T = m->*meshFields::m_triangles();
        float smooth = 0.f;
        if (!(m->*meshFields::m_normals()).empty()) {  // smoothed: the library recomputes the normals from the angle
            std::map<const object3d_t *, float>::const_iterator sa;
            if (!hints || (sa = hints->smooth_angle.find(m)) == hints->smooth_angle.end()) return YR_ERR_UNSUPPORTED;
            smooth = sa->second;
        }
        if (!(m->*meshFields::m_unt())) {  // made through transform(): its orco matrix
            mats.back().resize(16);
            put16(&mats.back()[0], m->*meshFields::m_backOrco());
        }
        verts.back().resize(3 * V.size());
        for (size_t i = 0; i < V.size(); i++) put3(&verts.back()[3 * i], V[i]);
        tris.back().resize(3 * T.size());
        tri_shaders.back().resize(T.size());
        uint32_t obj_shader = 0;
        yr_status st = add_shader::run(m->getShader(), hints, shader_index, shaders, obj_shader);
        if (st != YR_OK) return st;
        bool per_triangle = false;
        for (size_t i = 0; i < T.size(); i++) {
            tris.back()[3 * i] = (uint32_t)(T[i].a - &V[0]);
            tris.back()[3 * i + 1] = (uint32_t)(T[i].b - &V[0]);
            tris.back()[3 * i + 2] = (uint32_t)(T[i].c - &V[0]);
            const shader_t *ts = T[i].getShader();
            uint32_t k = obj_shader;
            if (ts && ts != m->getShader()) {
                if ((st = add_shader::run(ts, hints, shader_index, shaders, k)) != YR_OK) return st;
                per_triangle = true;
            }
            tri_shaders.back()[i] = k;
        }
        yr_object_desc d;
        memset(&d, 0, sizeof(d));
        d.verts = &verts.back()[0];
        d.nverts = (uint32_t)V.size();
        d.tris = &tris.back()[0];
        d.ntris = (uint32_t)T.size();
        d.shader = per_triangle ? YR_PER_TRIANGLE : obj_shader;
        d.tri_shaders = per_triangle ? &tri_shaders.back()[0] : NULL;
        d.cast_shadows = m->castShadows() ? 1 : 0;
        d.smooth_angle = smooth;
        // texture coordinates: triangle i holds facesuv[6i .. 6i+5] (setUV)
        const std::vector<GFLOAT> &uv = m->*meshFields::m_facesuv();
        if (!uv.empty() && uv.size() >= 6 * T.size()) d.uvs = &uv[0];
        objs.push_back(d);
    }
    // vectors may have moved while growing: point the records again
    for (size_t i = 0; i < objs.size(); i++) {
        if (mats[i].size() == 32) {  // a reference
            objs[i].instance_matrix = &mats[i][0];
            objs[i].instance_inverse = &mats[i][16];
            continue;
        }
        objs[i].verts = verts[i].empty() ? NULL : &verts[i][0];
        objs[i].tris = tris[i].empty() ? NULL : &tris[i][0];
        if (objs[i].shader == YR_PER_TRIANGLE) objs[i].tri_shaders = &tri_shaders[i][0];
        if (mats[i].size() == 16) objs[i].orco_matrix = &mats[i][0];
    }

    std::vector<yr_light_desc> lights;
    for (std::list<light_t *>::const_iterator l = light_list.begin(); l != light_list.end(); ++l) {
        // every light lights both the camera hits and the path vertices
        if (!(*l)->useInRender() || !(*l)->useInIndirect()) return YR_ERR_UNSUPPORTED;
        if (hints && hints->refused.count(*l)) return YR_ERR_UNSUPPORTED;
        std::map<const light_t *, yr_light_desc>::const_iterator hl;
        if (hints && (hl = hints->lights.find(*l)) != hints->lights.end()) {
            lights.push_back(hl->second);
            continue;
        }
        const pointLight_t *p = dynamic_cast<const pointLight_t *>(*l);
        if (!p || p->*pointFields::m_glow() != 0) return YR_ERR_UNSUPPORTED;
        yr_light_desc d;
        memset(&d, 0, sizeof(d));
        d.type = YR_LIGHT_POINT;
        put3(d.color, p->*pointFields::m_color());  // already colour * power
        d.power = 1.0f;
        put3(d.p[0], p->*pointFields::m_from());
        d.cast_shadows = (p->*pointFields::m_cast()) ? 1 : 0;
        lights.push_back(d);
    }

    const camera_t &cam = *render_camera;
    if (cam.*cameraFields::m_type() != camera_t::CM_PERSPECTIVE || cam.*cameraFields::m_aperture() != 0)
        return YR_ERR_UNSUPPORTED;
    if (fog_density != 0 || alpha_maskbackground) return YR_ERR_UNSUPPORTED;
    if (background && !(hints && hints->has_background)) return YR_ERR_UNSUPPORTED;

    yr_scene_desc d;
    memset(&d, 0, sizeof(d));
    d.objects = objs.empty() ? NULL : &objs[0];
    d.nobjects = (uint32_t)objs.size();
    d.shaders = shaders.empty() ? NULL : &shaders[0];
    d.nshaders = (uint32_t)shaders.size();
    d.lights = lights.empty() ? NULL : &lights[0];
    d.nlights = (uint32_t)lights.size();
    // the pinhole itself comes from the camera's vectors below; the
    // constructor-argument record only carries the resolution
    put3(d.camera.pos, cam.position());
    put3(d.camera.look, cam.position() + cam.*cameraFields::m_vto());
    put3(d.camera.up, cam.position() + cam.*cameraFields::m_vup());
    d.camera.resx = cam.resX();
    d.camera.resy = cam.resY();
    d.camera.aspect = 1.0f;
    d.camera.focal = 1.0f;

    yr_render_params &r = d.render;  // (seed 0: the reference has no rotation seed)
    if (background)
        for (int k = 0; k < 3; k++) r.background[k] = hints->background[k];
    r.self_bias = self_bias;
    r.raydepth = maxraylevel;
    // the library resamples every pixel in one AA pass (AA_threshold 0)
    if (AA_passes == 0) {
        r.spp = 1;
    } else if (AA_passes == 1 && AA_threshold <= 0 && !AA_jitterfirst && AA_minsamples >= 1) {
        r.spp = 1 + (uint32_t)AA_minsamples;
    } else {
        return YR_ERR_UNSUPPORTED;
    }
    r.aa_pixelwidth = AA_pixelwidth;
    r.flags = (do_tonemap ? YR_RENDER_TONEMAP : 0) | (clamp_rgb ? YR_RENDER_CLAMP_RGB : 0) |
              (alpha_premultiply ? YR_RENDER_ALPHA_PREMULTIPLY : 0);
    r.exposure = -exposure;  // setExposure stored -e (scene.h:163)
    // setGamma stored 1/g (scene.h:162): the g whose reciprocal is gamma_R
    r.gamma = 0.0f;
    if (gamma_R != 0) {
        float g = (float)(1.0 / gamma_R);
        for (int k = 0; k < 4 && (CFLOAT)(1.0 / g) != gamma_R; k++)
            g = (CFLOAT)(1.0 / g) < gamma_R ? nextafterf(g, 0.0f) : nextafterf(g, 1e30f);
        r.gamma = g;
    }
    // region (setRegion, scene.h:216): the pixels whose centre's screen
    // position scene_t::render accepts (scene.cc:749-752)
    const int W = cam.resX(), H = cam.resY();
    int x0 = W, x1 = 0, y0 = H, y1 = 0;
    for (int j = 0; j < W; j++) {
        const PFLOAT sx = 2.0 * (((PFLOAT)j + 0.5) / (PFLOAT)W) - 1.0;
        if (sx >= scxmin && sx < scxmax) {
            if (j < x0) x0 = j;
            x1 = j + 1;
        }
    }
    for (int i = 0; i < H; i++) {
        const PFLOAT sy = 1.0 - 2.0 * (((PFLOAT)i + 0.5) / (PFLOAT)H);
        if (sy >= scymin && sy < scymax) {
            if (i < y0) y0 = i;
            y1 = i + 1;
        }
    }
    if (x1 <= x0 || y1 <= y0) return YR_ERR_INVALID_ARG;
    rx0 = x0;
    ry0 = y0;
    rw = x1 - x0;
    rh = y1 - y0;
    if (!(x0 == 0 && x1 == W && y0 == 0 && y1 == H)) {
        r.region[0] = x0;
        r.region[1] = x1;
        r.region[2] = y0;
        r.region[3] = y1;
    }

    yr_status st = yr_scene_create(&d, dev, &handle);
    if (st != YR_OK) {
        handle = 0;
        return st;
    }
    float pos[3], vto[3], vup[3], vright[3];
    put3(pos, cam.position());
    put3(vto, cam.*cameraFields::m_vto());
    put3(vup, cam.*cameraFields::m_vup());
    put3(vright, cam.*cameraFields::m_vright());
    return yr_scene_set_camera_vectors(handle, pos, vto, vup, vright);
}

// yr_render_progressive's callback: one wave's region pixels to putPixel
struct putPixels_t {
    colorOutput_t *out;
    const float *rgba;
    int W, x0, y0, rw;
};
static int put_pixels(void *user, uint32_t first, uint32_t count) {
    const putPixels_t &p = *(const putPixels_t *)user;
    for (uint32_t k = first; k < first + count; k++) {
        const int x = p.x0 + (int)(k % (uint32_t)p.rw), y = p.y0 + (int)(k / (uint32_t)p.rw);
        const float *c = &p.rgba[4 * ((size_t)y * p.W + x)];
        if (!p.out->putPixel(x, y, color_t(c[0], c[1], c[2]), c[3], 0)) return 0;  // the output asked to stop
    }
    return 1;
}

void cudascene_t::render(colorOutput_t &out) {
    if (!handle) {
        status = capture();
        if (status != YR_OK) {
            std::cerr << "cudascene_t: " << yr_status_string(status) << std::endl;
            if (handle) yr_scene_destroy(handle);
            handle = 0;
            return;
        }
    }
    const int W = render_camera->resX(), H = render_camera->resY();
    std::vector<float> rgba((size_t)W * H * 4);
    yr_render_stats st;
    memset(&st, 0, sizeof(st));
    putPixels_t pp = {&out, &rgba[0], W, rx0, ry0, rw};
    // waves of about 64 rows, so the output sees the frame as it is made
    status = yr_render_progressive(handle, &rgba[0], (uint32_t)(64 * rw), put_pixels, &pp, &st, 0);
    if (status != YR_OK) {
        if (status != YR_ERR_CANCELLED) std::cerr << "cudascene_t: " << yr_status_string(status) << std::endl;
        return;
    }
    // pixels outside the region are rendered as 0 by scene_t::render too
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            if (x >= rx0 && x < rx0 + rw && y >= ry0 && y < ry0 + rh) continue;
            if (!out.putPixel(x, y, color_t(0.0), 0, 0)) return;
        }
}

__END_YAFRAY
