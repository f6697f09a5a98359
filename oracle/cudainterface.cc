// cudaInterface_t (cudainterface.h): the reference's interfaceImpl_t with
// its renders through cudascene_t.  Each add* call first lets the
// reference's own implementation build the plugin object, then translates
// the same parameter map into the library's record for that object, with
// the factory's parameter names and defaults (arealight.cc:235-254,
// hemilight.cc, pathlight.cc:753-807, basicshaders.cc:217-365, basictex.cc
// factories, sunsky.cc:12-17).  What the library does not model is marked
// refused, and a render of a scene that uses it returns
// YR_ERR_UNSUPPORTED.
#include "cudainterface.h"

#include <cstring>
#include <iostream>

#include "HDR_io.h"
#include "camera.h"
#include "targaIO.h"

extern "C" {
#include "../include/yr.h"
}

__BEGIN_YAFRAY

namespace {

void put3(float *d, const point3d_t &p) { d[0] = p.x; d[1] = p.y; d[2] = p.z; }
void put3(float *d, const color_t &c) { d[0] = c.getR(); d[1] = c.getG(); d[2] = c.getB(); }

std::string str_param(paramMap_t &p, const char *name, const char *def) {
    std::string dflt(def);
    const std::string *v = &dflt;
    p.getParam(name, v);
    return *v;
}
template <class T> T num_param(paramMap_t &p, const char *name, T def) {
    T v = def;
    p.getParam(name, v);
    return v;
}
color_t color_param(paramMap_t &p, const char *name, const color_t &def) {
    color_t c = def;
    p.getParam(name, c);
    return c;
}

// newNoise (noise.cc): unknown names give the improved Perlin noise
uint32_t noise_type(const std::string &n) {
    static const char *names[] = {"newperlin", "stdperlin", "blender", "voronoi_f1", "voronoi_f2",
                                  "voronoi_f3", "voronoi_f4", "voronoi_f2f1", "voronoi_crackle", "cellnoise"};
    for (uint32_t k = 0; k < 10; k++)
        if (n == names[k]) return k;
    return YR_NOISE_NEWPERLIN;
}
uint32_t wave_shape(const std::string &n) { return n == "saw" ? 1u : (n == "tri" ? 2u : 0u); }

// The texture block of a modulator: the texture factory's parameters
// (basictex.cc) into the record.  false: a texture the library does not
// model (image, random_noise, or an unknown type).
bool texture_record(paramMap_t &p, yr_shader_desc &d) {
    const std::string type = str_param(p, "type", "");
    put3(d.tex_color1, color_param(p, "color1", color_t(0.0)));
    put3(d.tex_color2, color_param(p, "color2", color_t(1.0)));
    if (type == "clouds") {  // basictex.cc:98-115
        d.tex_type = YR_TEX_CLOUDS;
        d.tex_noise = noise_type(str_param(p, "noise_type", ""));
        d.tex_depth = num_param<int>(p, "depth", 2);
        d.tex_size = num_param<float>(p, "size", 1.f);
        d.tex_hard = num_param<bool>(p, "hard", false) ? 1u : 0u;
        const std::string bias = str_param(p, "bias", "");
        d.tex_variant = bias == "positive" ? 1u : (bias == "negative" ? 2u : 0u);
    } else if (type == "marble" || type == "wood") {  // basictex.cc:158-176, 223-243
        d.tex_type = type == "marble" ? YR_TEX_MARBLE : YR_TEX_WOOD;
        d.tex_noise = noise_type(str_param(p, "noise_type", ""));
        d.tex_depth = num_param<int>(p, "depth", 2);
        d.tex_turbulence = num_param<float>(p, "turbulence", 1.f);
        d.tex_size = num_param<float>(p, "size", 1.f);
        d.tex_hard = num_param<bool>(p, "hard", false) ? 1u : 0u;
        d.tex_shape = wave_shape(str_param(p, "shape", ""));
        if (type == "marble") d.tex_sharpness = num_param<float>(p, "sharpness", 1.f);
        else d.tex_variant = str_param(p, "wood_type", "") == "rings" ? 1u : 0u;
    } else if (type == "voronoi") {  // basictex.cc:621-652
        d.tex_type = YR_TEX_VORONOI;
        const std::string ct = str_param(p, "color_type", "");
        d.tex_shape = ct == "col1" ? 1u : (ct == "col2" ? 2u : (ct == "col3" ? 3u : 0u));
        d.tex_weights[0] = num_param<float>(p, "weight1", 1.f);
        d.tex_weights[1] = num_param<float>(p, "weight2", 0.f);
        d.tex_weights[2] = num_param<float>(p, "weight3", 0.f);
        d.tex_weights[3] = num_param<float>(p, "weight4", 0.f);
        d.tex_mk_exponent = num_param<float>(p, "mk_exponent", 2.5f);
        d.tex_intensity = num_param<float>(p, "intensity", 1.f);
        d.tex_size = num_param<float>(p, "size", 1.f);
        static const char *metrics[] = {"real", "squared", "manhattan", "chebychev", "minkovsky_half",
                                        "minkovsky_four", "minkovsky"};
        const std::string dm = str_param(p, "distance_metric", "");
        d.tex_metric = YR_DIST_REAL;
        for (uint32_t k = 0; k < 7; k++)
            if (dm == metrics[k]) d.tex_metric = k;
    } else if (type == "musgrave") {  // basictex.cc:687-708
        const std::string mt = str_param(p, "type", "");
        d.tex_type = YR_TEX_MUSGRAVE_FBM;
        if (mt == "multifractal") d.tex_type = YR_TEX_MUSGRAVE_MULTIFRACTAL;
        else if (mt == "heteroterrain") d.tex_type = YR_TEX_MUSGRAVE_HETEROTERRAIN;
        else if (mt == "hybridmf") d.tex_type = YR_TEX_MUSGRAVE_HYBRIDMF;
        else if (mt == "ridgedmf") d.tex_type = YR_TEX_MUSGRAVE_RIDGEDMF;
        d.tex_noise = noise_type(str_param(p, "noise_type", ""));
        d.tex_H = num_param<float>(p, "H", 1.f);
        d.tex_lacunarity = num_param<float>(p, "lacunarity", 2.f);
        d.tex_octaves = num_param<float>(p, "octaves", 2.f);
        d.tex_offset = num_param<float>(p, "offset", 1.f);
        d.tex_gain = num_param<float>(p, "gain", 1.f);
        d.tex_size = num_param<float>(p, "size", 1.f);
        d.tex_intensity = num_param<float>(p, "intensity", 1.f);
    } else if (type == "distorted_noise") {  // basictex.cc:737-754
        d.tex_type = YR_TEX_DISTORTED_NOISE;
        d.tex_noise = noise_type(str_param(p, "noise_type1", ""));
        d.tex_noise2 = noise_type(str_param(p, "noise_type2", ""));
        d.tex_distort = num_param<float>(p, "distort", 1.f);
        d.tex_size = num_param<float>(p, "size", 1.f);
    } else if (type == "gradient") {  // basictex.cc:812-823
        d.tex_type = YR_TEX_GRADIENT;
        static const char *kinds[] = {"linear", "quadratic", "cubic", "diagonal", "sphere", "halo"};
        const std::string gt = str_param(p, "gradient_type", "");
        d.tex_shape = YR_GRAD_LINEAR;
        for (uint32_t k = 0; k < 6; k++)
            if (gt == kinds[k]) d.tex_shape = k;
        d.tex_variant = num_param<bool>(p, "flip_xy", false) ? 1u : 0u;
    } else {
        return false;
    }
    return true;
}

}  // namespace

cudaInterface_t::cudaInterface_t(int device, const std::string &pluginpath)
    : interfaceImpl_t(1, pluginpath), dev(device), status(YR_OK) {}

void cudaInterface_t::clear() {
    interfaceImpl_t::clear();
    hints.clear();
    texture_params.clear();
    background_colors.clear();
    other_backgrounds.clear();
}

void cudaInterface_t::addObject_trimesh(const std::string &name, std::vector<point3d_t> &verts,
                                        const std::vector<int> &faces, std::vector<GFLOAT> &uvcoords,
                                        std::vector<CFLOAT> &vcol, const std::vector<std::string> &shaders,
                                        const std::vector<int> &faceshader, float sm_angle, bool castShadows,
                                        bool useR, bool receiveR, bool caus, bool has_orco,
                                        const color_t &caus_rcolor, const color_t &caus_tcolor, float caus_IOR) {
    std::map<std::string, object3d_t *>::iterator old = object_table.find(name);
    const object3d_t *before = old == object_table.end() ? NULL : old->second;
    interfaceImpl_t::addObject_trimesh(name, verts, faces, uvcoords, vcol, shaders, faceshader, sm_angle,
                                       castShadows, useR, receiveR, caus, has_orco, caus_rcolor, caus_tcolor,
                                       caus_IOR);
    std::map<std::string, object3d_t *>::iterator now = object_table.find(name);
    if (now == object_table.end() || now->second == before) return;  // not made
    hints.smooth_angle.erase(now->second);
    hints.refused.erase(now->second);
    // the library computes autoSmooth's normals itself from the angle
    // (interface_impl.cc:245-246 smooths when the angle is above 0); it
    // reads angles below 1 degree as flat shading, so those are refused,
    // as are explicit orco points
    if (sm_angle > 0.0) hints.smooth_angle[now->second] = sm_angle;
    if ((sm_angle > 0.0 && sm_angle < 1.0) || has_orco) hints.refused.insert(now->second);
}

void cudaInterface_t::addObject_reference(const std::string &name, const std::string &original) {
    interfaceImpl_t::addObject_reference(name, original);
}

void cudaInterface_t::addLight(paramMap_t &p) {
    const std::string name = str_param(p, "name", "");
    std::map<std::string, light_t *>::iterator old = light_table.find(name);
    const light_t *before = old == light_table.end() ? NULL : old->second;
    if (before) {
        hints.lights.erase(before);
        hints.refused.erase(before);
    }
    interfaceImpl_t::addLight(p);
    std::map<std::string, light_t *>::iterator now = light_table.find(name);
    if (now == light_table.end() || now->second == before) return;
    const light_t *l = now->second;
    const std::string type = str_param(p, "type", "");
    yr_light_desc d;
    memset(&d, 0, sizeof(d));
    d.cast_shadows = 1;
    if (type == "pointlight") {  // read from the object itself (cudascene_t)
        return;
    } else if (type == "arealight") {  // arealight.cc:235-254
        d.type = YR_LIGHT_AREA;
        const char *corner[4] = {"a", "b", "c", "d"};
        for (int k = 0; k < 4; k++) {
            point3d_t q(0, 0, 0);
            p.getParam(corner[k], q);
            put3(d.p[k], q);
        }
        put3(d.color, color_param(p, "color", color_t(0.0)));
        d.power = num_param<float>(p, "power", 1.f);
        d.samples = num_param<int>(p, "samples", 50);
        d.psamples = num_param<int>(p, "psamples", 0);
        if (num_param<bool>(p, "dummy", false)) {  // a light for photons only
            hints.refused.insert(l);
            return;
        }
    } else if (type == "hemilight") {  // hemilight.cc factory
        d.type = YR_LIGHT_HEMI;
        color_t c(0.0);
        if (!p.getParam("color", c)) {  // the background's colour, set at render time
            hints.refused.insert(l);
            return;
        }
        put3(d.color, c);
        d.power = num_param<float>(p, "power", 1.f);
        d.samples = num_param<int>(p, "samples", 16);
        if (d.samples < 1) d.samples = 1;
        d.maxdist = num_param<float>(p, "maxdistance", -1.f);
    } else if (type == "pathlight") {  // pathlight.cc:753-807
        d.type = YR_LIGHT_PATH;
        d.color[0] = d.color[1] = d.color[2] = 1.f;
        d.power = num_param<float>(p, "power", 1.f);
        d.depth = num_param<int>(p, "depth", 3);
        d.samples = num_param<int>(p, "samples", 16);
        if (d.samples < 1) d.samples = 1;
        d.threshold = num_param<float>(p, "threshold", 0.1f);
        // the irradiance cache, the "direct" mode and the occlusion mode
        // are not modelled
        if (num_param<bool>(p, "cache", false) || num_param<bool>(p, "direct", false) ||
            str_param(p, "mode", "") == "occlusion") {
            hints.refused.insert(l);
            return;
        }
    } else {
        hints.refused.insert(l);
        return;
    }
    hints.lights[l] = d;
}

void cudaInterface_t::addTexture(paramMap_t &p) {
    interfaceImpl_t::addTexture(p);
    const std::string name = str_param(p, "name", "");
    if (!name.empty()) texture_params[name] = p;
}

void cudaInterface_t::addShader(paramMap_t &p, std::list<paramMap_t> &modulators) {
    const std::string name = str_param(p, "name", "");
    std::map<std::string, shader_t *>::iterator old = shader_table.find(name);
    const shader_t *before = old == shader_table.end() ? NULL : old->second;
    if (before) {
        hints.shaders.erase(before);
        hints.refused.erase(before);
    }
    interfaceImpl_t::addShader(p, modulators);
    std::map<std::string, shader_t *>::iterator now = shader_table.find(name);
    if (now == shader_table.end() || now->second == before) return;
    const shader_t *s = now->second;
    // genericShader_t::factory (basicshaders.cc:217-365)
    if (str_param(p, "type", "") != "generic") {
        hints.refused.insert(s);
        return;
    }
    yr_shader_desc d;
    memset(&d, 0, sizeof(d));
    put3(d.color, color_param(p, "color", color_t(0.0)));
    put3(d.specular, color_param(p, "specular", color_t(0.0)));
    d.hard = num_param<float>(p, "hard", 1.f);
    // reflection, refraction and an environment shader are not on the path
    const color_t zero(0.0);
    if (color_param(p, "reflected", zero).energy() > 0 || color_param(p, "transmitted", zero).energy() > 0 ||
        color_param(p, "transmited", zero).energy() > 0 || str_param(p, "environment", "") != "") {
        hints.refused.insert(s);
        return;
    }
    if (modulators.empty()) {
        hints.shaders[s] = d;
        return;
    }
    if (modulators.size() > 1) {  // the record holds one modulator
        hints.refused.insert(s);
        return;
    }
    paramMap_t &m = modulators.front();
    std::map<std::string, paramMap_t>::iterator tex = texture_params.find(str_param(m, "texname", ""));
    if (tex == texture_params.end() || !texture_record(tex->second, d)) {
        hints.refused.insert(s);
        return;
    }
    // modulator_t settings (basicshaders.cc:271-360)
    const float size = num_param<float>(m, "size", 1.f);
    d.mod_size[0] = num_param<float>(m, "sizex", 1.f);
    d.mod_size[1] = num_param<float>(m, "sizey", 1.f);
    d.mod_size[2] = num_param<float>(m, "sizez", 1.f);
    if (size != 1.f) d.mod_size[0] = d.mod_size[1] = d.mod_size[2] = size;
    d.mod_ofs[0] = num_param<float>(m, "ofsx", 0.f);
    d.mod_ofs[1] = num_param<float>(m, "ofsy", 0.f);
    d.mod_ofs[2] = num_param<float>(m, "ofsz", 0.f);
    d.mod_color = num_param<float>(m, "color", 0.f);
    d.mod_specular = num_param<float>(m, "specular", 0.f);
    d.mod_hard = num_param<float>(m, "hard", 0.f);
    // string2texmode (texture.cc:31-51): screen / difference / divide /
    // darken / lighten leave the colour as it is and are not taken
    const std::string mode = str_param(m, "mode", "mix");
    if (mode == "add") d.mod_mode = YR_MOD_ADD;
    else if (mode == "sub") d.mod_mode = YR_MOD_SUB;
    else if (mode == "mul") d.mod_mode = YR_MOD_MUL;
    else if (mode == "screen" || mode == "difference" || mode == "divide" || mode == "darken" || mode == "lighten")
        d.mod_mode = 0xffffffffu;
    else d.mod_mode = YR_MOD_MIX;
    // string2texcotype (texture.h:135-149): unknown names give "uv"
    const std::string texco = str_param(m, "texco", "orco");
    uint32_t tc = YR_TEXCO_UV;
    if (texco == "global") tc = YR_TEXCO_GLOBAL;
    else if (texco == "orco") tc = YR_TEXCO_ORCO;
    else if (texco == "window") tc = YR_TEXCO_WINDOW;
    else if (texco == "normal") tc = YR_TEXCO_NORMAL;
    else if (texco == "reflect") tc = YR_TEXCO_REFLECT;
    // string2texprojection: position in "nxyz", anything else disables the axis
    const char *pname[3] = {"proj_x", "proj_y", "proj_z"};
    const char *pdef[3] = {"x", "y", "z"};
    uint32_t proj[3];
    for (int k = 0; k < 3; k++) {
        const std::string a = str_param(m, pname[k], pdef[k]);
        proj[k] = a == "x" ? YR_PROJ_X : (a == "y" ? YR_PROJ_Y : (a == "z" ? YR_PROJ_Z : YR_PROJ_NONE));
    }
    d.tex_map = tc | (proj[0] << 8) | (proj[1] << 16) | (proj[2] << 24);
    // displacement, the transmission / reflection channels, the image
    // mappings and the modulator's own matrix are not modelled
    bool other = d.mod_mode == 0xffffffffu || num_param<float>(m, "transmission", 0.f) != 0.f ||
                 num_param<float>(m, "reflection", 0.f) != 0.f || num_param<float>(m, "normal", 0.f) != 0.f ||
                 str_param(m, "mapping", "flat") != "flat";
    static const char *mnames[16] = {"m00", "m01", "m02", "m03", "m10", "m11", "m12", "m13",
                                     "m20", "m21", "m22", "m23", "m30", "m31", "m32", "m33"};
    for (int k = 0; k < 16; k++)
        if (num_param<float>(m, mnames[k], (k % 5) == 0 ? 1.f : 0.f) != ((k % 5) == 0 ? 1.f : 0.f)) other = true;
    if (other) {
        hints.refused.insert(s);
        return;
    }
    hints.shaders[s] = d;
}

void cudaInterface_t::addFilter(paramMap_t &p) {
    interfaceImpl_t::addFilter(p);  // (both filter kinds are disabled in the reference: none is made)
}

void cudaInterface_t::addBackground(paramMap_t &p) {
    interfaceImpl_t::addBackground(p);
    const std::string name = str_param(p, "name", "");
    if (name.empty() || background_table.find(name) == background_table.end()) return;
    background_colors.erase(name);
    other_backgrounds.erase(name);
    if (str_param(p, "type", "") == "constant")  // sunsky.cc:12-17
        background_colors[name] = color_param(p, "color", color_t(1.0));
    else
        other_backgrounds.insert(name);
}

// interfaceImpl_t::render's settings (interface_impl.cc:677-830), with its
// parameter names, defaults and limits
bool cudaInterface_t::setup(paramMap_t &params, scene_t &scene, bool tonemap) {
    const std::string camera = str_param(params, "camera_name", "");
    std::map<std::string, camera_t *>::iterator cam = camera_table.find(camera);
    if (camera.empty() || cam == camera_table.end()) {
        std::cerr << "cudaInterface_t: no camera to render" << std::endl;
        status = YR_ERR_INVALID_ARG;
        return false;
    }
    int AA_passes = 0, AA_minsamples = 1;
    if (params.getParam("samples", AA_passes)) AA_passes -= 1;  // the obsolete name counts the first pass
    else params.getParam("AA_passes", AA_passes);
    if (AA_passes < 0) AA_passes = 1;
    params.getParam("AA_minsamples", AA_minsamples);
    if (AA_passes && AA_minsamples < 1) AA_minsamples = 1;
    PFLOAT AA_pixelwidth = num_param<float>(params, "AA_pixelwidth", 1.5f), AA_threshold = 0.05f;
    if (AA_pixelwidth < 1.0) AA_pixelwidth = 1.0;
    else if (AA_pixelwidth > 2.0) AA_pixelwidth = 2.0;
    if (!params.getParam("tolerance", AA_threshold)) params.getParam("AA_threshold", AA_threshold);
    scene.setCamera(cam->second);
    for (std::map<std::string, object3d_t *>::iterator i = object_table.begin(); i != object_table.end(); ++i)
        scene.addObject(i->second);
    for (std::map<std::string, light_t *>::iterator i = light_table.begin(); i != light_table.end(); ++i)
        scene.addLight(i->second);
    for (std::map<std::string, filter_t *>::iterator i = filter_table.begin(); i != filter_table.end(); ++i)
        scene.addFilter(i->second);
    scene.setMaxRayDepth(num_param<int>(params, "raydepth", 3));
    const std::string background = str_param(params, "background_name", "");
    hints.has_background = false;
    if (!background.empty() && background_table.find(background) != background_table.end()) {
        scene.setBackground(background_table[background]);
        std::map<std::string, color_t>::iterator bc = background_colors.find(background);
        if (bc != background_colors.end()) {
            hints.has_background = true;
            put3(hints.background, bc->second);
        }
    }
    scene.alphaPremultiply(str_param(params, "alpha_premultiply", "off") == "on");
    scene.alphaMaskBackground(str_param(params, "alpha_maskbackground", "off") == "on");
    scene.setExposure(num_param<float>(params, "exposure", 0.f));
    scene.setGamma(num_param<float>(params, "gamma", 1.f));
    scene.tonemap(tonemap);
    scene.setFog(num_param<float>(params, "fog_density", 0.f), color_param(params, "fog_color", color_t(1.0)));
    scene.setAASamples(AA_passes, AA_minsamples, AA_pixelwidth, AA_threshold,
                       num_param<bool>(params, "AA_jitterfirst", false));
    scene.clampRGB(num_param<bool>(params, "clamp_rgb", false));
    scene.setRegion(num_param<float>(params, "border_xmin", -1.5f), num_param<float>(params, "border_xmax", 1.5f),
                    num_param<float>(params, "border_ymin", -1.5f), num_param<float>(params, "border_ymax", 1.5f));
    scene.setBias(num_param<float>(params, "bias", 0.1f));
    return true;
}

void cudaInterface_t::render(paramMap_t &params, colorOutput_t &output) {
    cudascene_t scene(dev);
    scene.setHints(&hints);
    // an external render always tone-maps (interface_impl.cc:812-814)
    if (!setup(params, scene, true)) return;
    scene.render(output);
    status = scene.lastStatus();
    output.flush();
}

// a float image of the frame, for the file encoders
class imageOutput_t : public colorOutput_t {
  public:
    imageOutput_t(int w, int h) : W(w), H(h), rgba((size_t)w * h * 4, 0.f) {}
    virtual bool putPixel(int x, int y, const color_t &c, CFLOAT alpha = 0, PFLOAT depth = 0) {
        if (x < 0 || y < 0 || x >= W || y >= H) return true;
        float *p = &rgba[4 * ((size_t)y * W + x)];
        p[0] = c.getR();
        p[1] = c.getG();
        p[2] = c.getB();
        p[3] = alpha;
        return true;
    }
    virtual void flush() {}
    int W, H;
    std::vector<float> rgba;
};

void cudaInterface_t::render(paramMap_t &params) {
    const std::string camera = str_param(params, "camera_name", "");
    std::map<std::string, camera_t *>::iterator cam = camera_table.find(camera);
    if (camera.empty() || cam == camera_table.end()) {
        std::cerr << "cudaInterface_t: no camera to render" << std::endl;
        status = YR_ERR_INVALID_ARG;
        return;
    }
    const std::string outfile = str_param(params, "outfile", "salida.tga");
    const std::string type = str_param(params, "output_type", "tga");
    const bool save_alpha = num_param<bool>(params, "save_alpha", false);
    // HDR (and EXR, which this build writes as HDR, interface_impl.cc:641-655)
    // bypasses the tone map; TGA applies it
    const bool hdr = type == "hdr" || type.find("exr") != std::string::npos;
    imageOutput_t img(cam->second->resX(), cam->second->resY());
    cudascene_t scene(dev);
    scene.setHints(&hints);
    if (!setup(params, scene, !hdr)) return;
    scene.render(img);
    status = scene.lastStatus();
    if (status != YR_OK) return;
    status = yr_image_write(outfile.c_str(), hdr ? YR_IMAGE_HDR : YR_IMAGE_TGA, &img.rgba[0], img.W, img.H,
                            (!hdr && save_alpha) ? (int32_t)YR_IMAGE_ALPHA : 0);
    if (status != YR_OK) std::cerr << "cudaInterface_t: " << yr_status_string(status) << std::endl;
}

__END_YAFRAY
