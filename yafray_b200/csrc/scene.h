// Host-side scene object behind the opaque yr_scene handle.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "dev_common.cuh"
#include "host_build.h"

namespace yr {

// genericShader_t colour parameters + one musgrave/clouds modulator
struct DevShader {
    C3 color;        // scolor
    C3 specular;     // ks
    float hard;
    int tex_type;    // YR_TEX_*
    C3 tc1, tc2;     // texture color1 / color2
    float H, lacunarity, octaves, tsize, intensity;
    float mod_color;
    float mod_spec, mod_hard;  // modulator "specular" / "hard" weights
    float msize[3], mofs[3];
    int tdepth, thard;
    int texco;           // YR_TEXCO_*
    int proj[3];         // source axis (0..2) of texture x / y / z, -1 = none
    int mod_mode;        // YR_MOD_*
    int noise, noise2;   // YR_NOISE_* (noise_type / noise_type1, noise_type2)
    int tshape;          // marble / wood shape, gradient type, voronoi colour type
    int tvariant;        // wood rings, clouds bias, gradient flip_xy
    float turb;          // marble / wood turbulence
    float sharp;         // marble: 1/sharpness when sharpness > 1, else 1
    float offset, gain;  // musgrave
    float distort;       // distorted noise
    float weights[4];    // voronoi weight1..4
    float mk_exp;        // voronoi minkovsky exponent
    int metric;          // voronoi YR_DIST_*
    float viscale;       // voronoi intensity / sum |weight| (0 when the sum is 0)
    float vinvw;         // voronoi 1 / sum |weight| (0 when the sum is 0)
};

struct DevLight {
    int type;            // YR_LIGHT_*
    int samples;         // area: filled quad samples; hemi/path: samples
    int depth;           // path: maxdepth
    int cast;            // point: cast_shadows
    C3 color;            // point: color*power (pointLight_t ctor); others: color
    float power;         // area "pow", hemi/path power
    V3 from;             // point position / area centre
    V3 direction;        // area: unit normal of the quad
    V3 corner, tox, toy; // area: corner a, b-a, d-a
    float maxdist;       // hemi
    float sampdiv;       // hemi: power/samples
    int pt_base;         // area: first entry in DevRender::area_pts
    int psamples;        // area: probes of the penumbra guess (0: none)
    C3 rawc;             // the light's "color" parameter (before any power scale)
    int probe_off;       // area with psamples: first probe slot of a vertex
};

struct DevCamera {
    V3 pos, vright, vup, vto;
    int resx, resy;
};

struct DevRender {
    DevCamera cam;
    const DevShader *shaders;
    const DevLight *lights;
    const float *area_pts;      // per area sample: point, jit.first, jit.second (9 floats)
    const uint32_t *tri_shader; // shader per global triangle
    int nlights;
    int nshaders;
    uint32_t spp;
    float pw;                   // AA pixel width
    float totsamdiv;            // 1/(spp-1) as PFLOAT (scene.cc:776-777)
    uint32_t seed;
    float self_bias;
    int raydepth;
    C3 background;
    int rx0, ry0, rw, rh;       // pixel region (x0, y0, width, height)
    int path_light;             // index of the path light or -1
    int path_samples;
    int path_depth;
    int tonemap;                // YR_RENDER_TONEMAP
    int clamp_rgb;              // YR_RENDER_CLAMP_RGB
    int premultiply;            // YR_RENDER_ALPHA_PREMULTIPLY
    float exposure;             // scene_t::exposure = -"exposure"
    float gamma_r;              // scene_t::gamma_R = 1/"gamma" (0 for gamma 0)
    int has_guess;              // some area light guesses the penumbra first (psamples > 0)
    float path_threshold;       // path light "threshold" of its adaptive extra rounds (0: one round)
};

// Device allocation tracked by the scene (freed in yr_scene_destroy).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

}  // namespace yr

struct yr_scene {
    int device = 0;
    yr::DevScene dev{};
    yr::DevRender rdr{};
    std::vector<yr::DevBuf> bufs;
    std::vector<yr::DevShader> shaders;
    std::vector<yr::DevLight> lights;
    std::vector<yr_shader_desc> shader_desc;
    std::vector<yr_light_desc> light_desc;
    std::vector<float> area_pts;
    yr_camera_desc camera{};
    yr_render_params render{};
    yr_scene_info info{};
    int max_tree_depth = 0;
    int *status = nullptr;          // device status word, then the ray-query work counter
    int *status_host = nullptr;     // pinned mirror
    yr::DevShader *d_shaders = nullptr;
    yr::DevLight *d_lights = nullptr;
    // small per-scene scratch (host staging image), grown on demand
    std::vector<yr::DevBuf> scratch;
    bool pooled = false;            // counted among the device's live scenes
    // adjoint parameter vector: first index of each shader's and light's
    // parameters; unit specular direction of each shader
    uint32_t nparams = 0;
    std::vector<int> sh_pbase, li_pidx;
    std::vector<float> spec_dir;      // 4 per shader
    int *d_sh_pbase = nullptr, *d_li_pidx = nullptr;
    float4 *d_spec_dir = nullptr;
};

namespace yr {
// derived device records from the ABI descriptors (scene.cu)
void make_shader(const yr_shader_desc &d, DevShader &o);
bool valid_shader(const yr_shader_desc &d);
yr_status make_lights(const std::vector<yr_light_desc> &in, std::vector<DevLight> &out, std::vector<float> &pts);
void make_camera(const yr_camera_desc &c, DevCamera &o);
yr_status upload_params(yr_scene *s);
// read and clear the device status word (synchronizes `stream`)
yr_status take_status(yr_scene *s, cudaStream_t stream);
// Render scratch shared by all scenes of a device: a render takes a block
// for its duration (it synchronizes its stream before it returns) and gives
// it back, so scenes rendered one after another share one block.  The
// blocks are freed when the device's last scene is destroyed.
yr_status pool_acquire(int device, size_t bytes, DevBuf &out);
void pool_release(int device, const DevBuf &b);

struct PoolBlock {
    int device;
    cudaStream_t stream;
    DevBuf buf;
    PoolBlock(int d, cudaStream_t s) : device(d), stream(s) {}
    ~PoolBlock() {
        if (buf.p) {
            int cur = 0;
            cudaGetDevice(&cur);
            cudaSetDevice(device);
            cudaStreamSynchronize(stream);  // nothing in flight may still use it
            pool_release(device, buf);
            cudaSetDevice(cur);
        }
    }
};

// drop the cached batch state of every batch that holds `s` (batch.cu,
// adjoint.cu)
void batch_forget(const yr_scene *s);
void adj_batch_forget(const yr_scene *s);
}  // namespace yr
