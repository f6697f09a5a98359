// cudascene_t: a YafRay 0.0.9 scene class whose render(colorOutput_t&)
// renders through the B200 library (include/yr.h) instead of the CPU
// block loop.  This is the class a YafRay maintainer adds to yafraycore
// (yafraycore/cudascene.{h,cc}) to make the library a drop-in: the loader
// picks it where it picks threadedscene_t (loader/render.cc:1131-1153,
// interface_impl.cc:562,755), everything that fills the scene (objects,
// lights, shaders, camera, render settings) stays as it is.
//
// Built here against the reference's headers as they are (no access
// changes) and linked with the reference's objects and libyafray_b200.so,
// as test infrastructure: oracle/Makefile's yr_ref_cudascene renders a
// scene built from the reference's own objects through this class.
#ifndef YR_CUDASCENE_H
#define YR_CUDASCENE_H

#include <map>
#include <set>

#include "scene.h"

extern "C" {
#include "../include/yr.h"
}

__BEGIN_YAFRAY

// What the scene's objects do not tell the library by themselves, for a
// front end that saw the plugins' parameter maps (cudaInterface_t): the
// records of lights and shaders it translated, each object's autosmooth
// angle, the constant background colour, and the objects it could not
// translate (refused at render time).
struct cudaHints_t {
    std::map<const light_t *, yr_light_desc> lights;
    std::map<const shader_t *, yr_shader_desc> shaders;
    std::map<const object3d_t *, float> smooth_angle;
    std::set<const void *> refused;
    bool has_background;
    float background[3];
    cudaHints_t() : has_background(false) { background[0] = background[1] = background[2] = 0.f; }
    void clear() {
        lights.clear();
        shaders.clear();
        smooth_angle.clear();
        refused.clear();
        has_background = false;
    }
};

class cudascene_t : public scene_t {
  public:
    explicit cudascene_t(int device = 0)
        : hints(0), handle(0), dev(device), status(YR_OK), rx0(0), ry0(0), rw(0), rh(0) {}
    virtual ~cudascene_t();
    // scene_t::render(colorOutput_t&) (scene.h:136): the frame through
    // yr_render_progressive, each finished wave's pixels handed to the
    // output with colorOutput_t::putPixel (output.h:36-38) as
    // renderArea_t::out does (renderblock.cc:8-20); a putPixel that returns
    // false stops the render (lastStatus() YR_ERR_CANCELLED).  A scene the
    // library cannot take, or a device error, leaves the output untouched
    // and is reported by lastStatus(); nothing falls back to the CPU
    // renderer.
    virtual void render(colorOutput_t &out);
    yr_status lastStatus() const { return status; }
    static scene_t *factory(int device = 0) { return new cudascene_t(device); }
    // records for what the objects do not tell (may be NULL; not owned)
    void setHints(const cudaHints_t *h) { hints = h; }

  private:
    yr_status capture();  // the scene's objects, lights and camera -> yr_scene
    const cudaHints_t *hints;
    yr_scene *handle;
    int dev;
    yr_status status;
    int rx0, ry0, rw, rh;  // the render region in pixels
};

__END_YAFRAY

#endif
