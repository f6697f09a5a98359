// cudaInterface_t: YafRay 0.0.9's host API (yafrayInterface_t,
// external.h:144-183: the calls the Blender exporter and the XML loader's
// front ends make) with every render going through the B200 library.
//
// It is interfaceImpl_t (interface_impl.cc) with two changes: the scene it
// renders is a cudascene_t instead of a threadedscene_t, and it keeps what
// the objects the plugins build do not tell by themselves (the area, hemi
// and path lights' and the modulated shaders' parameters, each mesh's
// autosmooth angle, the constant background) as library records for that
// scene.  Objects, shaders, textures, lights and cameras are still made by
// the reference's own factories, so the scene is the reference's; only the
// pixel loop moves to the GPU.  A front end gets it where it gets
// interfaceImpl_t (the getYafray symbol, interface_impl.cc:876-879).
//
// Built here against the reference's headers as they are, linked with the
// reference's objects and libyafray_b200.so, as test infrastructure:
// oracle/Makefile's yr_ref_cudascene drives the same calls through
// interfaceImpl_t and through this class (its iface command).
#ifndef YR_CUDAINTERFACE_H
#define YR_CUDAINTERFACE_H

#include <list>
#include <map>
#include <string>

#include "cudascene.h"
#include "interface_impl.h"

__BEGIN_YAFRAY

class cudaInterface_t : public interfaceImpl_t {
  public:
    // device: the GPU; pluginpath as interfaceImpl_t's (plugins are loaded
    // from there, or registered by the caller through registerFactory)
    explicit cudaInterface_t(int device = 0, const std::string &pluginpath = "");
    virtual void addObject_trimesh(const std::string &name, std::vector<point3d_t> &verts,
                                   const std::vector<int> &faces, std::vector<GFLOAT> &uvcoords,
                                   std::vector<CFLOAT> &vcol, const std::vector<std::string> &shaders,
                                   const std::vector<int> &faceshader, float sm_angle, bool castShadows, bool useR,
                                   bool receiveR, bool caus, bool has_orco, const color_t &caus_rcolor,
                                   const color_t &caus_tcolor, float caus_IOR);
    virtual void addObject_reference(const std::string &name, const std::string &original);
    virtual void addLight(paramMap_t &p);
    virtual void addTexture(paramMap_t &p);
    virtual void addShader(paramMap_t &p, std::list<paramMap_t> &modulators);
    virtual void addFilter(paramMap_t &p);
    virtual void addBackground(paramMap_t &p);
    // interfaceImpl_t::render(params, output) (interface_impl.cc:675-835)
    // with a cudascene_t: the same parameters, the pixels through
    // output.putPixel, then output.flush()
    virtual void render(paramMap_t &p, colorOutput_t &output);
    // interfaceImpl_t::render(params) (interface_impl.cc:442-673): the same,
    // into the file "outfile" as TGA ("output_type" tga, tone-mapped, alpha
    // with "save_alpha") or Radiance HDR ("hdr"; "exr" falls back to HDR
    // as in a build without OpenEXR), written by the library's encoders
    virtual void render(paramMap_t &p);
    virtual void clear();
    // YR_OK, or why the last render did not run (YR_ERR_UNSUPPORTED for a
    // scene the library does not model, a device error, YR_ERR_CANCELLED
    // when the output stopped it); nothing falls back to the CPU renderer
    yr_status lastStatus() const { return status; }

  private:
    // the render settings of interfaceImpl_t::render, applied to `scene`;
    // false (and lastStatus) when the camera is missing
    bool setup(paramMap_t &params, scene_t &scene, bool tonemap);
    int dev;
    yr_status status;
    cudaHints_t hints;
    std::map<std::string, paramMap_t> texture_params;   // addTexture's maps by name
    std::map<std::string, color_t> background_colors;   // "constant" backgrounds by name
    std::set<std::string> other_backgrounds;            // any other background type
};

__END_YAFRAY

#endif
