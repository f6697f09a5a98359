/*
 * yr.h - C ABI of the B200 ray-casting hot path for YafRay 0.0.9.
 *
 * A YafRay host (scene, XML loader, light/shader plugin API) keeps building
 * its scene as today and calls these entry points instead of the per-ray C++
 * virtuals.  Plain C types only: no CUDA or torch types cross this boundary
 * (streams are passed as `void*` = cudaStream_t).
 *
 * Every entry returns a yr_status; nothing calls exit() or throws across the
 * ABI (the reference exits on internal inconsistencies, kdtree.cc:300).
 * Device-side problems (iteration caps, stack overflow, corrupt trees) are
 * written to a device status word and returned by the call that launched
 * the kernel.
 *
 * Threading: calls are reentrant per (yr_scene, stream); one yr_scene may be
 * used from one host thread at a time.  (The reference calls shoot() and
 * illuminate() from N pthreads with a per-thread renderState_t,
 * scene.h:51-73.)
 */
#ifndef YR_H
#define YR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define YR_API __attribute__((visibility("default")))
#else
#define YR_API
#endif

typedef enum yr_status {
    YR_OK = 0,
    YR_ERR_INVALID_ARG = 1,     /* NULL pointer, bad index, bad size          */
    YR_ERR_CUDA = 2,            /* a CUDA runtime call failed                  */
    YR_ERR_OUT_OF_MEMORY = 3,   /* device or host allocation failed           */
    YR_ERR_ITERATION_CAP = 4,   /* a device loop hit its iteration cap        */
    YR_ERR_STACK_OVERFLOW = 5,  /* kd / object-tree stack deeper than the cap */
    YR_ERR_BAD_TREE = 6,        /* node or primitive index out of range       */
    YR_ERR_CANCELLED = 7,       /* the output sink asked to stop              */
    YR_ERR_UNSUPPORTED = 8,     /* feature not on this path                   */
    YR_ERR_EMPTY_SCENE = 9,     /* no objects / no triangles                  */
    YR_ERR_NO_DEVICE = 10,      /* no CUDA device or kernel image missing     */
    YR_ERR_TOO_LARGE = 11       /* request above a documented maximum size    */
} yr_status;

YR_API const char *yr_status_string(yr_status s);
YR_API const char *yr_version(void);

/* ------------------------------------------------------------------------
 * Flattened kd-tree (the device format).
 *
 * Replaces kdTreeNode (kdtree.h:23-61): 8 bytes instead of 16 on 64-bit,
 * because the leaf stores a 32-bit index instead of a pointer.
 *   interior: word = bit pattern of the float split position,
 *             flags = axis (0..2) | right_child << 2   (left child = this+1)
 *   leaf:     flags = 3 | nprims << 2,
 *             word  = triangle index when nprims == 1 (kdTreeNode::onePrimitive),
 *                     else offset into `prims` (kdTreeNode::primitives)
 * Triangle indices are local to the object (0..ntris-1); right_child is
 * local to the object's node array.  `bound` is kdTree_t::treeBound
 * (the triangle bound grown by 1e-4 of its diagonal, kdtree.cc:83-89).
 * ------------------------------------------------------------------------ */
typedef struct yr_kd_node {
    uint32_t word;
    uint32_t flags;
} yr_kd_node;

typedef struct yr_kdtree {
    yr_kd_node *nodes;
    uint32_t nnodes;
    uint32_t *prims;
    uint32_t nprims;
    float bound[6];          /* min xyz, max xyz                               */
    int32_t max_depth;       /* kdTree_t::maxDepth after the ctor's defaults  */
    int32_t max_leaf_size;   /* kdTree_t::maxLeafSize                          */
    float cost_ratio;        /* kdTree_t::costRatio (incl. the large-N penalty) */
    float empty_bonus;
} yr_kdtree;

/* Build the SAH kd-tree of one mesh on the host, with the parameters that
 * meshObject_t uses (mesh.cc:162,487: depth -1, leaf size -1, cost 1.2,
 * empty bonus 0.40).  Replaces kdTree_t::kdTree_t (kdtree.cc:57-138).
 * verts: 3*nverts floats; tris: 3*ntris vertex indices. */
YR_API yr_status yr_kdtree_build(const float *verts, uint32_t nverts,
                                 const uint32_t *tris, uint32_t ntris,
                                 yr_kdtree **out);
YR_API void yr_kdtree_free(yr_kdtree *tree);

/* kdTree_t::kdTree_t(prims, n, depth, leafSize, cost_ratio, emptyBonus)
 * with explicit parameters (kdtree.h:127-128; <= 0 depth / leaf size pick
 * the ctor's defaults) and `nthreads` host threads (subtrees below the top
 * levels are built concurrently; the tree is the same as with 1 thread). */
typedef struct yr_kdtree_params {
    int32_t max_depth;
    int32_t max_leaf_size;
    float cost_ratio;
    float empty_bonus;
    int32_t large_scene_penalty;  /* kdtree.cc:79-80 cost ratio penalty      */
    int32_t reserved;
} yr_kdtree_params;

YR_API yr_status yr_kdtree_build_ex(const float *verts, uint32_t nverts, const uint32_t *tris, uint32_t ntris,
                                    const yr_kdtree_params *params, int nthreads, yr_kdtree **out);

/* The same trees as yr_kdtree_build_ex, node for node and leaf list for
 * leaf list, for several meshes at once, built on GPU `device`: the binned
 * sweep of nodes above 128 triangles (kdTree_t::pigeonMinCost,
 * kdtree.cc:167-304) level by level over all meshes, then one thread per
 * node of at most 128 triangles running kdTree_t::buildTree's recursion
 * (kdtree.cc:416-582, with triBoxClip, triclip.cc:50-240, and the exact
 * sweep kdTree_t::minimalCost, kdtree.cc:311-406).  Inputs and outputs are
 * host memory; out[i] (freed by yr_kdtree_free) is mesh i's tree.
 * Coordinates must be finite (YR_ERR_INVALID_ARG otherwise). */
typedef struct yr_kdtree_mesh {
    const float *verts;      /* 3*nverts floats                                */
    uint32_t nverts;
    const uint32_t *tris;    /* 3*ntris vertex indices                         */
    uint32_t ntris;
} yr_kdtree_mesh;

YR_API yr_status yr_kdtree_build_gpu(const yr_kdtree_mesh *meshes, uint32_t nmeshes,
                                     const yr_kdtree_params *params, int32_t device, yr_kdtree **out);

/* Object tree node (geomeTree_t, geometree.h:8-32): left < 0 marks a leaf
 * whose `right` is the object index; node 0 is the root, children follow
 * in depth-first order (left subtree first). */
typedef struct yr_object_node {
    float bmin[3];
    int32_t left;
    float bmax[3];
    int32_t right;
} yr_object_node;

/* referenceObject_t::getBound (reference.cc:135-165): the box of the eight
 * corners of `bound` (min xyz, max xyz) placed by the row-major 4x4 matrix
 * M, as the object tree sees an instance. */
YR_API yr_status yr_instance_bound(const float *bound, const float *matrix, float *out);

/* buildObjectTree (object3d.cc:30-53): greedy nearest-pair clustering of
 * the objects' bounds (6 floats each: min xyz, max xyz) with the
 * bound_distance metric, in object-list order.  `out` must hold 2n-1 nodes. */
YR_API yr_status yr_object_tree_build(const float *bounds, uint32_t n, yr_object_node *out, uint32_t *nout);

/* ------------------------------------------------------------------------
 * Scene description.  The records below are also the on-disk layout of the
 * "YRS1" scene files the tests and the benchmark exchange (little endian).
 * ------------------------------------------------------------------------ */

/* camera_t ctor arguments (camera.cc:27-87), pinhole (CM_PERSPECTIVE). */
typedef struct yr_camera_desc {
    float pos[3];
    float look[3];
    float up[3];             /* a POINT, as in the reference (vup = up - pos) */
    int32_t resx, resy;
    float aspect;            /* usually 1                                      */
    float focal;             /* "focal": width-1 image plane at this distance  */
} yr_camera_desc;

/* Procedural textures (basictex.cc).  Musgrave types share
 * textureMusgrave_t (basictex.cc:656-709) with the generator of its "type". */
enum {
    YR_TEX_NONE = 0,
    YR_TEX_MUSGRAVE_FBM = 1,             /* musgrave, type "fBm"           */
    YR_TEX_CLOUDS = 2,                   /* clouds (basictex.cc:64-104)     */
    YR_TEX_MARBLE = 3,                   /* marble (basictex.cc:110-175)    */
    YR_TEX_WOOD = 4,                     /* wood (basictex.cc:181-249)      */
    YR_TEX_VORONOI = 5,                  /* voronoi (basictex.cc:560-650)   */
    YR_TEX_MUSGRAVE_MULTIFRACTAL = 6,    /* musgrave, type "multifractal"   */
    YR_TEX_MUSGRAVE_HETEROTERRAIN = 7,   /* musgrave, type "heteroterrain"  */
    YR_TEX_MUSGRAVE_HYBRIDMF = 8,        /* musgrave, type "hybridmf"       */
    YR_TEX_MUSGRAVE_RIDGEDMF = 9,        /* musgrave, type "ridgedmf"       */
    YR_TEX_DISTORTED_NOISE = 10,         /* distorted_noise (basictex.cc:711-746) */
    YR_TEX_GRADIENT = 11                 /* gradient (basictex.cc:752-815)  */
};
/* Noise bases by the "noise_type" names of newNoise (basictex.cc:34-60). */
enum {
    YR_NOISE_NEWPERLIN = 0,       /* "newperlin" (the default)        */
    YR_NOISE_STDPERLIN = 1,       /* "stdperlin"                      */
    YR_NOISE_BLENDER = 2,         /* "blender"                        */
    YR_NOISE_VORONOI_F1 = 3,      /* "voronoi_f1" (distance: real)    */
    YR_NOISE_VORONOI_F2 = 4,      /* "voronoi_f2"                     */
    YR_NOISE_VORONOI_F3 = 5,      /* "voronoi_f3"                     */
    YR_NOISE_VORONOI_F4 = 6,      /* "voronoi_f4"                     */
    YR_NOISE_VORONOI_F2F1 = 7,    /* "voronoi_f2f1"                   */
    YR_NOISE_VORONOI_CRACKLE = 8, /* "voronoi_crackle"                */
    YR_NOISE_CELLNOISE = 9        /* "cellnoise"                      */
};
/* marble / wood "shape" */
enum { YR_WAVE_SIN = 0, YR_WAVE_SAW = 1, YR_WAVE_TRI = 2 };
/* voronoi texture "distance_metric" (voronoi_t::dMetricType) */
enum {
    YR_DIST_REAL = 0, YR_DIST_SQUARED = 1, YR_DIST_MANHATTAN = 2, YR_DIST_CHEBYCHEV = 3,
    YR_DIST_MINKOVSKY_HALF = 4, YR_DIST_MINKOVSKY_FOUR = 5, YR_DIST_MINKOVSKY = 6
};
/* gradient "gradient_type" */
enum {
    YR_GRAD_LINEAR = 0, YR_GRAD_QUADRATIC = 1, YR_GRAD_CUBIC = 2, YR_GRAD_DIAGONAL = 3,
    YR_GRAD_SPHERE = 4, YR_GRAD_HALO = 5
};
/* modulator "mode" (texture.cc:499-534) applied to the diffuse colour */
enum { YR_MOD_MIX = 0, YR_MOD_MUL = 1, YR_MOD_ADD = 2, YR_MOD_SUB = 3 };

/* genericShader_t (basicshaders.h:37-152) with at most one modulator
 * (texture.cc:499-534) on the diffuse colour, driving one procedural
 * texture.  The texture's parameters keep the names of its factory; each
 * texture reads the fields its factory reads and ignores the others. */
typedef struct yr_shader_desc {
    float color[3];          /* "color": diffuse albedo (scolor)               */
    float specular[3];       /* "specular": Phong colour (ks)                  */
    float hard;              /* "hard": Phong exponent                         */
    uint32_t tex_type;       /* YR_TEX_*                                       */
    float tex_color1[3];     /* musgrave "color1"                              */
    float tex_color2[3];     /* musgrave "color2"                              */
    float tex_H;             /* "H"                                            */
    float tex_lacunarity;    /* "lacunarity"                                   */
    float tex_octaves;       /* "octaves"                                      */
    float tex_size;          /* texture "size" (musgrave, clouds, marble, wood,
                                voronoi, distorted_noise)                     */
    float tex_intensity;     /* musgrave / voronoi "intensity" (iscale)        */
    float mod_color;         /* modulator "color": mix weight into C           */
    float mod_size[3];       /* modulator sizex/y/z                            */
    float mod_ofs[3];        /* modulator ofsx/y/z                             */
    uint32_t tex_noise;      /* YR_NOISE_*                                     */
    int32_t tex_depth;       /* clouds / marble / wood "depth": turbulence
                                octaves                                       */
    uint32_t tex_hard;       /* clouds / marble / wood "hard"                  */
    uint32_t tex_map;        /* modulator "texco" and "proj_x/y/z"
                                (modulator_t::doMapping, texture.cc:122-320,
                                procedural path): bits 0-7 YR_TEXCO_*, bits
                                8-15 / 16-23 / 24-31 the source axis of x / y
                                / z as YR_PROJ_*; 0 = global texco, x y z     */
    /* record version 2 */
    uint32_t mod_mode;       /* modulator "mode": YR_MOD_*                     */
    uint32_t tex_shape;      /* marble / wood "shape" YR_WAVE_*; gradient
                                "gradient_type" YR_GRAD_*; voronoi
                                "color_type" 0 int, 1-3 col1-col3             */
    uint32_t tex_variant;    /* wood "wood_type": 1 rings, 0 bands; clouds
                                "bias": 0 none, 1 positive, 2 negative;
                                gradient "flip_xy"                            */
    float tex_turbulence;    /* marble / wood "turbulence"                     */
    float tex_sharpness;     /* marble "sharpness"                             */
    float tex_offset;        /* musgrave "offset"                              */
    float tex_gain;          /* musgrave "gain"                                */
    float tex_distort;       /* distorted_noise "distort"                      */
    uint32_t tex_noise2;     /* distorted_noise "noise_type2" (tex_noise is
                                "noise_type1")                                */
    float tex_weights[4];    /* voronoi "weight1".."weight4"                   */
    float tex_mk_exponent;   /* voronoi "mk_exponent"                          */
    uint32_t tex_metric;     /* voronoi "distance_metric" YR_DIST_*            */
    /* record version 3 */
    float mod_specular;      /* modulator "specular": weight of the texture
                                colour in the specular colour ks, by the same
                                mode as "color" (modulator_t::modulate,
                                texture.cc:499-534); 0 = not modulated        */
    float mod_hard;          /* modulator "hard": weight of the texture value
                                (getFloat) in the Phong exponent; 0 = not
                                modulated.  The adjoint refuses shaders with
                                either weight above 0                          */
} yr_shader_desc;

/* yr_shader_desc.tex_map.  TEXCO_ORCO reads the hit point as orco does for
 * a mesh without orco coordinates and without a transform
 * (meshObject_t::toObjectOrco, mesh.cc:510-514); TEXCO_NORMAL reads the
 * shading normal; TEXCO_WINDOW the camera sample's screen position
 * (x, y in [-1, 1], z 0) at a camera hit and (0, 0, 0) at a path vertex,
 * whose surface point has no screen position (scene.cc:234, 749);
 * TEXCO_REFLECT the eye direction reflected about the face-forwarded
 * normal, the eye being the direction the shading call looks from
 * (texture.cc:148-165); TEXCO_UV the hit's texture coordinates as
 * (2u - 1, 1 - 2v, 0) (texture.cc:127-133, yr_object_desc.uvs). */
enum { YR_TEXCO_GLOBAL = 0, YR_TEXCO_ORCO = 1, YR_TEXCO_NORMAL = 2, YR_TEXCO_WINDOW = 3, YR_TEXCO_REFLECT = 4,
       YR_TEXCO_UV = 5 };
enum { YR_PROJ_DEFAULT = 0, YR_PROJ_X = 1, YR_PROJ_Y = 2, YR_PROJ_Z = 3, YR_PROJ_NONE = 4 };

enum { YR_LIGHT_POINT = 0, YR_LIGHT_AREA = 1, YR_LIGHT_HEMI = 2, YR_LIGHT_PATH = 3 };

/* One record for every light plugin on the path:
 *   point: pointlight.cc:70-90   (p[0] = "from")
 *   area:  arealight.cc:235-254  (p[0..3] = "a","b","c","d", samples,
 *          psamples)
 *   hemi:  hemilight.cc:117+     (samples, maxdist, use_QMC always)
 *   path:  pathlight.cc:753-807  (samples, depth, threshold; use_QMC,
 *          cache off, no photon maps) */
typedef struct yr_light_desc {
    uint32_t type;
    float color[3];
    float power;
    float p[4][3];
    int32_t samples;
    int32_t depth;
    float maxdist;
    uint32_t cast_shadows;   /* point light "cast_shadows" (default 1)        */
    int32_t psamples;        /* area light "psamples" (0..64): probes of the
                                penumbra guess (areaLight_t::guessLight,
                                arealight.cc:176-198) before the samples; 0 =
                                every point samples the light.  Probe j of a
                                point with QMC sample index m looks at grid
                                point floor(samples * u), u = halton(5,
                                m*psamples + j) rotated like the light's first
                                dimension (see yr_render)                    */
    float threshold;         /* path light "threshold" (the factory's default
                                0.1): after the first round of paths, up to 3
                                more rounds where the rounds' four partial
                                sums disagree (pathLight_t::takeSample,
                                pathlight.cc:349-374); <= 0 = one round only.
                                Round r of camera sample s takes the QMC
                                index (r*spp + s)*samples + i for path i     */
    uint32_t reserved;
} yr_light_desc;

/* Render parameters.  The pixel loop follows scene_t::render(renderArea_t&)
 * (scene.cc:724-823) with every pixel resampled: sample 0 at the pixel
 * centre, samples 1..spp-1 at the AA positions of one pass with
 * AA_minsamples = spp-1.  QMC indices are explicit (see yr_render). */
typedef struct yr_render_params {
    float self_bias;         /* render "bias" (scene_t::self_bias, default 0.1) */
    int32_t raydepth;        /* render "raydepth" (maxraylevel, default 3)     */
    uint32_t spp;            /* camera samples per pixel (>= 1)               */
    float aa_pixelwidth;     /* AA_pixelwidth (default 1)                      */
    uint32_t seed;           /* Cranley-Patterson rotation seed               */
    float background[3];     /* constant background colour (black = none)     */
    uint32_t flags;          /* YR_RENDER_* bits                               */
    int32_t region[4];       /* x0, x1, y0, y1: render only these pixels
                                (scene_t::setRegion / the loader's -r option);
                                all zero = the whole image                    */
    /* record version 3 */
    float exposure;          /* render "exposure" (scene_t::setExposure; 0 =
                                off); applied with YR_RENDER_TONEMAP          */
    float gamma;             /* render "gamma" (scene_t::setGamma; 1 = off)   */
} yr_render_params;

/* yr_render_params.flags:
 * YR_RENDER_SHADOW_TREE: answer shadow rays with one kd-tree over all
 *   shadow-casting triangles instead of walking the object tree
 *   (scene_t::isShadowed order); the answers are identical, the walk
 *   differs.  Built at scene creation only when requested.
 * YR_RENDER_EXACT_ORDER: evaluate every object-tree slab test exactly as
 *   bound_t::cross does and walk the reference's object tree for shadow
 *   rays too, so that objects are visited in the reference's order and node
 *   counts match it; by default the object tree uses a conservative
 *   reciprocal-multiply slab test (same hits except between exactly
 *   equidistant objects) and shadow rays walk an SAH BVH over the shadow
 *   casters (same answers; faster). */
#define YR_RENDER_SHADOW_TREE 1u
#define YR_RENDER_EXACT_ORDER 2u
/* YR_RENDER_TONEMAP: every camera sample passes through
 *   color_t::expgam_Adjust(exposure, gamma, clamp_rgb) before the pixel
 *   average (scene.cc:763, 807), as scene_t::render does when the loader
 *   writes a TGA (tonemap(true); HDR / EXR output turns it off).
 * YR_RENDER_CLAMP_RGB: render "clamp_rgb": with TONEMAP, exposure 0 and
 *   gamma 1, each sample is clamped to [0, 1].
 * YR_RENDER_ALPHA_PREMULTIPLY: render "alpha_premultiply": the pixel's RGB
 *   times its alpha (scene.cc:818-822). */
#define YR_RENDER_TONEMAP 4u
#define YR_RENDER_CLAMP_RGB 8u
#define YR_RENDER_ALPHA_PREMULTIPLY 16u
/* Build the meshes' kd-trees on the scene's GPU at yr_scene_create
 * (yr_kdtree_build_gpu; the trees are the host build's). */
#define YR_RENDER_GPU_KD_BUILD 32u

typedef struct yr_object_desc {
    const float *verts;      /* 3*nverts                                       */
    uint32_t nverts;
    const uint32_t *tris;    /* 3*ntris                                        */
    uint32_t ntris;
    uint32_t shader;         /* index into the shader table; YR_PER_TRIANGLE =
                                use tri_shaders (triangle_t::setShader)       */
    uint32_t cast_shadows;   /* object3d_t::castShadows                        */
    const uint32_t *tri_shaders; /* ntris shader indices when shader ==
                                YR_PER_TRIANGLE, else ignored                 */
    const yr_kdtree *tree;   /* optional prebuilt tree (e.g. flattened from
                                YafRay's own kdTree_t); NULL = build here     */
    float smooth_angle;      /* meshObject_t::autoSmooth angle in degrees
                                (mesh.cc:201-279): < 1 flat shading, >= 180
                                one normal per vertex, else per corner over
                                the faces within the angle                    */
    uint32_t reserved;
    const float *instance_matrix; /* non-NULL: this object is a reference to
                                object `instance_of` (referenceObject_t,
                                reference.cc:9-171): that mesh placed by the
                                row-major 4x4 matrix M (16 floats).  Rays are
                                taken into the mesh's space by M's inverse
                                and hits brought back by M (points) and the
                                row-normalised rotation part of M (normals);
                                the geometry fields above are ignored and the
                                shader and shadow flag are the original's.
                                An instance of an instance is refused.      */
    const float *instance_inverse; /* optional M^-1 (16 floats, row-major);
                                NULL = computed here by Gauss-Jordan with
                                exact divisions.  The reference computes it
                                with the shipped build's vectorised division
                                (an approximate reciprocal refined once, whose
                                last bit depends on the CPU: 1/1 gives
                                0.99999994 on x86), so a caller that wants the
                                reference's rays bit for bit passes
                                referenceObject_t::back here.                */
    uint32_t instance_of;
    uint32_t reserved2;
    const float *uvs;        /* optional texture coordinates per triangle: u, v
                                at corners a, b, c (6 floats per triangle, the
                                mesh's facesuv); NULL = none.  The hit's (u, v)
                                is their barycentric blend (triangle_t::
                                getSurface, triangle.cc:156-160); without
                                them it is (-1, -1) on a flat mesh and (0, 0)
                                on a smoothed one, as the reference's          */
    const float *orco_matrix; /* optional 4x4 row-major matrix (16 floats, row
                                3 unused) giving the "orco" texture point of
                                this mesh as orco_matrix * P: a mesh that went
                                through meshObject_t::transform (every mesh
                                the loader or yafrayInterface_t makes, even
                                with an identity transform) has
                                toObjectOrco(P) = backOrco * P (mesh.cc:
                                422-515), backOrco mapping the mesh's bound
                                onto [-1, 1]^3.  The reference inverts it with
                                the shipped build's approximate division, so
                                the caller passes meshObject_t::backOrco
                                itself.  NULL = the point itself (a mesh made
                                without a transform, mesh.cc:510-514); a
                                reference applies its original's matrix to
                                M^-1 P (reference.cc:102-106)                 */
} yr_object_desc;

#define YR_PER_TRIANGLE 0xffffffffu

typedef struct yr_scene_desc {
    const yr_object_desc *objects;
    uint32_t nobjects;
    const yr_shader_desc *shaders;
    uint32_t nshaders;
    const yr_light_desc *lights;
    uint32_t nlights;
    yr_camera_desc camera;
    yr_render_params render;
} yr_scene_desc;

typedef struct yr_scene yr_scene;

/* Upload the scene to `device`: builds missing kd-trees and the object tree
 * (buildObjectTree, object3d.cc:30-53) on the host, flattens them, copies
 * triangles as {a,Nx},{b,Ny},{c,Nz} float4 triples.  The library owns the
 * device copies; yr_scene_destroy frees them. */
YR_API yr_status yr_scene_create(const yr_scene_desc *desc, int device, yr_scene **out);
YR_API yr_status yr_scene_destroy(yr_scene *scene);
/* Host-side statistics of the uploaded scene. */
typedef struct yr_scene_info {
    uint32_t nobjects, ntriangles, nnodes, nprims, nlights;
    uint64_t device_bytes;
    double build_seconds;    /* host kd-tree + object-tree build time         */
} yr_scene_info;
YR_API yr_status yr_scene_info_get(const yr_scene *scene, yr_scene_info *info);
/* Replace the colour parameters of the shaders / lights without a rebuild
 * (used by the inverse-rendering loop). */
YR_API yr_status yr_scene_set_params(yr_scene *scene, const yr_shader_desc *shaders,
                                     const yr_light_desc *lights);
/* Set the camera from a constructed camera_t's own vectors instead of its
 * constructor arguments (a host that holds a camera_t, as a scene_t
 * subclass does with render_camera, has no look / up points to give):
 * position, vto, vup, vright as camera_t's constructor leaves them
 * (camera.cc:27-87, CM_PERSPECTIVE); camera rays are then
 * normalize(vto + vright*px + vup*py) from pos (camera_t::shootRay,
 * camera.cc:184-188).  The resolution stays yr_camera_desc's.  Replaces
 * the camera yr_scene_create derived from yr_camera_desc; call it before
 * rendering (batched renders captured earlier keep the old camera, so they
 * are re-captured). */
YR_API yr_status yr_scene_set_camera_vectors(yr_scene *scene, const float *pos, const float *vto,
                                             const float *vup, const float *vright);

/* ------------------------------------------------------------------------
 * Ray queries (device pointers, asynchronous on `stream`).
 * ------------------------------------------------------------------------ */
typedef struct yr_ray {
    float org[3];
    float tmax;              /* "dis": <0 means infinity (mesh.cc:529)        */
    float dir[3];            /* unit direction                                 */
    uint32_t flags;          /* reserved, 0                                    */
} yr_ray;

typedef struct yr_hit {
    float t;                 /* surfacePoint_t::Z()                            */
    uint32_t object;         /* 0xffffffff = miss                              */
    uint32_t triangle;       /* object-local triangle index                   */
    uint32_t nodes_visited;  /* kd nodes + object-tree nodes touched          */
} yr_hit;

/* Closest hit over all objects: scene_t::firstHit (scene.cc:688-721):
 * origin moved by dir*MIN_RAYDIST, objects front to back through the object
 * tree, each object's kdTree_t::Intersect (kdtree.cc:591-727), Z > 0.
 * `shadow_only` = 1 skips objects that do not cast shadows (firstHit's
 * shadow argument). */
YR_API yr_status yr_trace_closest(yr_scene *scene, const yr_ray *rays, uint32_t n,
                                  yr_hit *hits, int shadow_only, void *stream);

typedef struct yr_shadow_ray {
    float p[3];              /* shading point sp.P()                           */
    uint32_t object;         /* sp.getObject() (for the self_bias rule)        */
    float l[3];              /* light point, or direction if flags&1          */
    uint32_t flags;          /* bit0: l is a direction (isShadowed(dir))       */
} yr_shadow_ray;

/* scene_t::isShadowed (scene.cc:107-185): origin p+dir*self_bias for the
 * point's own object, p+dir*MIN_RAYDIST for the others, any hit with
 * 0 < t < |l-p| via kdTree_t::IntersectS (kdtree.cc:730-866). */
YR_API yr_status yr_trace_shadow(yr_scene *scene, const yr_shadow_ray *rays, uint32_t n,
                                 uint8_t *occluded, void *stream);

/* ------------------------------------------------------------------------
 * Rendering.
 * ------------------------------------------------------------------------ */
/* Kernel classes reported in yr_render_stats (per-class arrays). */
enum {
    YR_K_PRIMARY = 0,        /* camera rays + closest hit                     */
    YR_K_SHADE_CAMERA = 1,   /* light sampling at camera hits                 */
    YR_K_SHADOW = 2,         /* shadow-ray queue traversal (any hit)          */
    YR_K_GATHER = 3,         /* per-vertex light sums                         */
    YR_K_BOUNCE = 4,         /* bounce-ray queue traversal (closest hit)      */
    YR_K_SHADE_PATH = 5,     /* light sampling at bounce vertices            */
    YR_K_OTHER = 6,          /* finish, queue bookkeeping                     */
    YR_K_COUNT = 8
};

typedef struct yr_render_stats {
    uint64_t rays_primary;
    uint64_t rays_shadow;
    uint64_t rays_bounce;
    double ms;               /* device time of the render (CUDA events)      */
    /* input: nonzero = time every kernel class with CUDA events and count
     * kd nodes / triangle tests per class (costs a few microseconds per
     * launch) */
    uint32_t want_kernel_stats;
    uint32_t reserved;
    double kernel_ms[YR_K_COUNT];        /* summed event time per class       */
    uint32_t kernel_launches[YR_K_COUNT];
    uint64_t kernel_rays[YR_K_COUNT];    /* rays traversed per class          */
    uint64_t kernel_nodes[YR_K_COUNT];   /* kd + object-tree nodes visited    */
    uint64_t kernel_tests[YR_K_COUNT];   /* ray-triangle tests                */
} yr_render_stats;

/* Render the whole image: RGBA float, resy rows of resx pixels, row 0 at the
 * top (colorOutput_t::putPixel(x, y) order).  `rgba` is a device pointer
 * unless `rgba_on_host` != 0, in which case the library stages it.
 * QMC: path, hemi and area-light samples use explicit Halton indices with a
 * per-pixel Cranley-Patterson rotation instead of the reference's
 * sequential generator state.  halton(b, n) is the value that
 * Halton::setStart(n) followed by getNext() returns (mcqmc.h:24-49);
 * rot(pixel, dim) in [0,1) is a 32-bit hash of (seed, pixel, dim); a
 * rotated value is u = halton + rot, minus 1 when u >= 1.  For camera
 * sample s of a pixel, path sample i of P per camera sample:
 *   bounce level l direction: bases (prime[2l], prime[2l+1]), index s*P+i,
 *     dims (2l, 2l+1) (pathtools.cc:9-43);
 *   area / hemi light k at path vertex v (0 = camera hit), sample j of J:
 *     bases (2, 3), index m*J+j with m = s at the camera hit and s*P+i on
 *     a path, dims 64+16k+2v (+1); area jitter = u - 0.5 along the cell
 *     axes (arealight.cc:136-153). */
YR_API yr_status yr_render(yr_scene *scene, float *rgba, int rgba_on_host,
                           yr_render_stats *stats, void *stream);

/* yr_render for callers that cannot allocate GPU memory at render time -
 * for example a renderer plugin loaded into an application that owns all
 * of the GPU's memory through its own allocator and forbids its plugins to
 * call cudaMalloc / cudaFree, or a host that has reserved every byte of the
 * device for itself before the render starts.  It renders the same image
 * as yr_render but draws its scratch from one fixed 64 MiB block that every
 * GPU loading this library holds until the process exits, instead of
 * allocating.
 * (No counterpart in the reference: YafRay renders on the CPU.)
 *   - `rgba` is a device pointer (resx*resy*4 floats); nothing is staged.
 *   - The render runs in as many passes as the block needs; a render whose
 *     single pixel (all its samples) needs more than the block fails with
 *     YR_ERR_TOO_LARGE.
 *   - The first call on a device looks the block's address up (once per
 *     device, with that device current); make that first call before any
 *     stream capture.
 *   - All calls share the block and it keeps the last call's contents:
 *     calls that overlap on the GPU (different streams or threads) race and
 *     must be serialized by the caller.
 *   - No CUDA events are created: stats->ms and the kernel times stay 0;
 *     the ray counts are filled in.
 *   - Like yr_render, the call waits for `stream` before it returns (it
 *     reads the render's device status word back). */
YR_API yr_status yr_render_noalloc(yr_scene *scene, float *rgba, yr_render_stats *stats, void *stream);

/* Progressive render with cancellation - the output side of YafRay's
 * block loop, where each finished block goes through colorOutput_t::putPixel
 * and a putPixel that returns false stops the render (renderblock.cc:8-20,
 * threadedscene.cc:186-197).  The frame is rendered wave by wave (waves of
 * at most `wave_pixels` pixels, 0 = as large as the scratch budget allows);
 * after each wave its pixels are in the HOST image `rgba` (resx*resy*4
 * floats) and `on_pixels(user, first, count)` is called with them: region
 * pixels first .. first+count-1 in row-major order of the render region
 * (region pixel k is (x0 + k % w, y0 + k / w); the whole image when no
 * region is set).  Returning 0 from on_pixels stops the render after that
 * wave and the call returns YR_ERR_CANCELLED; pixels not delivered keep the
 * buffer's previous content (pixels outside the region are 0).  The image
 * of a render that runs to the end is yr_render's; stats carry the rays of
 * the waves rendered (no event timing).  The call returns when the last
 * wave is delivered. */
typedef int (*yr_pixels_fn)(void *user, uint32_t first, uint32_t count);
YR_API yr_status yr_render_progressive(yr_scene *scene, float *rgba, uint32_t wave_pixels, yr_pixels_fn on_pixels,
                                       void *user, yr_render_stats *stats, void *stream);

/* Render `count` independent scenes (one device) as one launch.  Two
 * schedules, both giving each scene exactly yr_render's image:
 *   YR_BATCH_TILES: one persistent kernel; work items are tiles of whole
 *     pixels of one scene, pulled from a shared counter, and each block runs
 *     the render stages over its tile with block-local ray queues;
 *   YR_BATCH_WAVES: every scene's own wavefront (per-scene ray queues, the
 *     kernels of yr_render) on one of `streams` concurrent streams, the
 *     whole batch captured as one CUDA graph.
 * outs[i]: device RGBA float image of scene i (its resx*resy*4 floats).
 * params (in/out, may be NULL = all automatic): mode 0 and block_size /
 * queue_tile / streams 0 = autotuned the first time this list of scenes is
 * rendered (timed on the device, then cached); use_graph = capture the
 * launch in a CUDA graph and replay it on later calls (the waves schedule
 * always uses a graph).  On return the fields hold the configuration used.
 * Stats: ray counts and the device time of the launch. */
enum { YR_BATCH_AUTO = 0, YR_BATCH_TILES = 1, YR_BATCH_WAVES = 2 };
typedef struct yr_batch_params {
    int32_t block_size;      /* tiles: threads per block, 0 = autotuned       */
    int32_t queue_tile;      /* tiles: camera samples per item, 0 = autotuned */
    int32_t use_graph;       /* capture the launch in a CUDA graph            */
    int32_t stack_entries;   /* out: kd stack capacity of the kernel used     */
    int32_t mode;            /* YR_BATCH_*                                    */
    int32_t streams;         /* waves: concurrent streams, 0 = autotuned      */
} yr_batch_params;

YR_API yr_status yr_render_batch(yr_scene *const *scenes, uint32_t count, float *const *outs,
                                 yr_batch_params *params, yr_render_stats *stats, void *stream);

/* ------------------------------------------------------------------------
 * Adjoint.  Gradient of  L = sum_pixels w * |img - target|^2  ... see
 * yr_backward_desc.  Parameter vector layout, per scene:
 *   for each shader s: color[3], specular weight (the scalar that scales
 *   "specular"), tex amplitude (tex_intensity: musgrave and voronoi
 *   textures; its gradient is 0 for the others), tex base colour
 *   (tex_color1[3]; gradient 0 for voronoi, whose colour does not use it)
 *   for each light l: power
 * ------------------------------------------------------------------------ */
typedef struct yr_backward_desc {
    const float *target;     /* device RGBA target image                      */
    const float *image;      /* device RGBA forward image (from yr_render)    */
    float loss_scale;        /* L = loss_scale * sum (img-target)^2 over RGB  */
    uint32_t reserved;
} yr_backward_desc;

/* Number of floats in the parameter vector of `scene`. */
YR_API uint32_t yr_param_count(const yr_scene *scene);
/* Gather the current parameters into `params` (host pointer). */
YR_API yr_status yr_params_get(const yr_scene *scene, float *params);
/* Scatter `params` (host pointer) into the scene's shaders and lights. */
YR_API yr_status yr_params_set(yr_scene *scene, const float *params);
/* dparams: device pointer, yr_param_count floats, overwritten. */
YR_API yr_status yr_backward(yr_scene *scene, const yr_backward_desc *desc, float *dparams,
                             float *loss_out, void *stream);

/* One optimisation step of `count` independent scenes (one device) as one
 * CUDA graph: scene i is rendered into descs[i].image (device RGBA, written
 * here), then its gradient goes to dparams[i] (device, yr_param_count
 * floats) and its loss to losses[i] (host, may be NULL).  The scenes run
 * as per-scene wavefronts on `streams` concurrent streams (0 = 8).  The
 * graph is captured on the first call for a list of scenes and buffers and
 * replayed while they stay the same; parameters changed with
 * yr_params_set are picked up.  Results equal yr_render + yr_backward per
 * scene.  (No counterpart in the reference.) */
YR_API yr_status yr_backward_batch(yr_scene *const *scenes, uint32_t count, const yr_backward_desc *descs,
                                   float *const *dparams, float *losses, int32_t streams, void *stream);

/* ------------------------------------------------------------------------
 * Image outputs (host).  A rendered RGBA float image (row-major, top row
 * first, as yr_render writes it) encoded byte for byte as YafRay's
 * colorOutput_t writers encode the same pixels:
 *   YR_IMAGE_TGA: outTga_t (targaIO.cc:37-130), 24-bit BGR, or 32-bit BGRA
 *     with YR_IMAGE_ALPHA (the loader's save_alpha);
 *   YR_IMAGE_HDR: outHDR_t (HDR_io.cc:34-160), Radiance RGBE with
 *     run-length scanlines; alpha is not stored.
 * The loader renders a TGA with the per-sample tone map on
 * (YR_RENDER_TONEMAP) and an HDR with it off.
 * ------------------------------------------------------------------------ */
enum { YR_IMAGE_TGA = 0, YR_IMAGE_HDR = 1 };
#define YR_IMAGE_ALPHA 1u

/* Encode into `out` (host, `capacity` bytes); `size` receives the encoded
 * size.  With out == NULL only the size is returned. */
YR_API yr_status yr_image_encode(int32_t format, const float *rgba, int32_t width, int32_t height, int32_t flags,
                                 uint8_t *out, size_t capacity, size_t *size);
/* Encode and write to the file `path`. */
YR_API yr_status yr_image_write(const char *path, int32_t format, const float *rgba, int32_t width, int32_t height,
                                int32_t flags);

#ifdef __cplusplus
}
#endif
#endif /* YR_H */
