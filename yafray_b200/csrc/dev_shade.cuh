// Shading on the device: explicit-index Halton QMC with per-pixel
// Cranley-Patterson rotation, improved Perlin noise / fBm / turbulence,
// genericShader_t with its texture modulator, and the per-sample parts of
// the point, area, hemi and path lights.
#pragma once
#include "dev_common.cuh"
#include "scene.h"

namespace yr {

// ------------------------------------------------------------------ QMC
// Halton::setStart(n) followed by Halton::getNext() (mcqmc.h:24-49), i.e.
// the radical inverse of n+1, as the shipped build evaluates it
// (fast-math: r = (1 - 1e-10) - value, value = (hh + h) + (value - 1)).
// Halton::getNext from the radical inverse `value` of n (mcqmc.h:33-49)
__device__ __forceinline__ float halton_next(double value, double inv) {
    const double r = (1.0 - 0.0000000001) - value;
    if (inv < r) {
        value = value + inv;
    } else {
        double hh, h = inv;
        do {
            hh = h;
            h *= inv;
        } while (h >= r);
        value = (hh + h) + (value - 1.0);
    }
    return (float)value;
}

// Halton::setStart's radical inverse (mcqmc.h:24-31) for a base known at
// compile time (the divisions become multiplications)
template <uint32_t B>
__device__ __forceinline__ float halton_b(uint32_t n) {
    constexpr double inv = 1.0 / (double)B;
    double value = 0.0;
    if (B == 2) {
        // every term is a power of two below 2^-32 apart: the sum is exact,
        // and equals the bit-reversed index times 2^-32
        value = (double)__brev(n) * 0x1p-32;
    } else {
        double factor = inv;
        uint32_t i = n;
        while (i > 0) {
            value += (double)(i % B) * factor;
            i /= B;
            factor *= inv;
        }
    }
    return halton_next(value, inv);
}

__device__ __forceinline__ float halton(uint32_t base, uint32_t n) {
    switch (base) {
    case 2: return halton_b<2>(n);
    case 3: return halton_b<3>(n);
    case 5: return halton_b<5>(n);
    case 7: return halton_b<7>(n);
    default: break;
    }
    const double inv = 1.0 / (double)base;
    double value = 0.0, factor = inv;
    uint32_t i = n;
    while (i > 0) {
        value += (double)(i % base) * factor;
        i /= base;
        factor *= inv;
    }
    return halton_next(value, inv);
}

__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// Cranley-Patterson rotation offset of (pixel, dimension) in [0,1).
__host__ __device__ __forceinline__ float cp_rot(uint32_t seed, uint32_t pixel, uint32_t dim) {
    uint32_t h = fmix32(seed * 0x9e3779b9u + 0x632be5abu);
    h = fmix32(h ^ (pixel * 0x85ebca77u));
    h = fmix32(h ^ (dim * 0xc2b2ae3du + 0x27d4eb2fu));
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

__host__ __device__ __forceinline__ float cp_add(float v, float r) {
    float u = v + r;
    if (u >= 1.0f) u -= 1.0f;
    return u;
}

__device__ __constant__ uint32_t kPrimes[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};

// QMC dimensions: path level l uses dims (2l, 2l+1) with the l-th pair of
// primes (pathtools.cc:9-19); light k at vertex v uses dims 64+16k+2v (+1)
// with bases 2 and 3.
__device__ __forceinline__ uint32_t light_dim(int k, int v) { return 64u + 16u * (uint32_t)k + 2u * (uint32_t)v; }

// ---------------------------------------------------------------- noise
// The 256-entry permutation of Blender's noise (the first half of hash[512]
// in noise.cc:118-127; the second half repeats it), indexed modulo 256.
__device__ const uint8_t kPerm[256] = {
    162, 160,  25,  59, 248, 235, 170, 238, 243,  28, 103,  40,  29, 237,   0, 222,
    149,  46, 220,  63,  58, 130,  53,  77, 108, 186,  54, 208, 246,  12, 121,  50,
    209,  89, 244,   8, 139,  99, 137,  47, 184, 180, 151, 131, 242, 143,  24, 199,
     81,  20, 101, 135,  72,  32,  66, 168, 128, 181,  64,  19, 178,  34, 126,  87,
    188, 127, 107, 157, 134,  76, 200, 219, 124, 213,  37,  78,  90,  85, 116,  80,
    205, 179, 122, 187, 195, 203, 182, 226, 228, 236, 253, 152,  11, 150, 211, 158,
     92, 161, 100, 241, 129,  97, 225, 196,  36, 114,  73, 140, 144,  75, 132,  52,
     56, 171, 120, 202,  31,   1, 215, 147,  17, 193,  88, 169,  49, 249,  68, 109,
    191,  51, 156,  95,   9, 148, 163, 133,   6, 198, 154,  30, 123,  70,  21,  48,
     39,  43,  27, 113,  60,  91, 214, 111,  98, 172,  79, 194, 192,  14, 177,  35,
    167, 223,  71, 176, 119, 105,   5, 233, 230, 231, 118, 115,  15, 254, 110, 155,
     86, 239,  18, 165,  55, 252, 174, 217,   3, 142, 221,  16, 185, 206, 201, 141,
    218,  42, 189, 104,  23, 159, 190, 212,  10, 204, 210, 232,  67,  61, 112, 183,
      2, 125, 153, 216,  13,  96, 138,   4,  44,  62, 146, 229, 175,  83,   7, 224,
     41, 166, 197, 227, 245, 247,  74,  65,  38, 106,  22,  94,  82,  45,  33, 173,
    240, 145, 255, 234,  84, 250, 102,  26,  69,  57, 207, 117, 164, 136, 251,  93,};

__device__ __forceinline__ int perm(int i) { return (int)__ldg(&kPerm[i & 255]); }

// the two signed terms of newPerlin_t::grad (noise.h:33-39)
__device__ __forceinline__ void grad_parts(int hash, float x, float y, float z, float &U, float &V) {
    const int h = hash & 15;
    const float u = h < 8 ? x : y, v = h < 4 ? y : (h == 12 || h == 14 ? x : z);
    U = (h & 1) == 0 ? u : -u;
    V = (h & 2) == 0 ? v : -v;
}

// newPerlin_t::operator() (noise.cc:161-183): improved Perlin noise in
// [0,1], as the shipped build (-O3 -ffast-math) evaluates it: every grad()
// split into its two signed terms per cube corner and the three lerps
// regrouped into the sum below, in the order of operations of the
// compiler's optimized tree of noise.cc (bit-identical to the reference).
__device__ __forceinline__ float perlin(const V3 &pt) {
    const float px = pt.x, py = pt.y, pz = pt.z;
    const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
    const int X = ((int)fx) & 255, Y = ((int)fy) & 255, Z = ((int)fz) & 255;
    const float x = px - fx, y = py - fy, z = pz - fz;
    const float x1 = x - 1.f, y1 = y - 1.f, z1 = z - 1.f;
    const int A = perm(X) + Y, AA = perm(A) + Z, AB = perm(A + 1) + Z;
    const int B = perm(X + 1) + Y, BA = perm(B) + Z, BB = perm(B + 1) + Z;
    float U_aa, V_aa, U_ba, V_ba, U_ab, V_ab, U_bb, V_bb, U_aa1, V_aa1, U_ba1, V_ba1, U_ab1, V_ab1, U_bb1, V_bb1;
    grad_parts(perm(AA), x, y, z, U_aa, V_aa);
    grad_parts(perm(BA), x1, y, z, U_ba, V_ba);
    grad_parts(perm(AB), x, y1, z, U_ab, V_ab);
    grad_parts(perm(BB), x1, y1, z, U_bb, V_bb);
    grad_parts(perm(AA + 1), x, y, z1, U_aa1, V_aa1);
    grad_parts(perm(BA + 1), x1, y, z1, U_ba1, V_ba1);
    grad_parts(perm(AB + 1), x, y1, z1, U_ab1, V_ab1);
    grad_parts(perm(BB + 1), x1, y1, z1, U_bb1, V_bb1);
    const float t283 = x * x;
    const float t293 = y * y;
    const float t348 = x * 6.f;
    const float t349 = t348 - 15.f;
    const float t350 = x * t349;
    const float t351 = t350 + 10.f;
    const float t282 = x * t351;
    const float t352 = t282 * t283;
    const float t341 = y * 6.f;
    const float t342 = t341 - 15.f;
    const float t343 = y * t342;
    const float t344 = t343 + 10.f;
    const float t292 = y * t344;
    const float t345 = t292 * t293;
    const float t334 = z * 6.f;
    const float t335 = t334 - 15.f;
    const float t336 = z * t335;
    const float t337 = t336 + 10.f;
    const float t485 = U_aa + V_aa;
    const float t528 = U_ba - U_aa;
    const float t527 = V_ba + t528;
    const float t25 = t527 - V_aa;
    const float t26 = t25 * t352;
    const float t390 = U_ab + t528;
    const float t310 = U_bb + V_bb;
    const float t304 = V_aa - V_ab;
    const float t512 = U_aa - U_ba;
    const float t311 = t512 - U_ab;
    const float t303 = t310 + t311;
    const float t294 = t304 - V_ba;
    const float t504 = t294 + t303;
    const float t505 = t352 * t504;
    const float t321 = V_ab + t505;
    const float t322 = U_ab - U_aa;
    const float t312 = t321 + t322;
    const float t40 = t312 - V_aa;
    const float t41 = t40 * t345;
    const float t483 = t26 + t41;
    const float t477 = t483 + t485;
    const float t452 = U_ba1 + V_ba1;
    const float t458 = t512 - U_aa1;
    const float t440 = t452 + t458;
    const float t386 = U_bb1 + V_bb1;
    const float t381 = V_aa1 - V_ab1;
    const float t281 = U_ab1 + U_ba1;
    const float t383 = t386 - t281;
    const float t411 = U_ab1 - U_aa1;
    const float t410 = V_ab1 - V_aa1;
    const float t407 = V_aa + t410;
    const float t380 = V_ba - V_ba1;
    const float t346 = t380 + t381;
    const float t340 = V_ab - V_aa;
    const float t389 = U_aa1 - U_bb;
    const float t384 = t389 + t390;
    const float t347 = t383 + t384;
    const float t339 = t346 + t347;
    const float t323 = t340 - V_bb;
    const float t416 = t323 + t339;
    const float t414 = t352 * t416;
    const float t413 = U_aa - U_ab;
    const float t408 = t411 + t413;
    const float t404 = t407 + t408;
    const float t405 = t414 - V_ab;
    const float t425 = t404 + t405;
    const float t426 = t345 * t425;
    const float t466 = V_aa1 + t426;
    const float t442 = V_aa - V_aa1;
    const float t434 = t442 - V_ba;
    const float t427 = t434 + t440;
    const float t428 = t352 * t427;
    const float t468 = U_aa1 - U_aa;
    const float t464 = t466 + t468;
    const float t460 = t428 - V_aa;
    const float t83 = t460 + t464;
    const float tpowmult276 = z * z;
    const float tpowmult284 = z * tpowmult276;
    const float t489 = tpowmult284 * t337;
    const float t84 = t83 * t489;
    const float tnv123 = t84 + t477;
    return (float)(((double)tnv123 + 1.0) * 0.5);
}

// fBm_t::operator() (noise.cc:638-650) over newPerlin with getSignedNoise
// (noise.h:245-248).  pwHL = lacunarity^-H.
__device__ __forceinline__ float fbm(V3 tp, float H, float lacunarity, float octaves) {
    float value = 0, pwr = 1;
    const float pwHL = (float)pow((double)lacunarity, (double)-H);
    for (int i = 0; i < (int)octaves; i++) {
        value += ((float)2.0 * perlin(tp) - (float)1.0) * pwr;
        pwr *= pwHL;
        tp = V3{tp.x * lacunarity, tp.y * lacunarity, tp.z * lacunarity};
    }
    const float rmd = octaves - floorf(octaves);
    if (rmd != 0.f) value += rmd * ((float)2.0 * perlin(tp) - (float)1.0) * pwr;
    return value;
}

// turbulence (noise.cc:808-819), newPerlin (no offset)
__device__ __forceinline__ float turbulence(const V3 &pt, int oct, float size, bool hard) {
    float amp = 1, sum = 0;
    V3 tp = V3{pt.x * size, pt.y * size, pt.z * size};
    for (int i = 0; i <= oct; i++, amp *= 0.5f, tp = V3{tp.x * 2.0f, tp.y * 2.0f, tp.z * 2.0f}) {
        float val = perlin(tp);
        if (hard) val = (float)fabs(2.0 * (double)val - 1.0);
        sum += amp * val;
    }
    return sum * ((float)(1 << oct) / (float)((1 << (oct + 1)) - 1));
}

}  // namespace yr

#include "dev_tex.cuh"

namespace yr {

// --------------------------------------------------------------- shading
struct Surf {
    V3 P, N, Ng, NU, NV;
    V3 orco;  // the texture's "orco" point: P, or M^-1 P on a reference
    int object;
    int shader;
    float Z;
    float sx, sy;  // screen position of the camera sample (camera hits; 0 at path vertices)
    float u, v;    // texture coordinates (triangle_t::getSurface)
};

// createCS (vector3d.h:240-258)
__device__ __forceinline__ void create_cs(const V3 &N, V3 &u, V3 &v) {
    if ((N.x == 0.f) && (N.y == 0.f)) {
        u = (N.z < 0.f) ? v3(-1.f, 0.f, 0.f) : v3(1.f, 0.f, 0.f);
        v = v3(0.f, 1.f, 0.f);
    } else {
        const float d = (float)(1.0 / sqrt((double)(N.y * N.y + N.x * N.x)));
        u = v3(N.y * d, -N.x * d, 0.f);
        v = cross(N, u);
    }
}

// FACE_FORWARD(Ng, N, I) (shader.h:157)
__device__ __forceinline__ V3 face_forward(const V3 &Ng, const V3 &N, const V3 &I) {
    return (dot(Ng, I) < 0.f) ? -N : N;
}

// reflect (vector3d.h:221-226)
__device__ __forceinline__ V3 reflect(const V3 &n, const V3 &v) {
    const float vn = dot(v, n);
    if (vn < 0.f) return -v;
    return (2 * vn) * n - v;
}

// meshObject_t::shoot + triangle_t::getSurface (mesh.cc:570-576,
// triangle.cc:138-207): P = from + Z*ray; N = Ng for a flat triangle, else
// the corner normals interpolated at P (getInterpolation's dominant-axis
// barycentrics) and normalized.  The shipped build evaluates the
// interpolation as r = 1/denum, fb = alpha r, fc = beta r,
// fa = 1 - (alpha + beta) r, and the sum as na fa + (nb fb + nc fc).
__device__ __forceinline__ Surf make_surface(const DevScene &S, const DevRender &R, int object, uint32_t tri,
                                             float Z, const V3 &from_w, const V3 &ray_w) {
    Surf s;
    s.sx = s.sy = 0.f;
    // a reference's hit is formed in its original's space (the ray taken
    // there by M's inverse) and brought back below (reference.cc:100-112)
    const int inst = S.objects[object].inst;
    const DevInst *I = inst >= 0 ? S.insts + inst : nullptr;
    const V3 from = I ? xf_point(I->back, from_w) : from_w;
    const V3 ray = I ? xf_vec(I->back, ray_w) : ray_w;
    s.P = from + Z * ray;
    const float4 p = __ldg(S.tris + 3 * (size_t)tri), q = __ldg(S.tris + 3 * (size_t)tri + 1),
                 r = __ldg(S.tris + 3 * (size_t)tri + 2);
    s.Ng = v3(p.w, q.w, r.w);
    s.N = s.Ng;
    // without texture coordinates or corner normals getSurface returns
    // u = v = -1 at once; otherwise the coordinates' barycentric blend, or 0
    // without any (triangle.cc:138-160)
    const uint32_t oflags = S.objects[object].flags;
    s.u = s.v = (oflags & 6u) ? 0.f : -1.f;
    if (oflags & 6u) {
        const V3 a = v3(p.x, p.y, p.z), b = v3(q.x, q.y, q.z), c = v3(r.x, r.y, r.z), &h = s.P;
        const float nx = fabsf(s.Ng.x), ny = fabsf(s.Ng.y), nz = fabsf(s.Ng.z);
        float uu0, vv0, uu1, vv1, uu2, vv2;
        if (nx >= ny && nx >= nz) {
            uu0 = h.y - a.y; vv0 = h.z - a.z; uu1 = b.y - a.y; vv1 = b.z - a.z; uu2 = c.y - a.y; vv2 = c.z - a.z;
        } else if (ny >= nx && ny >= nz) {
            uu0 = h.x - a.x; vv0 = h.z - a.z; uu1 = b.x - a.x; vv1 = b.z - a.z; uu2 = c.x - a.x; vv2 = c.z - a.z;
        } else {
            uu0 = h.x - a.x; vv0 = h.y - a.y; uu1 = b.x - a.x; vv1 = b.y - a.y; uu2 = c.x - a.x; vv2 = c.y - a.y;
        }
        const float alpha = uu0 * vv2 - vv0 * uu2;
        const float beta = uu1 * vv0 - vv1 * uu0;
        const float denum = uu1 * vv2 - vv1 * uu2;
        const float rd = 1.f / denum;
        const float fb = alpha * rd, fc = beta * rd, fa = 1.f - (alpha + beta) * rd;
        if (oflags & 2u) {
            const float *cn = S.tri_nrm + 9 * (size_t)tri;
            const V3 nn = v3(__ldg(cn + 0) * fa + (__ldg(cn + 3) * fb + __ldg(cn + 6) * fc),
                             __ldg(cn + 1) * fa + (__ldg(cn + 4) * fb + __ldg(cn + 7) * fc),
                             __ldg(cn + 2) * fa + (__ldg(cn + 5) * fb + __ldg(cn + 8) * fc));
            s.N = normalize(nn);
        }
        if (oflags & 4u) {
            const float *uv = S.tri_uv + 6 * (size_t)tri;
            s.u = __ldg(uv + 0) * fa + (__ldg(uv + 2) * fb + __ldg(uv + 4) * fc);
            s.v = __ldg(uv + 1) * fa + (__ldg(uv + 3) * fb + __ldg(uv + 5) * fc);
        }
    }
    create_cs(s.N, s.NU, s.NV);
    s.orco = s.P;
    if (I) {  // N, Ng, NU, NV by MRot; P by M; orco = M^-1 P (toObjectOrco)
        s.N = rot_vec(I->rot, s.N);
        s.Ng = rot_vec(I->rot, s.Ng);
        s.P = xf_point(I->m, s.P);
        s.NU = rot_vec(I->rot, s.NU);
        s.NV = rot_vec(I->rot, s.NV);
        s.orco = xf_point(I->back, s.P);
    }
    const int om = S.objects[object].orco;
    if (om >= 0) {  // a transformed mesh: toObjectOrco = backOrco * point (mesh.cc:510-515)
        const float4 r0 = __ldg(S.orco_m + 3 * om), r1 = __ldg(S.orco_m + 3 * om + 1), r2 = __ldg(S.orco_m + 3 * om + 2);
        const float m[12] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w};
        s.orco = xf_point(m, s.orco);
    }
    s.object = object;
    s.shader = (int)__ldg(R.tri_shader + tri);
    s.Z = Z;
    return s;
}

// Texture point of the procedural path of modulator_t::doMapping
// (texture.cc:122-320): the texco source (hit point, orco point, shading
// normal, screen position, or the eye reflected about the face-forwarded
// normal), then per axis size*(source[proj] + ofs), or size*ofs when the
// axis is switched off.  `eye`: the direction the shading call looks from.
__device__ __forceinline__ V3 tex_point(const DevShader &sh, const Surf &sp, const V3 &eye) {
    V3 src = sh.texco == YR_TEXCO_NORMAL ? sp.N : (sh.texco == YR_TEXCO_ORCO ? sp.orco : sp.P);
    if (sh.texco == YR_TEXCO_WINDOW) src = v3(sp.sx, sp.sy, 0.f);
    if (sh.texco == YR_TEXCO_UV) src = v3((float)((double)sp.u * 2.0 - 1.0), (float)(1.0 - (double)sp.v * 2.0), 0.f);
    if (sh.texco == YR_TEXCO_REFLECT) {  // texture.cc:158-165
        const V3 neye = normalize(eye);
        src = reflect(face_forward(sp.Ng, sp.N, neye), neye);
    }
    float t[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int a = sh.proj[k];
        t[k] = a < 0 ? sh.msize[k] * sh.mofs[k] : sh.msize[k] * (comp(src, a) + sh.mofs[k]);
    }
    return v3(t[0], t[1], t[2]);
}

// What the adjoint keeps of a vertex's texture: its colour and the
// colour's derivatives by the texture intensity and by color1.
struct TexDeriv {
    C3 tex;
    C3 dint;
    float dc1;
};

// modulator_t::modulate (texture.cc:499-534), all three channels: the
// diffuse colour C, the specular colour S and the Phong exponent H, each
// by its own weight (a channel whose weight is not above 0 keeps its
// value), in the modulator's mode - mix: C = mix(tex, C, wc), S =
// mix(tex, S, ws), H = f*wh + H*(1-wh); mul: mix(tex, 1, w) * C (S alike),
// H = (f*wh + (1-wh)) * H; add: tex*w + C, f*wh + H; sub: tex*(-w) + C,
// f*(-wh) + H - with tex the texture's colour and f its value (getFloat).
__device__ __forceinline__ void modulated_all(const DevShader *shp, const Surf &sp, const V3 &eye, C3 &C, C3 &S,
                                              float &H) {
    const DevShader &sh = *shp;
    C = sh.color;
    S = sh.specular;
    H = sh.hard;
    if (sh.tex_type == YR_TEX_NONE || !(sh.mod_color > 0.f || sh.mod_spec > 0.f || sh.mod_hard > 0.f)) return;
    const TexEval te = texture_eval(shp, tex_point(sh, sp, eye));
    const C3 tex = te.col;
    const float f = te.f, wc = sh.mod_color, ws = sh.mod_spec, wh = sh.mod_hard;
    const C3 one = c3(1.f, 1.f, 1.f);
    switch (sh.mod_mode) {
    case YR_MOD_MUL:
        if (wc > 0.f) C = (wc > 1.0f ? tex : tex * wc + (1 - wc) * one) * C;
        if (ws > 0.f) S = (ws > 1.0f ? tex : tex * ws + (1 - ws) * one) * S;
        if (wh > 0.f) H = (f * wh + (1 - wh)) * H;
        break;
    case YR_MOD_ADD:
        if (wc > 0.f) C = (tex * wc) + C;
        if (ws > 0.f) S = (tex * ws) + S;
        if (wh > 0.f) H = f * wh + H;
        break;
    case YR_MOD_SUB:
        if (wc > 0.f) C = (tex * -wc) + C;
        if (ws > 0.f) S = (tex * -ws) + S;
        if (wh > 0.f) H = (f * -wh) + H;
        break;
    default:
        if (wc > 0.f) C = wc > 1.0f ? tex : tex * wc + (1 - wc) * C;
        if (ws > 0.f) S = ws > 1.0f ? tex : tex * ws + (1 - ws) * S;
        if (wh > 0.f) H = f * wh + H * (1 - wh);
        break;
    }
}

// modulator_t::modulate (texture.cc:499-534), colour channel: the texture
// colour at the modulator's texture point, mixed into the diffuse colour
// by the modulator's mode - mix: mix(tex, C, w); mul: mix(tex, 1, w) * C;
// add: tex*w + C; sub: tex*(-w) + C, where mix (color.cc:103-109) is
// a*w + (1-w)*b and returns a for w > 1.  `td` (optional) receives what
// the adjoint needs.
// `shp` points at the shader record in device memory.
__device__ __forceinline__ C3 modulated_color(const DevShader *shp, const Surf &sp, const V3 &eye,
                                              TexDeriv *td = nullptr) {
    const DevShader &sh = *shp;
    const C3 C = sh.color;
    if (sh.tex_type == YR_TEX_NONE || !(sh.mod_color > 0.f)) return C;
    if (sh.mod_spec > 0.f || sh.mod_hard > 0.f) {  // one texture evaluation for all three channels
        C3 c, s;
        float h;
        modulated_all(shp, sp, eye, c, s, h);
        return c;
    }
    const TexEval te = texture_eval(shp, tex_point(sh, sp, eye));
    if (td) {
        td->tex = te.col;
        td->dint = te.dint;
        td->dc1 = te.dc1;
    }
    const C3 tex = te.col;
    const float w = sh.mod_color;
    switch (sh.mod_mode) {
    case YR_MOD_MUL: return (w > 1.0f ? tex : tex * w + (1 - w) * c3(1.f, 1.f, 1.f)) * C;
    case YR_MOD_ADD: return (tex * w) + C;
    case YR_MOD_SUB: return (tex * -w) + C;
    default:
        if (w > 1.0f) return tex;
        return tex * w + (1 - w) * C;
    }
}

// The parts of genericShader_t::fromLight (basicshaders.cc:46-70) that
// depend only on the shading point and the eye, computed once per vertex:
// the face-forwarded normal and the reflected eye direction.
struct LitPre {
    V3 N;
    V3 refl;
    bool spec;   // the shader has a specular colour
};

__device__ __forceinline__ LitPre lit_pre(const DevShader &sh, const Surf &sp, const V3 &eye) {
    LitPre L;
    const V3 edir = normalize(eye);
    L.N = face_forward(sp.Ng, sp.N, edir);
    L.refl = reflect(L.N, edir);
    L.spec = sh.specular.r != 0.f || sh.specular.g != 0.f || sh.specular.b != 0.f;
    return L;
}

// genericShader_t::fromLight with edif = 1.  `lkc` is the (modulated)
// diffuse colour.  Without a specular colour the specular term is +0 for
// every light direction (its factors are finite and non-negative), so only
// that +0 is added.
__device__ __forceinline__ C3 from_light(const DevShader &sh, const C3 &lkc, const LitPre &pre, const V3 &ldir,
                                         const C3 &lcol) {
    const float inte = dot(pre.N, ldir);
    if (inte < 0.f) return c3(0.f, 0.f, 0.f);
    const C3 edif_inte = c3(1.f * inte, 1.f * inte, 1.f * inte);
    if (!pre.spec) return ((edif_inte * lcol) * lkc) + c3(0.f, 0.f, 0.f);
    float refle = dot(pre.refl, ldir);
    if (refle < 0.f) refle = 0.f;
    else refle = (float)pow((double)refle, (double)sh.hard);
    return ((edif_inte * lcol) * lkc) + (sh.specular * refle) * lcol;
}

// from_light split into the factor of the diffuse colour (D) and of the
// specular colour (Sp): from_light = D * lkc + specular * Sp.
__device__ __forceinline__ void from_light_parts(const DevShader &sh, const LitPre &pre, const V3 &ldir,
                                                 const C3 &lcol, C3 &D, C3 &Sp) {
    const float inte = dot(pre.N, ldir);
    if (inte < 0.f) {
        D = Sp = c3(0.f, 0.f, 0.f);
        return;
    }
    float refle = dot(pre.refl, ldir);
    if (refle < 0.f) refle = 0.f;
    else refle = (float)pow((double)refle, (double)sh.hard);
    D = inte * lcol;
    Sp = refle * lcol;
}

// haltonSampler_t::nextDirection (pathtools.cc:32-43) for explicit z1, z2
// in [0,1): cosine-weighted direction around N.
__device__ __forceinline__ V3 cos_hemi_dir(const V3 &N, const V3 &Ru, const V3 &Rv, float z1, float z2) {
    if (z1 > 1.0f) z1 = 1.0f;
    z2 = (float)((double)z2 * 6.283185307179586);
    const float c = (float)cos((double)z2), s = (float)sin((double)z2);
    const float s1 = (float)sqrt(1.0 - (double)z1);
    const float s2 = sqrtf(z1);
    return (Ru * c + Rv * s) * s1 + N * s2;
}

// hemiLight_t::getNext (hemilight.cc:103-114): uniform direction
__device__ __forceinline__ V3 uni_hemi_dir(const V3 &N, const V3 &Ru, const V3 &Rv, float z1, float z2) {
    z2 = (float)((double)z2 * 6.283185307179586);
    const float c = (float)cos((double)z2), s = (float)sin((double)z2);
    const float s1 = (float)sqrt(1.0 - (double)(z1 * z1));
    return (Ru * c + Rv * s) * s1 + N * z1;
}

}  // namespace yr
