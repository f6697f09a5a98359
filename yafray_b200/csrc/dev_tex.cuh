// Procedural noise bases and textures of the shading path (noise.cc,
// basictex.cc), in the order of operations of the shipped build
// (-O3 -ffast-math, read from g++'s optimized trees of those files): with
// --fmad=false every value below is bit-identical to the reference's,
// except where a CUDA libm function (sinf, powf, double pow) stands in
// for glibc's.  Included by dev_shade.cuh after the improved Perlin noise.
#pragma once

#include "noise_tables.h"

namespace yr {

// Blender's feature-point offsets (voronoi and cell bases) and gradient
// vectors (blender and standard Perlin bases)
__device__ const float kHashPnt[768] = YR_HASHPNT_INIT;
__device__ const float kHashVect[768] = YR_HASHVECT_INIT;

__device__ __forceinline__ const float *hash_vect(int i) { return kHashVect + 3 * (i & 255); }

// stdPerlin_t::operator() (noise.cc:374-434): t = x + 1e4 in float, corner
// values u = (q0*rx + q1*ry) + q2*rz, each lerp toward v formed as
// ((v0 + v1) + (v2 - u)) * s + u; stdp_p / stdp_g repeat the permutation
// and hashvectf with period 256.
__device__ __forceinline__ float std_perlin(const V3 &pt) {
    const float vec[3] = {pt.x, pt.y, pt.z};
    int b0[3], b1[3];
    float r0[3], r1[3], sv[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float t = vec[k] + 10000.0f;
        const int ti = (int)t;
        b0[k] = ti & 255;
        b1[k] = (b0[k] + 1) & 255;
        r0[k] = t - (float)ti;
        r1[k] = r0[k] - 1.0f;
        sv[k] = (float)((double)(r0[k] * r0[k]) * (3.0 - (double)r0[k] * 2.0));
    }
    const int i = perm(b0[0]), j = perm(b1[0]);
    const int b00 = perm(i + b0[1]), b10 = perm(j + b0[1]), b01 = perm(i + b1[1]), b11 = perm(j + b1[1]);
    auto at = [](int g, float rx, float ry, float rz) {
        const float *q = hash_vect(g);
        return (__ldg(q) * rx + __ldg(q + 1) * ry) + __ldg(q + 2) * rz;
    };
    auto lerp_to = [](int g, float rx, float ry, float rz, float u, float s) {
        const float *q = hash_vect(g);
        return ((__ldg(q) * rx + __ldg(q + 1) * ry) + (__ldg(q + 2) * rz - u)) * s + u;
    };
    const float sx = sv[0], sy = sv[1], sz = sv[2];
    float u = at(b00 + b0[2], r0[0], r0[1], r0[2]);
    const float a0 = lerp_to(b10 + b0[2], r1[0], r0[1], r0[2], u, sx);
    u = at(b01 + b0[2], r0[0], r1[1], r0[2]);
    const float c0 = lerp_to(b11 + b0[2], r1[0], r1[1], r0[2], u, sx);
    const float c = (c0 - a0) * sy + a0;
    u = at(b00 + b1[2], r0[0], r0[1], r1[2]);
    const float a1 = lerp_to(b10 + b1[2], r1[0], r0[1], r1[2], u, sx);
    u = at(b01 + b1[2], r0[0], r1[1], r1[2]);
    const float c1 = lerp_to(b11 + b1[2], r1[0], r1[1], r1[2], u, sx);
    const float d = (c1 - a1) * sy + a1;
    return (float)((double)((d - c) * sz + c) * 0.75 + 0.5);
}

// blenderNoise_t::operator() (noise.cc:439-510): corner weights in double
// as x*x*(2x - 3) + 1 and 1 - x*x*(2x + 3); the four corners of each z
// layer summed as ((v0 + v2) + (v1 + v3)) and scaled once by the layer's
// z weight: n = cn6*R1 + (cn3*R0 + 0.5), clamped to [0, 1].
__device__ __forceinline__ float blender_noise(const V3 &pt) {
    const float x = pt.x, y = pt.y, z = pt.z;
    const int ix = (int)floorf(x), iy = (int)floorf(y), iz = (int)floorf(z);
    const float ox = x - (float)ix, oy = y - (float)iy, oz = z - (float)iz;
    const float jx = ox - 1.0f, jy = oy - 1.0f, jz = oz - 1.0f;
    auto cn_o = [](float o) { return (float)((double)(o * o) * ((double)o * 2.0 - 3.0) + 1.0); };
    auto cn_j = [](float j) { return (float)(1.0 - (double)(j * j) * ((double)j * 2.0 + 3.0)); };
    const float cn1 = cn_o(ox), cn2 = cn_o(oy), cn3 = cn_o(oz), cn4 = cn_j(jx), cn5 = cn_j(jy), cn6 = cn_j(jz);
    const int b00 = perm(perm(ix & 255) + (iy & 255)), b10 = perm(perm((ix + 1) & 255) + (iy & 255)),
              b01 = perm(perm(ix & 255) + ((iy + 1) & 255)), b11 = perm(perm((ix + 1) & 255) + ((iy + 1) & 255));
    const int b20 = iz & 255, b21 = (iz + 1) & 255;
    auto g = [](int k, float a, float b, float c) {
        const float *h = kHashVect + 3 * perm(k);
        return (__ldg(h) * a + __ldg(h + 1) * b) + __ldg(h + 2) * c;
    };
    const float w0 = cn4 * cn5, w1 = cn2 * cn4, w2 = cn1 * cn5, w3 = cn1 * cn2;
    const float R0 = (w0 * g(b20 + b11, jx, jy, oz) + w2 * g(b20 + b01, ox, jy, oz)) +
                     (w1 * g(b20 + b10, jx, oy, oz) + w3 * g(b20 + b00, ox, oy, oz));
    const float R1 = (w0 * g(b21 + b11, jx, jy, jz) + w2 * g(b21 + b01, ox, jy, jz)) +
                     (w1 * g(b21 + b10, jx, oy, jz) + w3 * g(b21 + b00, ox, oy, jz));
    float n = cn6 * R1 + (cn3 * R0 + 0.5f);
    n = n > 1.0f ? 1.0f : n;
    n = n < 0.0f ? 0.0f : n;
    return n;
}

// voronoi_t distance metrics (noise.h:69-129), e = mk_exponent: sums
// grouped x + (y + z); manhattan and the minkovsky forms in double.
__device__ __forceinline__ float vor_dist(int metric, float x, float y, float z, float e) {
    switch (metric) {
    case YR_DIST_SQUARED: return x * x + (y * y + z * z);
    case YR_DIST_MANHATTAN: return (float)((double)fabsf(x) + ((double)fabsf(y) + (double)fabsf(z)));
    case YR_DIST_CHEBYCHEV: {
        const float ax = fabsf(x), ay = fabsf(y), az = fabsf(z);
        const float t = ay > az ? ay : az;
        return ax > t ? ax : t;
    }
    case YR_DIST_MINKOVSKY_HALF: {
        const float d = (float)((sqrt((double)fabsf(x)) + sqrt((double)fabsf(y))) + sqrt((double)fabsf(z)));
        return d * d;
    }
    case YR_DIST_MINKOVSKY_FOUR: {
        const float x2 = x * x, y2 = y * y, z2 = z * z;
        return (float)sqrt(sqrt((double)(x2 * x2 + (y2 * y2 + z2 * z2))));
    }
    case YR_DIST_MINKOVSKY: {
        const double ed = (double)e;
        return (float)pow((pow((double)fabsf(x), ed) + pow((double)fabsf(y), ed)) + pow((double)fabsf(z), ed),
                          (double)(1.0f / e));
    }
    default: return sqrtf(x * x + (y * y + z * z));
    }
}

// HASHPNT (noise.cc:6)
__device__ __forceinline__ const float *hash_pnt(int x, int y, int z) {
    return kHashPnt + 3 * perm(perm(perm(z & 255) + y) + x);
}

// voronoi_t::getFeatures (noise.cc:550-589): the four nearest feature
// points of the 27 cells around pt; offsets as (x - xx) - p[0]
struct Features {
    float da[4];
    V3 pa[4];
};

__device__ __forceinline__ void vor_features(const V3 &pt, int metric, float mex, Features &F) {
    const float x = pt.x, y = pt.y, z = pt.z;
    const int xi = (int)floorf(x), yi = (int)floorf(y), zi = (int)floorf(z);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        F.da[k] = 1e10f;
        F.pa[k] = v3(0.f, 0.f, 0.f);
    }
    for (int xx = xi - 1; xx <= xi + 1; xx++) {
        const float fx = (float)xx, ox = x - fx;
        for (int yy = yi - 1; yy <= yi + 1; yy++) {
            const float fy = (float)yy, oy = y - fy;
            for (int zz = zi - 1; zz <= zi + 1; zz++) {
                const float fz = (float)zz;
                const float *p = hash_pnt(xx, yy, zz);
                const float p0 = __ldg(p), p1 = __ldg(p + 1), p2 = __ldg(p + 2);
                const float d = vor_dist(metric, ox - p0, oy - p1, (z - fz) - p2, mex);
                if (!(d < F.da[3])) continue;
                const V3 fp = v3(p0 + fx, p1 + fy, p2 + fz);
                // insert before the first larger distance (the chain of
                // d < da[k] tests of the reference)
                if (d < F.da[0]) {
                    F.da[3] = F.da[2]; F.pa[3] = F.pa[2];
                    F.da[2] = F.da[1]; F.pa[2] = F.pa[1];
                    F.da[1] = F.da[0]; F.pa[1] = F.pa[0];
                    F.da[0] = d; F.pa[0] = fp;
                } else if (d < F.da[1]) {
                    F.da[3] = F.da[2]; F.pa[3] = F.pa[2];
                    F.da[2] = F.da[1]; F.pa[2] = F.pa[1];
                    F.da[1] = d; F.pa[1] = fp;
                } else if (d < F.da[2]) {
                    F.da[3] = F.da[2]; F.pa[3] = F.pa[2];
                    F.da[2] = d; F.pa[2] = fp;
                } else {
                    F.da[3] = d; F.pa[3] = fp;
                }
            }
        }
    }
}

// cellNoise_t::operator() (noise.cc:614-622)
__device__ __forceinline__ float cell_noise(const V3 &pt) {
    const int xi = (int)floorf(pt.x), yi = (int)floorf(pt.y), zi = (int)floorf(pt.z);
    unsigned int n = (unsigned)xi + (unsigned)yi * 1301u + (unsigned)zi * 314159u;
    n ^= (n << 13);
    return (float)((double)(float)(n * (n * n * 15731u + 789221u) + 1376312589u) / 4294967296.0);
}

// the basis of newNoise (basictex.cc:34-60); voronoi bases use the real
// distance (voronoi_t defaults)
static __device__ __noinline__ float noise_gen(int type, const V3 &p) {
    switch (type) {
    case YR_NOISE_STDPERLIN: return std_perlin(p);
    case YR_NOISE_BLENDER: return blender_noise(p);
    case YR_NOISE_VORONOI_F1:
    case YR_NOISE_VORONOI_F2:
    case YR_NOISE_VORONOI_F3:
    case YR_NOISE_VORONOI_F4:
    case YR_NOISE_VORONOI_F2F1:
    case YR_NOISE_VORONOI_CRACKLE: {  // voronoi_t::operator() (noise.cc:591-611)
        Features F;
        vor_features(p, YR_DIST_REAL, 2.5f, F);
        switch (type) {
        case YR_NOISE_VORONOI_F2: return F.da[1];
        case YR_NOISE_VORONOI_F3: return F.da[2];
        case YR_NOISE_VORONOI_F4: return F.da[3];
        case YR_NOISE_VORONOI_F2F1: return F.da[1] - F.da[0];
        case YR_NOISE_VORONOI_CRACKLE: {
            const float t = (F.da[1] - F.da[0]) * 10.0f;
            return t > 1.0f ? 1.0f : t;
        }
        default: return F.da[0];
        }
    }
    case YR_NOISE_CELLNOISE: return cell_noise(p);
    default: return perlin(p);
    }
}

// getSignedNoise (noise.h:245-248)
__device__ __forceinline__ float signed_noise(int type, const V3 &p) { return 2.0f * noise_gen(type, p) - 1.0f; }

// turbulence (noise.cc:808-819) over any basis; only the blender basis
// offsets the point by one (noiseGenerator_t::offset, noise.h:16-17, 55-63)
__device__ __forceinline__ float turbulence_gen(int type, const V3 &pt, int oct, float size, bool hard) {
    float amp = 1, sum = 0;
    const V3 q = type == YR_NOISE_BLENDER ? v3(pt.x + 1.0f, pt.y + 1.0f, pt.z + 1.0f) : pt;
    V3 tp = v3(q.x * size, q.y * size, q.z * size);
    for (int i = 0; i <= oct; i++, amp *= 0.5f, tp = v3(tp.x * 2.0f, tp.y * 2.0f, tp.z * 2.0f)) {
        float val = noise_gen(type, tp);
        if (hard) val = (float)fabs(2.0 * (double)val - 1.0);
        sum += amp * val;
    }
    return sum * ((float)(1 << oct) / (float)((1 << (oct + 1)) - 1));
}

// The musgrave generators (noise.cc:638-800) over basis nt, in the shipped
// build's groupings: sn + offset as (offset - 1) + 2n, heteroterrain
// value = ((sn + offset)*pwr + 1) * value, hybrid weight = (gain*w)*signal,
// the fractional octave's products reordered as written per case.
static __device__ __noinline__ float musgrave(int kind, int nt, V3 tp, float H, float lac, float oct, float offset,
                                       float gain) {
    const float pwHL = (float)pow((double)lac, (double)-H);
    const float rmd = oct - floorf(oct);
    const int io = (int)oct;
    auto scale = [&](V3 &p) { p = v3(p.x * lac, p.y * lac, p.z * lac); };
    auto sno = [&](const V3 &q) { return (offset - 1.0f) + noise_gen(nt, q) * 2.0f; };
    switch (kind) {
    case YR_TEX_MUSGRAVE_MULTIFRACTAL: {
        float value = 1, pwr = 1;
        for (int i = 0; i < io; i++) {
            value *= (pwr * signed_noise(nt, tp) + 1.0f);
            pwr *= pwHL;
            scale(tp);
        }
        if (rmd != 0.0f) value *= ((rmd * pwr) * signed_noise(nt, tp) + 1.0f);
        return value;
    }
    case YR_TEX_MUSGRAVE_HETEROTERRAIN: {
        float pwr = pwHL;
        float value = noise_gen(nt, tp) * 2.0f + (offset - 1.0f);
        scale(tp);
        for (int i = 1; i < io; i++) {
            value = (sno(tp) * pwr + 1.0f) * value;
            pwr *= pwHL;
            scale(tp);
        }
        if (rmd != 0.0f) value = (pwr * value) * (sno(tp) * rmd) + value;
        return value;
    }
    case YR_TEX_MUSGRAVE_HYBRIDMF: {
        float pwr = pwHL;
        float result = sno(tp);
        float weight = gain * result;
        scale(tp);
        for (int i = 1; weight > 0.001f && i < io; i++) {
            const float w = weight > 1.0f ? 1.0f : weight;
            const float signal = sno(tp) * pwr;
            pwr *= pwHL;
            result = signal * w + result;
            weight = (gain * w) * signal;
            scale(tp);
        }
        if (rmd != 0.0f) result = sno(tp) * (rmd * pwr) + result;
        return result;
    }
    case YR_TEX_MUSGRAVE_RIDGEDMF: {
        float pwr = pwHL;
        float signal = offset - fabsf(signed_noise(nt, tp));
        signal *= signal;
        float result = signal;
        for (int i = 1; i < io; i++) {
            scale(tp);
            float weight = gain * signal;
            weight = weight > 0.0f ? weight : 0.0f;
            weight = weight < 1.0f ? weight : 1.0f;
            const float q = offset - fabsf(signed_noise(nt, tp));
            signal = weight * (q * q);
            result = signal * pwr + result;
            pwr = pwHL * pwr;
        }
        return result;
    }
    default: {  // fBm
        float value = 0, pwr = 1;
        for (int i = 0; i < io; i++) {
            value += signed_noise(nt, tp) * pwr;
            pwr *= pwHL;
            scale(tp);
        }
        if (rmd != 0.f) value += rmd * signed_noise(nt, tp) * pwr;
        return value;
    }
    }
}

// marble / wood wave shapes (basictex.cc:124-140, 199-214); the sine as
// the shipped build's (sin(w) + 1) * 0.5
__device__ __forceinline__ float wave(int shape, float w) {
    if (shape == YR_WAVE_SAW) {
        w *= (float)(0.5 * 0.31830988618379067154)  /* 0.5 * M_1_PI */;
        return w - floorf(w);
    }
    if (shape == YR_WAVE_TRI) {
        w *= (float)(0.5 * 0.31830988618379067154)  /* 0.5 * M_1_PI */;
        return fabsf(2.0f * (w - floorf(w)) - 1.0f);
    }
    return (sinf(w) + 1.0f) * 0.5f;
}

// A texture at texture point p: its colour (getColor rgb), and for the
// adjoint the colour's derivative by the texture "intensity" (musgrave,
// voronoi; zero for the others) and by color1 (the same scale on every
// channel; zero for voronoi, whose colour does not use color1).
struct TexEval {
    C3 col;
    C3 dint;
    float dc1;
    float f;   // getFloat (the hardness modulator's value)
};

static __device__ __noinline__ TexEval texture_eval(const DevShader *__restrict__ shp, const V3 &p) {
    const DevShader &sh = *shp;
    TexEval r;
    r.dint = c3(0.f, 0.f, 0.f);
    const V3 ps = v3(p.x * sh.tsize, p.y * sh.tsize, p.z * sh.tsize);
    float f;
    switch (sh.tex_type) {
    case YR_TEX_CLOUDS: {  // textureClouds_t::getFloat (basictex.cc:76-85)
        float v = turbulence_gen(sh.noise, p, sh.tdepth, sh.tsize, sh.thard != 0);
        if (sh.tvariant == 1 || sh.tvariant == 2) {
            v *= v;
            if (sh.tvariant == 1) v = -v;
        }
        f = v;
        break;
    }
    case YR_TEX_MARBLE: {  // textureMarble_t::getFloat (basictex.cc:122-146)
        const double tu =
            sh.turb == 0.0f ? 0.0 : (double)(sh.turb * turbulence_gen(sh.noise, p, sh.tdepth, sh.tsize, sh.thard != 0));
        const float w = (float)((double)(p.x + p.y + p.z) * 5.0 + tu);
        f = powf(wave(sh.tshape, w), sh.sharp);
        break;
    }
    case YR_TEX_WOOD: {  // textureWood_t::getFloat (basictex.cc:192-216)
        float w = sh.tvariant ? sqrtf(p.x * p.x + p.y * p.y + p.z * p.z) * 20.0f : (p.x + p.y + p.z) * 10.0f;
        const double tu =
            sh.turb == 0.0f ? 0.0 : (double)(sh.turb * turbulence_gen(sh.noise, p, sh.tdepth, sh.tsize, sh.thard != 0));
        w = (float)((double)w + tu);
        f = wave(sh.tshape, w);
        break;
    }
    case YR_TEX_VORONOI: {  // textureVoronoi_t (basictex.cc:560-617)
        Features F;
        vor_features(ps, sh.metric, sh.mk_exp, F);
        // the weighted sum as the shipped build's vector reduction
        const float S = fabsf((sh.weights[0] * F.da[0] + sh.weights[2] * F.da[2]) +
                              (sh.weights[1] * F.da[1] + sh.weights[3] * F.da[3]));
        const float inte = sh.viscale * S;
        r.dc1 = 0.f;
        r.f = inte;
        if (sh.tshape == 0) {
            r.col = c3(inte, inte, inte);
            const float d = sh.vinvw * S;
            r.dint = c3(d, d, d);
            return r;
        }
        C3 col = c3(0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 4; k++) {  // cellNoiseColor (noise.cc:795-803) of each feature point
            const float *cl = hash_pnt((int)floorf(F.pa[k].x), (int)floorf(F.pa[k].y), (int)floorf(F.pa[k].z));
            const float aw = fabsf(sh.weights[k]);
            col = col + c3(aw * __ldg(cl), aw * __ldg(cl + 1), aw * __ldg(cl + 2));
        }
        float t1 = sh.viscale, dt = sh.vinvw;  // col * t1, and d t1 / d intensity
        if (sh.tshape >= 2) {
            const float dd = F.da[1] - F.da[0];
            const float t = dd > 0.1f ? 1.0f : dd * 10.0f;
            if (sh.tshape == 3) {
                t1 = t * inte;
                dt = t * (sh.vinvw * S);
            } else {
                t1 = sh.viscale * t;
                dt = sh.vinvw * t;
            }
        }
        r.col = col * t1;
        r.dint = col * dt;
        return r;
    }
    case YR_TEX_DISTORTED_NOISE: {  // textureDistortedNoise_t::getFloat (basictex.cc:721-727)
        const V3 rv = v3(signed_noise(sh.noise, v3(ps.x + 13.5f, ps.y + 13.5f, ps.z + 13.5f)),
                         signed_noise(sh.noise, ps), signed_noise(sh.noise, v3(ps.x - 13.5f, ps.y - 13.5f, ps.z - 13.5f)));
        f = signed_noise(sh.noise2, v3(ps.x + rv.x * sh.distort, ps.y + rv.y * sh.distort, ps.z + rv.z * sh.distort));
        break;
    }
    case YR_TEX_GRADIENT: {  // textureGradient_t::getFloat (basictex.cc:772-800)
        const float x = sh.tvariant ? p.y : p.x, y = sh.tvariant ? p.x : p.y;
        float gr;
        switch (sh.tshape) {
        case YR_GRAD_QUADRATIC:
            gr = (float)((1.0 + (double)x) * 0.5);
            f = gr < 0 ? 0.f : gr * gr;
            break;
        case YR_GRAD_CUBIC:
            gr = (float)((1.0 + (double)x) * 0.5);
            if (gr > 1) {  // getColor folds color1 + 1*(color2 - color1) to color2 in the shipped build
                r.col = sh.tc2;
                r.dc1 = 0.f;
                r.f = 1.f;
                return r;
            }
            f = gr < 0 ? 0.f : (float)((double)(gr * gr) * (3.0 - 2.0 * (double)gr));
            break;
        case YR_GRAD_DIAGONAL: f = (float)(((double)x + (double)y + 2.0) * 0.25); break;
        case YR_GRAD_SPHERE:
        case YR_GRAD_HALO:
            gr = (float)(1.0 - (double)sqrtf(x * x + y * y + p.z * p.z));
            f = gr < 0 ? 0.f : (sh.tshape == YR_GRAD_HALO ? gr * gr : gr);
            break;
        default: f = (float)((1.0 + (double)x) * 0.5);
        }
        break;
    }
    default: {  // musgrave: iscale * generator(p*size) (basictex.cc:677-680)
        const float m = musgrave(sh.tex_type, sh.noise, ps, sh.H, sh.lacunarity, sh.octaves, sh.offset, sh.gain);
        f = sh.intensity * m;
        r.dint = m * (sh.tc2 - sh.tc1);
    }
    }
    r.col = sh.tc1 + f * (sh.tc2 - sh.tc1);
    r.dc1 = 1.f - f;
    r.f = f;
    return r;
}

}  // namespace yr
