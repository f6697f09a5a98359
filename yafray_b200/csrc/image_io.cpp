// Image outputs of a render, byte for byte as YafRay's colorOutput_t
// writers produce them from the same float pixels:
//   outTga_t  (targaIO.cc:37-130): uncompressed true-colour Targa, top-left
//             origin, BGR or BGRA;
//   outHDR_t  (HDR_io.cc:34-160): Radiance RGBE with run-length scanlines
//             (Greg Ward's picture format; the run encoder of fwritecolrs).
// Conversions follow the shipped build (-O3 -ffast-math): colour bytes
// from x*255.f (0 below 0 and for NaN, 255 at 1 and above), alpha bytes
// from min(a, 1)*255.0 in double, RGBE mantissas from the float channel
// times (float)(frexp(d)*256/d) with d the largest channel in double.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/yr.h"

namespace {

// operator<<(unsigned char*, const color_t&) (color.cc:35-40)
inline uint8_t tga_byte(float x) {
    if (x >= 0.0f) return x < 1.0f ? (uint8_t)(x * 255.0f) : 255;
    return 0;
}

// outTga_t::putPixel alpha (targaIO.cc:65-66)
inline uint8_t tga_alpha(float a) {
    if (a >= 0.0f) return (uint8_t)((double)(a < 1.0f ? a : 1.0f) * 255.0);
    return 0;
}

size_t tga_size(int32_t w, int32_t h, int32_t save_alpha) {
    return 18 + (size_t)w * (size_t)h * (save_alpha ? 4u : 3u);
}

void tga_encode(const float *rgba, int32_t w, int32_t h, int32_t save_alpha, uint8_t *out) {
    static const uint8_t hdr[12] = {0, 0, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // uncompressed true colour
    memcpy(out, hdr, 12);
    const uint16_t ww = (uint16_t)w, hh = (uint16_t)h;
    out[12] = (uint8_t)(ww & 255);
    out[13] = (uint8_t)(ww >> 8);
    out[14] = (uint8_t)(hh & 255);
    out[15] = (uint8_t)(hh >> 8);
    out[16] = save_alpha ? 0x20 : 0x18;  // bits per pixel
    out[17] = save_alpha ? 0x28 : 0x20;  // top-left origin (+ 8 alpha bits)
    uint8_t *o = out + 18;
    for (size_t i = 0, n = (size_t)w * (size_t)h; i < n; i++) {
        const float *p = rgba + 4 * i;
        *o++ = tga_byte(p[2]);
        *o++ = tga_byte(p[1]);
        *o++ = tga_byte(p[0]);
        if (save_alpha) *o++ = tga_alpha(p[3]);
    }
}

// one pixel's RGBE (HDRwrite_t::fwritecolrs, HDR_io.cc:78-93)
inline void rgbe(const float *p, uint8_t *q) {
    const float d = std::fmax(p[0], std::fmax(p[1], p[2]));
    if ((double)d <= (double)1e-32f) {
        q[0] = q[1] = q[2] = q[3] = 0;
        return;
    }
    int e;
    const double dd = (double)d;
    const float m = (float)(std::frexp(dd, &e) * 256.0 / dd);
    q[0] = (uint8_t)(p[0] * m);
    q[1] = (uint8_t)(p[1] * m);
    q[2] = (uint8_t)(p[2] * m);
    q[3] = (uint8_t)(e + 128);
}

struct Sink {
    std::vector<uint8_t> &v;
    void put(uint8_t b) { v.push_back(b); }
};

// One scanline: flat for widths outside [8, 0x7fff], else the "new" RLE
// form: 2 2 w_hi w_lo, then each of the four components as runs (>= 4
// equal bytes: 128+n, byte) and literal spans (n <= 128, bytes), with short
// runs of 2-3 equal bytes ahead of a long run written as runs.
void hdr_scanline(const uint8_t *sc, int w, Sink &out) {
    const int kMinRun = 4;
    if (w < 8 || w > 0x7fff) {
        for (int i = 0; i < 4 * w; i++) out.put(sc[i]);
        return;
    }
    out.put(2);
    out.put(2);
    out.put((uint8_t)(w >> 8));
    out.put((uint8_t)(w & 255));
    for (int c = 0; c < 4; c++) {
        auto at = [&](int i) { return sc[4 * i + c]; };
        int cnt = 0;
        for (int j = 0; j < w; j += cnt) {
            int beg;
            for (beg = j; beg < w; beg += cnt) {  // the next long run
                for (cnt = 1; cnt < 127 && beg + cnt < w && at(beg + cnt) == at(beg); cnt++) {
                }
                if (cnt >= kMinRun) break;
            }
            if (beg - j > 1 && beg - j < kMinRun) {  // a short run right before it
                int c2 = j + 1;
                while (at(c2++) == at(j))
                    if (c2 == beg) {
                        out.put((uint8_t)(128 + beg - j));
                        out.put(at(j));
                        j = beg;
                        break;
                    }
            }
            while (j < beg) {  // literal span
                int n = beg - j;
                if (n > 128) n = 128;
                out.put((uint8_t)n);
                while (n--) out.put(at(j++));
            }
            if (cnt >= kMinRun) {
                out.put((uint8_t)(128 + cnt));
                out.put(at(beg));
            } else {
                cnt = 0;
            }
        }
    }
}

void hdr_encode(const float *rgba, int32_t w, int32_t h, std::vector<uint8_t> &v) {
    char head[256];
    int n = snprintf(head, sizeof(head), "#?RADIANCE\n# %s\nFORMAT=32-bit_rle_rgbe\nEXPOSURE=%25.13f\n\n-Y %d +X %d\n",
                     "Created with YafRay", 1.0, h, w);
    v.assign(head, head + n);
    Sink s{v};
    std::vector<uint8_t> sc(4 * (size_t)w);
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) rgbe(rgba + 4 * ((size_t)y * w + x), &sc[4 * (size_t)x]);
        hdr_scanline(sc.data(), w, s);
    }
}

yr_status write_file(const char *path, const uint8_t *p, size_t n) {
    FILE *f = fopen(path, "wb");
    if (!f) return YR_ERR_INVALID_ARG;
    const bool ok = fwrite(p, 1, n, f) == n;
    return (fclose(f) == 0 && ok) ? YR_OK : YR_ERR_INVALID_ARG;
}

}  // namespace

YR_API yr_status yr_image_encode(int32_t format, const float *rgba, int32_t width, int32_t height, int32_t flags,
                                 uint8_t *out, size_t capacity, size_t *size) {
    if (!rgba || !size || width <= 0 || height <= 0 || width > 0xffff || height > 0xffff) return YR_ERR_INVALID_ARG;
    if (format == YR_IMAGE_TGA) {
        const size_t n = tga_size(width, height, flags & YR_IMAGE_ALPHA);
        *size = n;
        if (!out) return YR_OK;
        if (capacity < n) return YR_ERR_INVALID_ARG;
        tga_encode(rgba, width, height, flags & YR_IMAGE_ALPHA, out);
        return YR_OK;
    }
    if (format == YR_IMAGE_HDR) {
        std::vector<uint8_t> v;
        hdr_encode(rgba, width, height, v);
        *size = v.size();
        if (!out) return YR_OK;
        if (capacity < v.size()) return YR_ERR_INVALID_ARG;
        memcpy(out, v.data(), v.size());
        return YR_OK;
    }
    return YR_ERR_INVALID_ARG;
}

YR_API yr_status yr_image_write(const char *path, int32_t format, const float *rgba, int32_t width, int32_t height,
                                int32_t flags) {
    if (!path) return YR_ERR_INVALID_ARG;
    size_t n = 0;
    yr_status st = yr_image_encode(format, rgba, width, height, flags, nullptr, 0, &n);
    if (st != YR_OK) return st;
    std::vector<uint8_t> buf(n);
    if ((st = yr_image_encode(format, rgba, width, height, flags, buf.data(), n, &n)) != YR_OK) return st;
    return write_file(path, buf.data(), n);
}
