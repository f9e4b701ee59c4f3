// 8-bit image output of Renderer::Render (Renderer.cpp:163-211): the
// tone-mapped framebuffer written as PNG (zlib deflate, one filter byte per
// row) or binary PPM, and the adaptive-sampling visualisation.
#include <zlib.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "prr.h"
#include "prr_internal.h"

namespace {

void put_be32(std::vector<uint8_t> &o, uint32_t v) {
    o.push_back((uint8_t) (v >> 24));
    o.push_back((uint8_t) (v >> 16));
    o.push_back((uint8_t) (v >> 8));
    o.push_back((uint8_t) v);
}

void chunk(std::vector<uint8_t> &o, const char *type, const uint8_t *data, size_t n) {
    put_be32(o, (uint32_t) n);
    const size_t at = o.size();
    o.insert(o.end(), type, type + 4);
    o.insert(o.end(), data, data + n);
    put_be32(o, (uint32_t) crc32(0L, o.data() + at, (uInt) (n + 4)));
}

bool ends_with(const std::string &s, const char *suffix) {
    const size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

} // namespace

using namespace prr;

extern "C" int prr_write_image(const char *path, const uint8_t *rgb, int width, int height) {
    if (!path || !rgb || width <= 0 || height <= 0)
        return fail(PRR_ERR_INVALID_ARGUMENT, "path, pixels and a positive size are required");
    const std::string p(path);
    FILE *f = std::fopen(path, "wb");
    if (!f)
        return fail(PRR_ERR_INVALID_ARGUMENT, "cannot open " + p);
    const size_t row = (size_t) width * 3;
    bool ok = true;
    if (ends_with(p, ".ppm")) {
        std::fprintf(f, "P6\n%d %d\n255\n", width, height);
        ok = std::fwrite(rgb, 1, row * height, f) == row * height;
    } else if (ends_with(p, ".png")) {
        std::vector<uint8_t> raw((row + 1) * height);
        for (int y = 0; y < height; y++) {
            raw[(size_t) y * (row + 1)] = 0; // filter: none
            std::memcpy(&raw[(size_t) y * (row + 1) + 1], rgb + (size_t) y * row, row);
        }
        uLongf zlen = compressBound((uLong) raw.size());
        std::vector<uint8_t> z(zlen);
        if (compress2(z.data(), &zlen, raw.data(), (uLong) raw.size(), 6) != Z_OK) {
            std::fclose(f);
            return fail(PRR_ERR_INTERNAL, "PNG compression failed");
        }
        static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
        std::vector<uint8_t> out(sig, sig + 8);
        uint8_t ihdr[13];
        const uint32_t w = (uint32_t) width, h = (uint32_t) height;
        const uint8_t be[8] = {(uint8_t) (w >> 24), (uint8_t) (w >> 16), (uint8_t) (w >> 8),
                               (uint8_t) w,         (uint8_t) (h >> 24), (uint8_t) (h >> 16),
                               (uint8_t) (h >> 8),  (uint8_t) h};
        std::memcpy(ihdr, be, 8);
        ihdr[8] = 8;  // bit depth
        ihdr[9] = 2;  // RGB
        ihdr[10] = 0; // deflate
        ihdr[11] = 0; // adaptive filtering (per-row type bytes)
        ihdr[12] = 0; // no interlace
        chunk(out, "IHDR", ihdr, 13);
        chunk(out, "IDAT", z.data(), zlen);
        chunk(out, "IEND", nullptr, 0);
        ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    } else {
        std::fclose(f);
        return fail(PRR_ERR_INVALID_ARGUMENT, "image path must end in .png or .ppm");
    }
    if (std::fclose(f) != 0 || !ok)
        return fail(PRR_ERR_INTERNAL, "writing " + p + " failed");
    return PRR_OK;
}

extern "C" int prr_sample_count_image(const int32_t *spp, int64_t n, int max_spp, uint8_t *out_rgb) {
    if ((n > 0 && (!spp || !out_rgb)) || n < 0 || max_spp <= 0)
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad sample-count image arguments");
    for (int64_t i = 0; i < n; i++) {
        const unsigned char v = (unsigned char) (255 * (float) spp[i] / (float) max_spp);
        out_rgb[i * 3] = out_rgb[i * 3 + 1] = out_rgb[i * 3 + 2] = v;
    }
    return PRR_OK;
}
