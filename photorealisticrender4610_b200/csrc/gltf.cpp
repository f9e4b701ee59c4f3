// glTF 2.0 ingest: the job of the reference's GLTFLoader (GLTFLoader.cpp:
// 13-281, on tinygltf): one MeshTriangle per triangle primitive with its
// per-corner normals, uvs and tangents, and a material per primitive from the
// glTF material (pbrMetallicRoughness factors, emissive factor, base-colour,
// metallic-roughness, normal and emissive textures), converted to the
// requested material class. Written here from the glTF 2.0 specification:
// a small JSON reader, the .glb container and .gltf files with external or
// base64 buffers, accessors read exactly as the reference reads them, and a
// PNG decoder on zlib (images come out as 8-bit RGBA, as tinygltf's default
// decode gives them). JPEG and interlaced PNG images are not decoded: their
// textures are left out and counted.
#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "prr.h"
#include "prr_internal.h"

namespace prr {
namespace {

// ------------------------------------------------------------------ JSON
struct Json {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    double num = 0;
    bool b = false;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;

    const Json *get(const char *key) const {
        if (kind != Obj)
            return nullptr;
        for (const auto &kv : obj)
            if (kv.first == key)
                return &kv.second;
        return nullptr;
    }
    const Json *at(size_t i) const { return kind == Arr && i < arr.size() ? &arr[i] : nullptr; }
    size_t size() const { return kind == Arr ? arr.size() : 0; }
};

double num_or(const Json *j, double d) { return j && j->kind == Json::Num ? j->num : d; }
int int_or(const Json *j, int d) { return j && j->kind == Json::Num ? (int) j->num : d; }

class JsonReader {
  public:
    JsonReader(const char *p, size_t n) : p_(p), end_(p + n) {}
    bool parse(Json &out, std::string &err) {
        if (!value(out, 0)) {
            err = "JSON: " + err_;
            return false;
        }
        ws();
        return true;
    }

  private:
    const char *p_, *end_;
    std::string err_;

    void ws() {
        while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r'))
            p_++;
    }
    bool fail(const char *m) {
        err_ = m;
        return false;
    }
    bool lit(const char *w) {
        const size_t n = std::strlen(w);
        if ((size_t) (end_ - p_) < n || std::memcmp(p_, w, n) != 0)
            return false;
        p_ += n;
        return true;
    }
    static void put_utf8(std::string &s, unsigned cp) {
        if (cp < 0x80) {
            s += (char) cp;
        } else if (cp < 0x800) {
            s += (char) (0xC0 | (cp >> 6));
            s += (char) (0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            s += (char) (0xE0 | (cp >> 12));
            s += (char) (0x80 | ((cp >> 6) & 0x3F));
            s += (char) (0x80 | (cp & 0x3F));
        } else {
            s += (char) (0xF0 | (cp >> 18));
            s += (char) (0x80 | ((cp >> 12) & 0x3F));
            s += (char) (0x80 | ((cp >> 6) & 0x3F));
            s += (char) (0x80 | (cp & 0x3F));
        }
    }
    bool hex4(unsigned &v) {
        if (end_ - p_ < 4)
            return false;
        v = 0;
        for (int i = 0; i < 4; i++) {
            const char c = *p_++;
            v <<= 4;
            if (c >= '0' && c <= '9')
                v |= (unsigned) (c - '0');
            else if (c >= 'a' && c <= 'f')
                v |= (unsigned) (c - 'a' + 10);
            else if (c >= 'A' && c <= 'F')
                v |= (unsigned) (c - 'A' + 10);
            else
                return false;
        }
        return true;
    }
    bool string(std::string &s) {
        if (p_ >= end_ || *p_ != '"')
            return fail("expected a string");
        p_++;
        while (p_ < end_ && *p_ != '"') {
            char c = *p_++;
            if (c != '\\') {
                s += c;
                continue;
            }
            if (p_ >= end_)
                return fail("bad escape");
            c = *p_++;
            switch (c) {
            case '"': s += '"'; break;
            case '\\': s += '\\'; break;
            case '/': s += '/'; break;
            case 'b': s += '\b'; break;
            case 'f': s += '\f'; break;
            case 'n': s += '\n'; break;
            case 'r': s += '\r'; break;
            case 't': s += '\t'; break;
            case 'u': {
                unsigned cp;
                if (!hex4(cp))
                    return fail("bad \\u escape");
                if (cp >= 0xD800 && cp < 0xDC00 && end_ - p_ >= 6 && p_[0] == '\\' && p_[1] == 'u') {
                    p_ += 2;
                    unsigned lo;
                    if (!hex4(lo))
                        return fail("bad surrogate");
                    cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                }
                put_utf8(s, cp);
                break;
            }
            default:
                return fail("bad escape");
            }
        }
        if (p_ >= end_)
            return fail("unterminated string");
        p_++;
        return true;
    }
    bool value(Json &v, int depth) {
        if (depth > 256)
            return fail("nesting too deep");
        ws();
        if (p_ >= end_)
            return fail("unexpected end");
        const char c = *p_;
        if (c == '{') {
            p_++;
            v.kind = Json::Obj;
            ws();
            if (p_ < end_ && *p_ == '}') {
                p_++;
                return true;
            }
            for (;;) {
                ws();
                std::string key;
                if (!string(key))
                    return false;
                ws();
                if (p_ >= end_ || *p_ != ':')
                    return fail("expected ':'");
                p_++;
                v.obj.emplace_back(std::move(key), Json());
                if (!value(v.obj.back().second, depth + 1))
                    return false;
                ws();
                if (p_ < end_ && *p_ == ',') {
                    p_++;
                    continue;
                }
                if (p_ < end_ && *p_ == '}') {
                    p_++;
                    return true;
                }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            p_++;
            v.kind = Json::Arr;
            ws();
            if (p_ < end_ && *p_ == ']') {
                p_++;
                return true;
            }
            for (;;) {
                v.arr.emplace_back();
                if (!value(v.arr.back(), depth + 1))
                    return false;
                ws();
                if (p_ < end_ && *p_ == ',') {
                    p_++;
                    continue;
                }
                if (p_ < end_ && *p_ == ']') {
                    p_++;
                    return true;
                }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = Json::Str;
            return string(v.str);
        }
        if (lit("true")) {
            v.kind = Json::Bool;
            v.b = true;
            return true;
        }
        if (lit("false")) {
            v.kind = Json::Bool;
            return true;
        }
        if (lit("null"))
            return true;
        // number
        const char *s = p_;
        if (p_ < end_ && (*p_ == '-' || *p_ == '+'))
            p_++;
        while (p_ < end_ && ((*p_ >= '0' && *p_ <= '9') || *p_ == '.' || *p_ == 'e' ||
                             *p_ == 'E' || *p_ == '-' || *p_ == '+'))
            p_++;
        if (p_ == s)
            return fail("unexpected character");
        v.kind = Json::Num;
        v.num = std::strtod(std::string(s, p_).c_str(), nullptr);
        return true;
    }
};

// ------------------------------------------------------------------ base64
bool base64(const std::string &in, std::vector<uint8_t> &out) {
    auto val = [](char c) -> int {
        if (c >= 'A' && c <= 'Z') return c - 'A';
        if (c >= 'a' && c <= 'z') return c - 'a' + 26;
        if (c >= '0' && c <= '9') return c - '0' + 52;
        if (c == '+' || c == '-') return 62;
        if (c == '/' || c == '_') return 63;
        return -1;
    };
    unsigned acc = 0;
    int bits = 0;
    for (char c : in) {
        if (c == '=' || c == '\n' || c == '\r' || c == ' ')
            continue;
        const int v = val(c);
        if (v < 0)
            return false;
        acc = (acc << 6) | (unsigned) v;
        bits += 6;
        if (bits >= 8) {
            bits -= 8;
            out.push_back((uint8_t) ((acc >> bits) & 0xFF));
        }
    }
    return true;
}

// ------------------------------------------------------------------ PNG
uint32_t be32(const uint8_t *p) {
    return ((uint32_t) p[0] << 24) | ((uint32_t) p[1] << 16) | ((uint32_t) p[2] << 8) | p[3];
}

// Decodes a PNG into 8-bit RGBA: grey and palette expanded, bit depths below
// 8 scaled to 0..255, 16-bit samples reduced to their high byte (the
// reference's loader shifts 16-bit texels right by 8, GLTFLoader.cpp:80-88).
// Returns false for what it does not decode (interlaced images, damage).
bool decode_png(const uint8_t *d, size_t n, int &w, int &h, std::vector<uint8_t> &rgba) {
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (n < 8 || std::memcmp(d, sig, 8) != 0)
        return false;
    size_t p = 8;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, pal;
    w = h = 0;
    while (p + 12 <= n) {
        const uint32_t len = be32(d + p);
        const uint8_t *type = d + p + 4;
        const uint8_t *data = d + p + 8;
        if (p + 12 + (size_t) len > n)
            return false;
        if (!std::memcmp(type, "IHDR", 4) && len >= 13) {
            w = (int) be32(data);
            h = (int) be32(data + 4);
            depth = data[8];
            ctype = data[9];
            interlace = data[12];
        } else if (!std::memcmp(type, "PLTE", 4)) {
            pal.assign(data, data + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), data, data + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        }
        p += 12 + len;
    }
    if (w <= 0 || h <= 0 || interlace != 0 || (int64_t) w * h > ((int64_t) 1 << 28))
        return false;
    int ch;
    switch (ctype) {
    case 0: ch = 1; break;
    case 2: ch = 3; break;
    case 3: ch = 1; break;
    case 4: ch = 2; break;
    case 6: ch = 4; break;
    default: return false;
    }
    if (depth != 1 && depth != 2 && depth != 4 && depth != 8 && depth != 16)
        return false;
    if ((ctype == 2 || ctype == 4 || ctype == 6) && depth < 8)
        return false;
    if (ctype == 3 && (depth == 16 || pal.empty()))
        return false;
    const size_t bits_pp = (size_t) ch * depth;
    const size_t row = ((size_t) w * bits_pp + 7) / 8;
    const size_t bpp = std::max<size_t>(1, bits_pp / 8);
    std::vector<uint8_t> raw((row + 1) * (size_t) h);
    uLongf raw_len = (uLongf) raw.size();
    if (uncompress(raw.data(), &raw_len, idat.data(), (uLong) idat.size()) != Z_OK ||
        raw_len != raw.size())
        return false;
    // undo the per-scanline filters
    std::vector<uint8_t> img(row * (size_t) h);
    for (int y = 0; y < h; y++) {
        const uint8_t f = raw[(size_t) y * (row + 1)];
        const uint8_t *src = &raw[(size_t) y * (row + 1) + 1];
        uint8_t *dst = &img[(size_t) y * row];
        const uint8_t *up = y > 0 ? &img[(size_t) (y - 1) * row] : nullptr;
        for (size_t x = 0; x < row; x++) {
            const int a = x >= bpp ? dst[x - bpp] : 0;
            const int b = up ? up[x] : 0;
            const int c = (up && x >= bpp) ? up[x - bpp] : 0;
            int v = src[x];
            switch (f) {
            case 0: break;
            case 1: v += a; break;
            case 2: v += b; break;
            case 3: v += (a + b) / 2; break;
            case 4: {
                const int pp = a + b - c;
                const int pa = std::abs(pp - a), pb = std::abs(pp - b), pc = std::abs(pp - c);
                v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
                break;
            }
            default:
                return false;
            }
            dst[x] = (uint8_t) v;
        }
    }
    // samples -> RGBA8
    rgba.assign((size_t) w * h * 4, 255);
    auto sample = [&](const uint8_t *r, int x, int c) -> int { // 8-bit value of sample c of pixel x
        if (depth == 8)
            return r[(size_t) x * ch + c];
        if (depth == 16)
            return r[((size_t) x * ch + c) * 2]; // high byte
        const int per = 8 / depth;
        const int idx = x; // sub-byte depths only occur with one channel
        const int byte = r[idx / per];
        const int shift = 8 - depth * (idx % per + 1);
        const int v = (byte >> shift) & ((1 << depth) - 1);
        return ctype == 3 ? v : v * (255 / ((1 << depth) - 1));
    };
    for (int y = 0; y < h; y++) {
        const uint8_t *r = &img[(size_t) y * row];
        for (int x = 0; x < w; x++) {
            uint8_t *o = &rgba[((size_t) y * w + x) * 4];
            if (ctype == 3) {
                const int k = sample(r, x, 0);
                if ((size_t) (k * 3 + 2) >= pal.size())
                    return false;
                o[0] = pal[k * 3];
                o[1] = pal[k * 3 + 1];
                o[2] = pal[k * 3 + 2];
            } else if (ch <= 2) {
                const int g = sample(r, x, 0);
                o[0] = o[1] = o[2] = (uint8_t) g;
                if (ch == 2)
                    o[3] = (uint8_t) sample(r, x, 1);
            } else {
                o[0] = (uint8_t) sample(r, x, 0);
                o[1] = (uint8_t) sample(r, x, 1);
                o[2] = (uint8_t) sample(r, x, 2);
                if (ch == 4)
                    o[3] = (uint8_t) sample(r, x, 3);
            }
        }
    }
    return true;
}

// ------------------------------------------------------------------ glTF
struct Gltf {
    Json doc;
    std::vector<std::vector<uint8_t>> buffers;
    std::string dir;
};

bool read_file(const std::string &path, std::vector<uint8_t> &out) {
    std::ifstream f(path, std::ios::binary);
    if (!f)
        return false;
    out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return true;
}

bool load_uri(const Gltf &g, const std::string &uri, std::vector<uint8_t> &out) {
    if (uri.compare(0, 5, "data:") == 0) {
        const size_t comma = uri.find(',');
        if (comma == std::string::npos || uri.find(";base64") == std::string::npos)
            return false;
        return base64(uri.substr(comma + 1), out);
    }
    return read_file(g.dir + uri, out);
}

bool open_gltf(const std::string &path, Gltf &g, std::string &err) {
    std::vector<uint8_t> bytes;
    if (!read_file(path, bytes)) {
        err = "cannot read " + path;
        return false;
    }
    const size_t slash = path.find_last_of('/');
    g.dir = slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
    const uint8_t *json = bytes.data();
    size_t json_len = bytes.size();
    std::vector<uint8_t> bin;
    bool glb = bytes.size() >= 12 && std::memcmp(bytes.data(), "glTF", 4) == 0;
    if (glb) {
        // 12-byte header, then chunks: JSON (0x4E4F534A) first, BIN (0x004E4942)
        auto le32 = [&](size_t o) {
            uint32_t v;
            std::memcpy(&v, bytes.data() + o, 4);
            return v;
        };
        const uint32_t total = std::min<uint32_t>(le32(8), (uint32_t) bytes.size());
        size_t o = 12;
        json = nullptr;
        while (o + 8 <= total) {
            const uint32_t len = le32(o), type = le32(o + 4);
            if (o + 8 + (size_t) len > total)
                break;
            if (type == 0x4E4F534Au && !json) {
                json = bytes.data() + o + 8;
                json_len = len;
            } else if (type == 0x004E4942u && bin.empty()) {
                bin.assign(bytes.begin() + o + 8, bytes.begin() + o + 8 + len);
            }
            o += 8 + ((len + 3) & ~3u);
        }
        if (!json) {
            err = "GLB without a JSON chunk";
            return false;
        }
    }
    if (!JsonReader((const char *) json, json_len).parse(g.doc, err))
        return false;
    const Json *bufs = g.doc.get("buffers");
    for (size_t i = 0; bufs && i < bufs->size(); i++) {
        const Json *uri = bufs->at(i)->get("uri");
        std::vector<uint8_t> data;
        if (uri && uri->kind == Json::Str) {
            if (!load_uri(g, uri->str, data)) {
                err = "cannot load buffer " + uri->str;
                return false;
            }
        } else if (glb && i == 0) {
            data = bin;
        }
        g.buffers.push_back(std::move(data));
    }
    return true;
}

int components(const std::string &type) {
    if (type == "SCALAR") return 1;
    if (type == "VEC2") return 2;
    if (type == "VEC3") return 3;
    if (type == "VEC4") return 4;
    if (type == "MAT2") return 4;
    if (type == "MAT3") return 9;
    if (type == "MAT4") return 16;
    return 0;
}
int component_bytes(int ct) {
    switch (ct) {
    case 5120: case 5121: return 1;
    case 5122: case 5123: return 2;
    case 5125: case 5126: return 4;
    default: return 0;
    }
}

// Where an accessor's elements start: the buffer bytes, element stride and
// count; false when it does not resolve inside its buffer.
bool accessor_view(const Gltf &g, int idx, const uint8_t *&base, size_t &stride, size_t &count,
                   int &nc, int &ct) {
    const Json *acc = g.doc.get("accessors") ? g.doc.get("accessors")->at((size_t) idx) : nullptr;
    if (!acc)
        return false;
    const int bvi = int_or(acc->get("bufferView"), -1);
    const Json *bv = g.doc.get("bufferViews") ? g.doc.get("bufferViews")->at((size_t) bvi) : nullptr;
    if (bvi < 0 || !bv)
        return false;
    const int bi = int_or(bv->get("buffer"), -1);
    if (bi < 0 || bi >= (int) g.buffers.size())
        return false;
    const Json *type = acc->get("type");
    nc = type && type->kind == Json::Str ? components(type->str) : 0;
    ct = int_or(acc->get("componentType"), 0);
    const int cs = component_bytes(ct);
    count = (size_t) num_or(acc->get("count"), 0);
    if (nc == 0 || cs == 0)
        return false;
    const size_t bstride = (size_t) num_or(bv->get("byteStride"), 0);
    stride = bstride ? bstride : (size_t) nc * cs;
    const size_t off = (size_t) num_or(bv->get("byteOffset"), 0) +
                       (size_t) num_or(acc->get("byteOffset"), 0);
    const std::vector<uint8_t> &buf = g.buffers[bi];
    if (count > 0 && off + (count - 1) * stride + (size_t) nc * cs > buf.size())
        return false;
    base = buf.data() + off;
    return true;
}

// tg_readFloats (GLTFLoader.cpp:13-40): float, or unsigned short / byte
// read as normalized; any other component type reads as 0.
bool read_floats(const Gltf &g, int idx, std::vector<float> &out, int &nc) {
    const uint8_t *base;
    size_t stride, count;
    int ct;
    if (!accessor_view(g, idx, base, stride, count, nc, ct))
        return false;
    out.resize(count * nc);
    for (size_t i = 0; i < count; i++) {
        const uint8_t *e = base + i * stride;
        for (int c = 0; c < nc; c++) {
            float v = 0;
            if (ct == 5126) {
                std::memcpy(&v, e + c * 4, 4);
            } else if (ct == 5123) {
                uint16_t u;
                std::memcpy(&u, e + c * 2, 2);
                v = u / 65535.0f;
            } else if (ct == 5121) {
                v = e[c] / 255.0f;
            }
            out[i * nc + c] = v;
        }
    }
    return true;
}

// tg_readIndices (GLTFLoader.cpp:42-62): packed u32 / u16 / u8.
bool read_indices(const Gltf &g, int idx, std::vector<uint32_t> &out) {
    const uint8_t *base;
    size_t stride, count;
    int nc, ct;
    if (!accessor_view(g, idx, base, stride, count, nc, ct))
        return false;
    out.resize(count);
    for (size_t i = 0; i < count; i++) {
        if (ct == 5125) {
            uint32_t v;
            std::memcpy(&v, base + i * 4, 4);
            out[i] = v;
        } else if (ct == 5123) {
            uint16_t v;
            std::memcpy(&v, base + i * 2, 2);
            out[i] = v;
        } else {
            out[i] = base[i];
        }
    }
    return true;
}

struct LoadedImage {
    bool ok = false;
    int w = 0, h = 0;
    std::vector<uint8_t> rgba;
};

LoadedImage decode_image(const Gltf &g, int image) {
    LoadedImage out;
    const Json *img = g.doc.get("images") ? g.doc.get("images")->at((size_t) image) : nullptr;
    if (!img)
        return out;
    std::vector<uint8_t> bytes;
    const Json *uri = img->get("uri");
    if (uri && uri->kind == Json::Str) {
        if (!load_uri(g, uri->str, bytes))
            return out;
    } else {
        const int bvi = int_or(img->get("bufferView"), -1);
        const Json *bv =
            g.doc.get("bufferViews") ? g.doc.get("bufferViews")->at((size_t) bvi) : nullptr;
        if (!bv)
            return out;
        const int bi = int_or(bv->get("buffer"), -1);
        if (bi < 0 || bi >= (int) g.buffers.size())
            return out;
        const size_t off = (size_t) num_or(bv->get("byteOffset"), 0);
        const size_t len = (size_t) num_or(bv->get("byteLength"), 0);
        if (off + len > g.buffers[bi].size())
            return out;
        bytes.assign(g.buffers[bi].begin() + off, g.buffers[bi].begin() + off + len);
    }
    out.ok = decode_png(bytes.data(), bytes.size(), out.w, out.h, out.rgba);
    return out;
}

} // namespace
} // namespace prr

using namespace prr;

extern "C" int prr_scene_add_gltf(prr_scene *scene, const char *path, int material_type,
                                  int override_material, int *out_first, int *out_count,
                                  int *out_undecoded) {
    if (!scene || !path)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene and path are required");
    if (material_type < PRR_GLTF_DIFFUSE || material_type > PRR_GLTF_EMIT)
        return fail(PRR_ERR_INVALID_ARGUMENT, "unknown material type");
    Gltf g;
    std::string err;
    if (!open_gltf(path, g, err))
        return fail(PRR_ERR_INVALID_ARGUMENT, "glTF: " + err);
    // decoded textures are added once per image and shared between materials
    std::map<int, int> image_tex;
    std::map<int, LoadedImage> images;
    int undecoded = 0;
    auto texture_of = [&](const Json *info) -> int {
        if (!info)
            return -1;
        const int ti = int_or(info->get("index"), -1);
        const Json *tex = g.doc.get("textures") ? g.doc.get("textures")->at((size_t) ti) : nullptr;
        if (ti < 0 || !tex)
            return -1;
        const int src = int_or(tex->get("source"), -1);
        if (src < 0)
            return -1;
        auto it = image_tex.find(src);
        if (it != image_tex.end())
            return it->second;
        LoadedImage im = decode_image(g, src);
        int id = -1;
        if (!im.ok) {
            undecoded++;
        } else if (prr_scene_add_texture(scene, im.rgba.data(), im.w, im.h, 4, &id) != PRR_OK) {
            id = -1;
        }
        image_tex[src] = id;
        return id;
    };
    const Json *meshes = g.doc.get("meshes");
    const Json *mats = g.doc.get("materials");
    int first = -1, count = 0;
    for (size_t mi = 0; meshes && mi < meshes->size(); mi++) {
        const Json *prims = meshes->at(mi)->get("primitives");
        for (size_t pi = 0; prims && pi < prims->size(); pi++) {
            const Json *prim = prims->at(pi);
            if (int_or(prim->get("mode"), 4) != 4)
                continue;
            const Json *attrs = prim->get("attributes");
            const int ipos = attrs ? int_or(attrs->get("POSITION"), -1) : -1;
            std::vector<float> pos, nrm, uvs, tan;
            int nc = 0;
            if (ipos < 0 || !read_floats(g, ipos, pos, nc) || nc != 3)
                return fail(PRR_ERR_INVALID_ARGUMENT, "glTF: primitive without readable POSITION");
            int c2;
            const int inrm = int_or(attrs->get("NORMAL"), -1);
            if (inrm >= 0 && (!read_floats(g, inrm, nrm, c2) || c2 != 3))
                return fail(PRR_ERR_INVALID_ARGUMENT, "glTF: bad NORMAL accessor");
            const int iuv = int_or(attrs->get("TEXCOORD_0"), -1);
            if (iuv >= 0 && (!read_floats(g, iuv, uvs, c2) || c2 != 2))
                return fail(PRR_ERR_INVALID_ARGUMENT, "glTF: bad TEXCOORD_0 accessor");
            const int itan = int_or(attrs->get("TANGENT"), -1);
            if (itan >= 0 && (!read_floats(g, itan, tan, c2) || c2 != 4))
                return fail(PRR_ERR_INVALID_ARGUMENT, "glTF: bad TANGENT accessor");
            std::vector<uint32_t> idx;
            const int iidx = int_or(prim->get("indices"), -1);
            if (iidx >= 0) {
                if (!read_indices(g, iidx, idx))
                    return fail(PRR_ERR_INVALID_ARGUMENT, "glTF: bad index accessor");
            } else {
                idx.resize(pos.size() / 3);
                for (size_t i = 0; i < idx.size(); i++)
                    idx[i] = (uint32_t) i;
            }
            const size_t nv = pos.size() / 3;
            for (uint32_t k : idx)
                if (k >= nv || (!nrm.empty() && k >= nrm.size() / 3) ||
                    (!uvs.empty() && k >= uvs.size() / 2) || (!tan.empty() && k >= tan.size() / 4))
                    return fail(PRR_ERR_INVALID_ARGUMENT, "glTF: index out of range");
            // material (GLTFLoader.cpp:175-216): a DiffuseMaterial filled from
            // the glTF material, then recast to the requested class
            int material = override_material;
            if (material < 0) {
                float p[9] = {0.8f, 0.8f, 0.8f, 0.5f, 0.0f, 1.5f, 0.0f, 0.0f, 0.0f};
                int tex[4] = {-1, -1, -1, -1};
                const int gm = int_or(prim->get("material"), -1);
                const Json *m = (gm >= 0 && mats) ? mats->at((size_t) gm) : nullptr;
                if (m) { // loadMaterial (GLTFLoader.cpp:64-138)
                    const Json *pbr = m->get("pbrMetallicRoughness");
                    const Json *bc = pbr ? pbr->get("baseColorFactor") : nullptr;
                    for (int k = 0; k < 3; k++)
                        p[k] = (float) num_or(bc ? bc->at(k) : nullptr, 1.0);
                    p[4] = (float) num_or(pbr ? pbr->get("metallicFactor") : nullptr, 1.0);
                    p[3] = (float) num_or(pbr ? pbr->get("roughnessFactor") : nullptr, 1.0);
                    const Json *ef = m->get("emissiveFactor");
                    for (int k = 0; k < 3; k++)
                        p[6 + k] = (float) num_or(ef ? ef->at(k) : nullptr, 0.0);
                    tex[0] = texture_of(pbr ? pbr->get("baseColorTexture") : nullptr);
                    tex[1] = texture_of(pbr ? pbr->get("metallicRoughnessTexture") : nullptr);
                    tex[2] = texture_of(m->get("normalTexture"));
                    tex[3] = texture_of(m->get("emissiveTexture"));
                }
                int kind = PRR_MAT_DIFFUSE;
                if (material_type == PRR_GLTF_GLASS) {
                    // GlassMaterial: baseColor, emission and textures copied;
                    // roughness, metallic and ior keep the class defaults
                    kind = PRR_MAT_GLASS;
                    p[3] = 0.5f;
                    p[4] = 0.0f;
                    p[5] = 1.5f;
                } else if (material_type == PRR_GLTF_MIRROR) {
                    // MirrorMaterial: baseColor, emission and the emissive texture
                    kind = PRR_MAT_MIRROR;
                    p[3] = 0.5f;
                    p[4] = 0.0f;
                    p[5] = 1.5f;
                    tex[0] = tex[1] = tex[2] = -1;
                } else if (material_type == PRR_GLTF_EMIT) {
                    // EmissiveMaterial keeps every default, its emission
                    // included (GLTFLoader.cpp:209-212 assigns it to itself)
                    kind = PRR_MAT_EMISSIVE;
                    const float d[9] = {0.8f, 0.8f, 0.8f, 0.5f, 0.0f, 1.5f, 0.0f, 0.0f, 0.0f};
                    std::memcpy(p, d, sizeof(p));
                    tex[0] = tex[1] = tex[2] = tex[3] = -1;
                }
                if (int rc = prr_scene_add_material(scene, kind, p, &material))
                    return rc;
                if (tex[0] >= 0 || tex[1] >= 0 || tex[2] >= 0 || tex[3] >= 0)
                    if (int rc = prr_scene_set_material_textures(scene, material, tex[0], tex[1],
                                                                 tex[2], tex[3]))
                        return rc;
            }
            // triangles with per-corner data (GLTFLoader.cpp:221-262)
            const size_t nt = idx.size() / 3;
            if (nt == 0)
                continue;
            std::vector<float> v(nt * 9), cn, cu, ctan;
            if (!nrm.empty())
                cn.resize(nt * 9);
            if (!uvs.empty())
                cu.resize(nt * 6);
            if (!tan.empty())
                ctan.resize(nt * 12);
            for (size_t t = 0; t < nt; t++)
                for (int q = 0; q < 3; q++) {
                    const uint32_t k = idx[t * 3 + q];
                    std::memcpy(&v[t * 9 + q * 3], &pos[k * 3], 3 * sizeof(float));
                    if (!cn.empty()) { // normalize (GLTFLoader.cpp:237-239, Vector.hpp:103-111)
                        const float *r = &nrm[k * 3];
                        float *o = &cn[t * 9 + q * 3];
                        const float m2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                        o[0] = r[0];
                        o[1] = r[1];
                        o[2] = r[2];
                        if (m2 > 0) {
                            const float inv = 1 / sqrtf(m2);
                            o[0] = r[0] * inv;
                            o[1] = r[1] * inv;
                            o[2] = r[2] * inv;
                        }
                    }
                    if (!cu.empty())
                        std::memcpy(&cu[t * 6 + q * 2], &uvs[k * 2], 2 * sizeof(float));
                    if (!ctan.empty())
                        std::memcpy(&ctan[t * 12 + q * 4], &tan[k * 4], 4 * sizeof(float));
                }
            int obj = -1;
            if (int rc = prr_scene_add_mesh_attr(scene, v.data(), cn.empty() ? nullptr : cn.data(),
                                                 cu.empty() ? nullptr : cu.data(),
                                                 ctan.empty() ? nullptr : ctan.data(),
                                                 (int64_t) nt, material, &obj))
                return rc;
            if (first < 0)
                first = obj;
            count++;
        }
    }
    if (out_first)
        *out_first = first;
    if (out_count)
        *out_count = count;
    if (out_undecoded)
        *out_undecoded = undecoded;
    return PRR_OK;
}
