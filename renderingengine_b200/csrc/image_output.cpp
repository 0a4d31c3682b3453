// Image outputs of a rendered film (host code, no device work; read the film
// with re_renderer_read_film first):
//   - re_image_hash_linear_rgb: the linear-RGB identity hash of
//     HashLinearRgbPixels (src/rt/cpu/ImageOutput.cpp:343-380): 64-bit
//     FNV-1a (Fowler, Noll, Vo) over the domain tag "RERGB" 1 3 0, the width
//     and height as little-endian 32-bit words, then every component's IEEE
//     bits little-endian with -0 folded to +0;
//   - re_image_write_exr: a 32-bit float RGB OpenEXR file, as
//     WriteLinearRgbExr (ImageOutput.cpp:156-216) produces with TinyEXR:
//     single-part scanline, channels B, G, R (FLOAT), ZIP compression in
//     blocks of 16 scanlines (OpenEXR's byte split and delta predictor,
//     then zlib), the raw block where compression does not shrink it.
// Both validate the image as ValidateLinearRgb (ImageOutput.cpp:28-79):
// non-zero dimensions, width x height x 3 components, every one finite.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "re_b200.h"
#include "runtime.h"

namespace re {
namespace {

constexpr uint64_t kFnvOffsetBasis = 14695981039346656037ull;
constexpr uint64_t kFnvPrime = 1099511628211ull;

re_status validate_rgb(uint32_t width, uint32_t height, const float* rgb, uint64_t component_count) {
    if (width == 0u || height == 0u) return set_error(RE_INVALID_ARGUMENT, "Image dimensions must both be greater than zero.");
    const uint64_t expected = uint64_t(width) * height * 3u;
    if (component_count != expected)
        return set_error(RE_INVALID_ARGUMENT, "Linear RGB span contains " + std::to_string(component_count) +
                                                  " components; expected " + std::to_string(expected) + ".");
    if (rgb == nullptr) return set_error(RE_INVALID_ARGUMENT, "Linear RGB pointer is null.");
    for (uint64_t i = 0; i < component_count; ++i)
        if (!std::isfinite(rgb[i]))
            return set_error(RE_INVALID_ARGUMENT, "Linear RGB component " + std::to_string(i) + " is NaN or infinite.");
    return RE_SUCCESS;
}

inline void fnv_byte(uint64_t& h, uint8_t b) {
    h ^= uint64_t(b);
    h *= kFnvPrime;
}

inline void fnv_u32(uint64_t& h, uint32_t v) {
    for (int k = 0; k < 4; ++k) fnv_byte(h, uint8_t((v >> (8 * k)) & 0xffu));
}

// Little-endian writers for the EXR header and chunks.
void put_bytes(std::vector<uint8_t>& o, const void* p, size_t n) {
    const auto* b = static_cast<const uint8_t*>(p);
    o.insert(o.end(), b, b + n);
}
void put_i32(std::vector<uint8_t>& o, int32_t v) {
    for (int k = 0; k < 4; ++k) o.push_back(uint8_t((uint32_t(v) >> (8 * k)) & 0xffu));
}
void put_f32(std::vector<uint8_t>& o, float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    put_i32(o, int32_t(u));
}
void put_cstr(std::vector<uint8_t>& o, const char* s) { put_bytes(o, s, std::strlen(s) + 1); }
void put_attr(std::vector<uint8_t>& o, const char* name, const char* type, const std::vector<uint8_t>& value) {
    put_cstr(o, name);
    put_cstr(o, type);
    put_i32(o, int32_t(value.size()));
    o.insert(o.end(), value.begin(), value.end());
}

constexpr int kZipLines = 16;        // OpenEXR ZIP_COMPRESSION block height
constexpr uint8_t kZipCompression = 3;
constexpr int32_t kPixelFloat = 2;

// OpenEXR ZIP block: bytes split into even / odd halves, a delta predictor
// (d = t[i] - t[i-1] + 128, mod 256), then zlib (fastest level; any level
// decodes the same).  Returns false when zlib
// fails; `out` empty means "store the raw block".
bool zip_block(const std::vector<uint8_t>& raw, std::vector<uint8_t>& out) {
    const size_t n = raw.size();
    std::vector<uint8_t> t(n);
    size_t a = 0, b = (n + 1) / 2;
    for (size_t i = 0; i < n; ++i) {
        if ((i & 1u) == 0u) t[a++] = raw[i];
        else t[b++] = raw[i];
    }
    int p = n ? t[0] : 0;
    for (size_t i = 1; i < n; ++i) {
        const int d = int(t[i]) - p + (128 + 256);
        p = t[i];
        t[i] = uint8_t(d & 0xff);
    }
    uLongf size = compressBound(uLong(n));
    out.resize(size);
    if (compress2(out.data(), &size, t.data(), uLong(n), Z_BEST_SPEED) != Z_OK) return false;
    out.resize(size);
    if (size >= n) out.clear();
    return true;
}

}  // namespace
}  // namespace re

extern "C" {

RE_API re_status re_image_hash_linear_rgb(uint32_t width, uint32_t height, const float* rgb, uint64_t component_count,
                                          uint64_t* hash_out) {
    using namespace re;
    if (hash_out == nullptr) return set_error(RE_INVALID_ARGUMENT, "hash output pointer is null");
    *hash_out = 0u;
    const re_status st = validate_rgb(width, height, rgb, component_count);
    if (st != RE_SUCCESS) return st;
    uint64_t h = kFnvOffsetBasis;
    const uint8_t domain[8] = {'R', 'E', 'R', 'G', 'B', 1u, 3u, 0u};
    for (uint8_t b : domain) fnv_byte(h, b);
    fnv_u32(h, width);
    fnv_u32(h, height);
    for (uint64_t i = 0; i < component_count; ++i) {
        const float c = rgb[i] == 0.0f ? 0.0f : rgb[i];
        uint32_t u;
        std::memcpy(&u, &c, 4);
        fnv_u32(h, u);
    }
    *hash_out = h;
    return clear_error();
}

RE_API re_status re_image_write_exr(const char* path, uint32_t width, uint32_t height, const float* rgb,
                                    uint64_t component_count) {
    using namespace re;
    const re_status st = validate_rgb(width, height, rgb, component_count);
    if (st != RE_SUCCESS) return st;
    if (path == nullptr || path[0] == '\0') return set_error(RE_INVALID_ARGUMENT, "EXR output path must not be empty.");
    if (width > 0x7fffffffu || height > 0x7fffffffu)
        return set_error(RE_INVALID_ARGUMENT, "EXR dimensions exceed the signed 32-bit limit.");
    std::vector<uint8_t> f;
    put_i32(f, 20000630);  // magic
    put_i32(f, 2);         // version 2, single-part scanline
    std::vector<uint8_t> v;
    for (const char* name : {"B", "G", "R"}) {
        put_cstr(v, name);
        put_i32(v, kPixelFloat);
        const uint8_t linear_reserved[4] = {0, 0, 0, 0};
        put_bytes(v, linear_reserved, 4);
        put_i32(v, 1);  // x sampling
        put_i32(v, 1);  // y sampling
    }
    v.push_back(0);
    put_attr(f, "channels", "chlist", v);
    put_attr(f, "compression", "compression", {kZipCompression});
    v.clear();
    put_i32(v, 0);
    put_i32(v, 0);
    put_i32(v, int32_t(width - 1u));
    put_i32(v, int32_t(height - 1u));
    put_attr(f, "dataWindow", "box2i", v);
    put_attr(f, "displayWindow", "box2i", v);
    put_attr(f, "lineOrder", "lineOrder", {0});
    v.clear();
    put_f32(v, 1.0f);
    put_attr(f, "pixelAspectRatio", "float", v);
    v.clear();
    put_f32(v, 0.0f);
    put_f32(v, 0.0f);
    put_attr(f, "screenWindowCenter", "v2f", v);
    v.clear();
    put_f32(v, 1.0f);
    put_attr(f, "screenWindowWidth", "float", v);
    f.push_back(0);  // end of header
    const uint32_t blocks = (height + kZipLines - 1u) / kZipLines;
    const size_t table = f.size();
    f.resize(table + size_t(blocks) * 8u);
    std::vector<uint8_t> raw, zipped;
    for (uint32_t k = 0; k < blocks; ++k) {
        const uint32_t y0 = k * kZipLines, lines = std::min<uint32_t>(kZipLines, height - y0);
        // Scanline by scanline, each channel's row of little-endian floats.
        raw.resize(size_t(lines) * width * 3u * 4u);
        uint8_t* dst = raw.data();
        for (uint32_t y = y0; y < y0 + lines; ++y)
            for (int c = 2; c >= 0; --c)  // B, G, R
                for (uint32_t x = 0; x < width; ++x, dst += 4)
                    std::memcpy(dst, &rgb[(size_t(y) * width + x) * 3u + size_t(c)], 4);
        if (!zip_block(raw, zipped)) return set_error(RE_RECORDING_FAILED, "zlib failed to compress an EXR block");
        const std::vector<uint8_t>& data = zipped.empty() ? raw : zipped;
        const uint64_t offset = f.size();
        for (int b = 0; b < 8; ++b) f[table + size_t(k) * 8u + size_t(b)] = uint8_t((offset >> (8 * b)) & 0xffu);
        put_i32(f, int32_t(y0));
        put_i32(f, int32_t(data.size()));
        f.insert(f.end(), data.begin(), data.end());
    }
    std::FILE* out = std::fopen(path, "wb");
    if (out == nullptr) return set_error(RE_INVALID_ARGUMENT, std::string("cannot open EXR output: ") + path);
    const bool ok = std::fwrite(f.data(), 1, f.size(), out) == f.size();
    const bool closed = std::fclose(out) == 0;
    if (!ok || !closed) return set_error(RE_RECORDING_FAILED, std::string("failed while writing EXR output: ") + path);
    return clear_error();
}

}  // extern "C"
