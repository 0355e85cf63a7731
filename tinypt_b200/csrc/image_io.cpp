// Image files of the CLI drop-in: the output formats of src/output.rs:59-132
// (PPM with exposure, tonemap and sRGB encoding; Radiance RGBE; OpenEXR in
// ACEScg) and the Radiance reader that env maps are loaded with
// (src/hdr.rs:20-87).  Host code.
#include "image_io.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace tpt {
namespace {

// linear_to_srgb (src/math.rs:185-191)
double linear_to_srgb(double c) { return c <= 0.0031308 ? 12.92 * c : 1.055 * std::pow(c, 1.0 / 2.4) - 0.055; }
double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

// Narkowicz's fitted ACES curve (src/output.rs:124-134).
double aces_fitted(double x) {
    x = std::max(x, 0.0);
    const double a = 2.51, b = 0.03, c = 2.43, d = 0.59, e = 0.14;
    return clamp01((x * (a * x + b)) / (x * (c * x + d) + e));
}

uint8_t to_u8(double x) { return (uint8_t)(linear_to_srgb(clamp01(x)) * 255.0 + 0.5); }

bool ends_with_ci(const std::string& s, const char* suf) {
    const size_t n = std::strlen(suf);
    if (s.size() < n) return false;
    for (size_t i = 0; i < n; ++i)
        if (std::tolower((unsigned char)s[s.size() - n + i]) != suf[i]) return false;
    return true;
}

// ---- Radiance RGBE ---------------------------------------------------------------
// One colour to shared-exponent bytes: the mantissas of the channels scaled
// by 2^-(e-8), e = floor(log2(max)) + 1 (src/hdr.rs color_to_rgbe).
void to_rgbe(const double* c, uint8_t* out) {
    const double r = std::max(c[0], 0.0), g = std::max(c[1], 0.0), b = std::max(c[2], 0.0);
    const double m = std::max(r, std::max(g, b));
    if (m < 1e-32) { out[0] = out[1] = out[2] = out[3] = 0; return; }
    const int e = (int)std::floor(std::log2(m)) + 1;
    const double f = std::ldexp(1.0, e - 8);
    out[0] = (uint8_t)std::min(std::max(r / f, 0.0), 255.0);
    out[1] = (uint8_t)std::min(std::max(g / f, 0.0), 255.0);
    out[2] = (uint8_t)std::min(std::max(b / f, 0.0), 255.0);
    out[3] = (uint8_t)(e + 128);
}

void from_rgbe(const uint8_t* p, double* c) {
    if (p[3] == 0) { c[0] = c[1] = c[2] = 0.0; return; }
    const double f = std::ldexp(1.0, (int)p[3] - 128 - 8);
    c[0] = p[0] * f; c[1] = p[1] * f; c[2] = p[2] * f;
}

// New-style RLE: per channel, runs of >= 4 equal bytes as (128 + n, byte),
// the rest as literal packets of up to 128 bytes.
void write_rle_scanline(std::ostream& o, const std::vector<uint8_t>& line, int w) {
    if (w < 8 || w > 0x7fff) {
        o.write((const char*)line.data(), (std::streamsize)line.size());
        return;
    }
    const uint8_t hdr[4] = {2, 2, (uint8_t)((w >> 8) & 0xff), (uint8_t)(w & 0xff)};
    o.write((const char*)hdr, 4);
    for (int ch = 0; ch < 4; ++ch) {
        auto at = [&](int x) { return line[(size_t)x * 4 + ch]; };
        int x = 0;
        while (x < w) {
            int run = 1;
            while (x + run < w && run < 127 && at(x + run) == at(x)) ++run;
            if (run >= 4) {
                const uint8_t pkt[2] = {(uint8_t)(128 + run), at(x)};
                o.write((const char*)pkt, 2);
                x += run;
                continue;
            }
            const int start = x;
            int n = 0;
            while (x < w && n < 128) {
                int look = 1;
                while (x + look < w && look < 127 && at(x + look) == at(x)) ++look;
                if (look >= 4) break;
                ++x;
                ++n;
            }
            const uint8_t cnt = (uint8_t)n;
            o.write((const char*)&cnt, 1);
            for (int i = 0; i < n; ++i) {
                const uint8_t v = at(start + i);
                o.write((const char*)&v, 1);
            }
        }
    }
}

void read_rle_scanline(std::istream& in, std::vector<uint8_t>& line, int w) {
    auto get = [&]() {
        const int c = in.get();
        if (c == EOF) throw std::runtime_error("truncated HDR data");
        return (uint8_t)c;
    };
    if (w < 8 || w > 0x7fff) {
        for (auto& b : line) b = get();
        return;
    }
    uint8_t h[4];
    for (auto& b : h) b = get();
    if (h[0] != 2 || h[1] != 2 || (((int)h[2] << 8) | h[3]) != w) {  // flat scanline
        std::memcpy(line.data(), h, 4);
        for (size_t i = 4; i < line.size(); ++i) line[i] = get();
        return;
    }
    for (int ch = 0; ch < 4; ++ch) {
        int x = 0;
        while (x < w) {
            const uint8_t code = get();
            if (code > 128) {
                const int n = code - 128;
                const uint8_t v = get();
                if (x + n > w) throw std::runtime_error("HDR run past the end of the scanline");
                for (int i = 0; i < n; ++i) line[(size_t)(x++) * 4 + ch] = v;
            } else {
                const int n = code;
                if (x + n > w) throw std::runtime_error("HDR literal past the end of the scanline");
                for (int i = 0; i < n; ++i) line[(size_t)(x++) * 4 + ch] = get();
                if (n == 0) throw std::runtime_error("empty HDR literal packet");
            }
        }
    }
}

// ---- ACEScg (src/aces.rs) ------------------------------------------------------
struct M3 { double m[3][3]; };
M3 mul(const M3& a, const M3& b) {
    M3 r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) r.m[i][j] += a.m[i][k] * b.m[k][j];
    return r;
}
void mulv(const M3& a, const double* v, double* o) {
    for (int i = 0; i < 3; ++i) o[i] = a.m[i][0] * v[0] + a.m[i][1] * v[1] + a.m[i][2] * v[2];
}
M3 inverse(const M3& a) {
    const double (*m)[3] = a.m;
    const double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                       m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                       m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    M3 r;
    r.m[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) / det;
    r.m[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det;
    r.m[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
    r.m[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) / det;
    r.m[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det;
    r.m[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det;
    r.m[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) / det;
    r.m[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det;
    r.m[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det;
    return r;
}
void xy_to_xyz(double x, double y, double* o) { o[0] = x / y; o[1] = 1.0; o[2] = (1.0 - x - y) / y; }
// RGB -> XYZ of a colour space given by its primaries and white point.
M3 rgb_to_xyz(const double prim[3][2], const double white[2]) {
    double r[3], g[3], b[3], w[3], s[3];
    xy_to_xyz(prim[0][0], prim[0][1], r);
    xy_to_xyz(prim[1][0], prim[1][1], g);
    xy_to_xyz(prim[2][0], prim[2][1], b);
    const M3 m{{{r[0], g[0], b[0]}, {r[1], g[1], b[1]}, {r[2], g[2], b[2]}}};
    xy_to_xyz(white[0], white[1], w);
    mulv(inverse(m), w, s);
    const M3 d{{{s[0], 0, 0}, {0, s[1], 0}, {0, 0, s[2]}}};
    return mul(m, d);
}
// Bradford chromatic adaptation between two XYZ whites.
M3 bradford(const double* src, const double* dst) {
    const M3 b{{{0.8951, 0.2664, -0.1614}, {-0.7502, 1.7135, 0.0367}, {0.0389, -0.0685, 1.0296}}};
    double s[3], d[3];
    mulv(b, src, s);
    mulv(b, dst, d);
    const M3 sc{{{d[0] / s[0], 0, 0}, {0, d[1] / s[1], 0}, {0, 0, d[2] / s[2]}}};
    return mul(inverse(b), mul(sc, b));
}
// Linear sRGB (Rec.709 primaries, D65) -> ACEScg (AP1 primaries, ACES white).
M3 srgb_to_acescg() {
    const double rec709[3][2] = {{0.64, 0.33}, {0.30, 0.60}, {0.15, 0.06}};
    const double d65[2] = {0.3127, 0.3290};
    const double ap1[3][2] = {{0.713, 0.293}, {0.165, 0.830}, {0.128, 0.044}};
    const double aces_w[2] = {0.32168, 0.33767};
    double w_src[3], w_dst[3];
    xy_to_xyz(d65[0], d65[1], w_src);
    xy_to_xyz(aces_w[0], aces_w[1], w_dst);
    return mul(inverse(rgb_to_xyz(ap1, aces_w)), mul(bradford(w_src, w_dst), rgb_to_xyz(rec709, d65)));
}

// ---- OpenEXR, single part, scanline, uncompressed, FLOAT B/G/R --------------------
void put_u32(std::string& s, uint32_t v) { for (int i = 0; i < 4; ++i) s.push_back((char)((v >> (8 * i)) & 0xff)); }
void put_i32(std::string& s, int32_t v) { put_u32(s, (uint32_t)v); }
void put_u64(std::string& s, uint64_t v) { for (int i = 0; i < 8; ++i) s.push_back((char)((v >> (8 * i)) & 0xff)); }
void put_f32(std::string& s, float f) { uint32_t u; std::memcpy(&u, &f, 4); put_u32(s, u); }
void attr(std::string& h, const char* name, const char* type, const std::string& value) {
    h += name; h.push_back('\0');
    h += type; h.push_back('\0');
    put_i32(h, (int32_t)value.size());
    h += value;
}

void write_exr(const std::string& path, int w, int h, const double* rgb) {
    const M3 m = srgb_to_acescg();
    std::string hdr;
    put_u32(hdr, 20000630u);  // magic
    put_u32(hdr, 2u);         // version 2, single-part scanline
    std::string ch;
    for (const char* name : {"B", "G", "R"}) {  // channels in alphabetical order
        ch += name; ch.push_back('\0');
        put_i32(ch, 2);                          // FLOAT
        ch.push_back(0); ch.push_back(0); ch.push_back(0); ch.push_back(0);  // pLinear + reserved
        put_i32(ch, 1); put_i32(ch, 1);          // sampling
    }
    ch.push_back('\0');
    attr(hdr, "channels", "chlist", ch);
    attr(hdr, "compression", "compression", std::string(1, '\0'));
    std::string box;
    put_i32(box, 0); put_i32(box, 0); put_i32(box, w - 1); put_i32(box, h - 1);
    attr(hdr, "dataWindow", "box2i", box);
    attr(hdr, "displayWindow", "box2i", box);
    attr(hdr, "lineOrder", "lineOrder", std::string(1, '\0'));
    std::string par; put_f32(par, 1.0f);
    attr(hdr, "pixelAspectRatio", "float", par);
    std::string swc; put_f32(swc, 0.0f); put_f32(swc, 0.0f);
    attr(hdr, "screenWindowCenter", "v2f", swc);
    std::string sww; put_f32(sww, 1.0f);
    attr(hdr, "screenWindowWidth", "float", sww);
    hdr.push_back('\0');
    const uint64_t line_bytes = (uint64_t)w * 3 * 4;
    const uint64_t first = hdr.size() + (uint64_t)h * 8;
    std::string table;
    for (int y = 0; y < h; ++y) put_u64(table, first + (uint64_t)y * (8 + line_bytes));
    std::ofstream o(path, std::ios::binary);
    if (!o) throw std::runtime_error("cannot create " + path);
    o << hdr << table;
    std::string line;
    for (int y = 0; y < h; ++y) {
        line.clear();
        put_i32(line, y);
        put_i32(line, (int32_t)line_bytes);
        std::vector<float> b(w), g(w), r(w);
        for (int x = 0; x < w; ++x) {
            double a[3];
            mulv(m, rgb + 3 * ((size_t)y * w + x), a);
            r[x] = (float)a[0]; g[x] = (float)a[1]; b[x] = (float)a[2];
        }
        for (float f : b) put_f32(line, f);
        for (float f : g) put_f32(line, f);
        for (float f : r) put_f32(line, f);
        o << line;
    }
    if (!o) throw std::runtime_error("write failed: " + path);
}

}  // namespace

void write_image(const std::string& path, int w, int h, const double* rgb, double exposure, int tonemap) {
    if (w <= 0 || h <= 0 || !rgb) throw std::runtime_error("bad image");
    if (ends_with_ci(path, ".exr")) {
        write_exr(path, w, h, rgb);
        return;
    }
    std::ofstream o(path, std::ios::binary);
    if (!o) throw std::runtime_error("cannot create " + path);
    if (ends_with_ci(path, ".hdr")) {  // scene-referred linear RGBE
        o << "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y " << h << " +X " << w << "\n";
        std::vector<uint8_t> line((size_t)w * 4);
        for (int y = 0; y < h; ++y) {
            for (int x = 0; x < w; ++x) to_rgbe(rgb + 3 * ((size_t)y * w + x), &line[(size_t)x * 4]);
            write_rle_scanline(o, line, w);
        }
    } else {  // PPM (P3): exposure, tonemap, sRGB, 8 bit
        const double scale = std::pow(2.0, exposure);
        std::string out = "P3\n" + std::to_string(w) + " " + std::to_string(h) + "\n255\n";
        for (int y = 0; y < h; ++y) {
            for (int x = 0; x < w; ++x) {
                const double* c = rgb + 3 * ((size_t)y * w + x);
                for (int k = 0; k < 3; ++k) {
                    double v = c[k] * scale;
                    v = tonemap == 1 ? aces_fitted(v) : v;
                    out += std::to_string((int)to_u8(clamp01(v)));
                    out += ' ';
                }
            }
            out += '\n';
        }
        o << out;
    }
    if (!o) throw std::runtime_error("write failed: " + path);
}

void read_hdr(const std::string& path, int& w, int& h, std::vector<double>& rgb) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + path);
    std::string line;
    std::getline(in, line);
    if (line.rfind("#?RADIANCE", 0) != 0 && line.rfind("#?RGBE", 0) != 0) throw std::runtime_error("invalid HDR header");
    for (;;) {
        if (!std::getline(in, line)) throw std::runtime_error("missing HDR resolution");
        if (line.find_first_not_of(" \t\r") == std::string::npos) break;
    }
    if (!std::getline(in, line)) throw std::runtime_error("missing HDR resolution");
    std::istringstream rs(line);
    std::string ys, xs;
    long hh = 0, ww = 0;
    if (!(rs >> ys >> hh >> xs >> ww) || hh <= 0 || ww <= 0 || ys.size() != 2 || xs.size() != 2)
        throw std::runtime_error("invalid HDR resolution line");
    w = (int)ww;
    h = (int)hh;
    rgb.assign((size_t)w * h * 3, 0.0);
    std::vector<uint8_t> sl((size_t)w * 4);
    for (int y = 0; y < h; ++y) {
        read_rle_scanline(in, sl, w);
        for (int x = 0; x < w; ++x) {
            const int sx = xs[0] == '-' ? w - 1 - x : x;
            const int dy = ys[0] == '-' ? y : h - 1 - y;
            from_rgbe(&sl[(size_t)sx * 4], &rgb[3 * ((size_t)dy * w + x)]);
        }
    }
}

}  // namespace tpt
