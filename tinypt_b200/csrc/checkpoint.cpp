// Checkpoint files compatible with the reference (src/checkpoint.rs:1-138):
// "HYPCKPT\0", u32 version 1, u64 scene hash, u32 width, u32 height, u64
// next task id, then acc (w*h x 3 f64) and acc_w (w*h f64), little endian,
// written to path.tmp and renamed.  Tasks are the film's tiles in the
// reference's order (src/render.rs:75-100, Morton keys :284-299), so a
// checkpoint taken by either renderer resumes in the other.  Host code.
#include "checkpoint.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <stdexcept>

namespace tpt {
namespace {

const char kMagic[8] = {'H', 'Y', 'P', 'C', 'K', 'P', 'T', '\0'};
constexpr uint32_t kVersion = 1;

uint64_t spread_bits(uint64_t v) {  // interleave_bits: a zero bit between each of the low 32 bits
    uint64_t x = v & 0x00000000ffffffffull;
    x = (x | (x << 16)) & 0x0000ffff0000ffffull;
    x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
    x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}

template <class T>
void put(std::ofstream& o, T v) {
    unsigned char b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));  // little-endian host
    o.write(reinterpret_cast<const char*>(b), sizeof(T));
}
template <class T>
bool get(std::ifstream& in, T& v) {
    unsigned char b[sizeof(T)];
    if (!in.read(reinterpret_cast<char*>(b), sizeof(T))) return false;
    std::memcpy(&v, b, sizeof(T));
    return true;
}

}  // namespace

std::vector<TileRect> film_tiles(int w, int h, int tile, bool morton) {
    if (w <= 0 || h <= 0 || tile <= 0) throw std::runtime_error("bad tile grid");
    std::vector<TileRect> t;
    for (int y = 0; y < h; y += tile)
        for (int x = 0; x < w; x += tile) t.push_back({x, y, std::min(x + tile, w), std::min(y + tile, h)});
    if (morton) {
        const uint64_t tx = (uint64_t)((w + tile - 1) / tile), ty = (uint64_t)((h + tile - 1) / tile);
        auto key = [&](const TileRect& r) {
            const uint64_t x = std::min((uint64_t)(r.x0 / tile), tx ? tx - 1 : 0);
            const uint64_t y = std::min((uint64_t)(r.y0 / tile), ty ? ty - 1 : 0);
            return spread_bits(x) | (spread_bits(y) << 1);
        };
        std::stable_sort(t.begin(), t.end(), [&](const TileRect& a, const TileRect& b) { return key(a) < key(b); });
    }
    return t;
}

void save_checkpoint(const std::string& path, uint64_t scene_hash, int w, int h, uint64_t next_id,
                     const double* acc, const double* acc_w) {
    const std::string tmp = path + ".tmp";
    {
        std::ofstream o(tmp, std::ios::binary);
        if (!o) throw std::runtime_error("cannot create " + tmp);
        o.write(kMagic, 8);
        put<uint32_t>(o, kVersion);
        put<uint64_t>(o, scene_hash);
        put<uint32_t>(o, (uint32_t)w);
        put<uint32_t>(o, (uint32_t)h);
        put<uint64_t>(o, next_id);
        const size_t n = (size_t)w * (size_t)h;
        o.write(reinterpret_cast<const char*>(acc), (std::streamsize)(3 * n * sizeof(double)));
        o.write(reinterpret_cast<const char*>(acc_w), (std::streamsize)(n * sizeof(double)));
        if (!o) throw std::runtime_error("write failed: " + tmp);
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) throw std::runtime_error("cannot rename " + tmp);
}

bool load_checkpoint(const std::string& path, uint64_t scene_hash, int w, int h, uint64_t& next_id, double* acc,
                     double* acc_w) {
    // src/checkpoint.rs:86-138: no file -> None; a header field that differs
    // -> None; a file that cannot be opened or ends early (header included)
    // -> an I/O error.
    std::error_code ec;
    if (!std::filesystem::exists(path, ec)) return false;
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open checkpoint " + path);
    auto need = [&](bool ok) {
        if (!ok) throw std::runtime_error("truncated checkpoint " + path);
    };
    char magic[8];
    need((bool)in.read(magic, 8));
    if (std::memcmp(magic, kMagic, 8) != 0) return false;
    uint32_t ver = 0, fw = 0, fh = 0;
    uint64_t hash = 0, nid = 0;
    need(get(in, ver));
    if (ver != kVersion) return false;
    need(get(in, hash));
    if (hash != scene_hash) return false;
    need(get(in, fw));
    need(get(in, fh));
    if ((int)fw != w || (int)fh != h) return false;
    need(get(in, nid));
    const size_t n = (size_t)w * (size_t)h;
    std::vector<double> a(3 * n), aw(n);
    need((bool)in.read(reinterpret_cast<char*>(a.data()), (std::streamsize)(a.size() * sizeof(double))));
    need((bool)in.read(reinterpret_cast<char*>(aw.data()), (std::streamsize)(aw.size() * sizeof(double))));
    std::memcpy(acc, a.data(), a.size() * sizeof(double));
    std::memcpy(acc_w, aw.data(), aw.size() * sizeof(double));
    next_id = nid;
    return true;
}

void merge_tiles(const std::vector<TileRect>& tiles, size_t first, int w, const double* acc_new,
                 const double* w_new, double* acc, double* acc_w) {
    for (size_t k = first; k < tiles.size(); ++k) {
        const TileRect& r = tiles[k];
        for (int y = r.y0; y < r.y1; ++y)
            for (int x = r.x0; x < r.x1; ++x) {
                const size_t i = (size_t)y * (size_t)w + (size_t)x;
                acc[3 * i] += acc_new[3 * i];
                acc[3 * i + 1] += acc_new[3 * i + 1];
                acc[3 * i + 2] += acc_new[3 * i + 2];
                acc_w[i] += w_new[i];
            }
    }
}

}  // namespace tpt
