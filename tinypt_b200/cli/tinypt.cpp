// Command-line renderer with the reference's flags (src/main.rs:22-101):
// loads a Mitsuba XML scene (--scene) or builds the built-in scene, renders
// it on the GPU through the C ABI, resolves the film and writes the image in
// the format of the output path's extension.
//
//   tinypt [--scene FILE] [--out|-o FILE] [--spp N] [--env FILE.hdr] [--no-env]
//          [--denoise|--no-denoise] [--adaptive|--no-adaptive]
//          [--adaptive-min-spp N] [--adaptive-threshold X] [--seed N]
//          [--tonemap none|aces] [--exposure EV] [--morton|--no-morton]
//          [--mode wavefront|plain] [--dry-run]
//
// --mode and --dry-run are this renderer's own: --mode picks the FP32
// wavefront form (default) or the plain f64 form; --dry-run prints the
// configuration after the scene is loaded and exits before any GPU work.
// Flag values parse as Rust's str::parse does in the reference (no
// surrounding spaces, no hex floats, a value out of range is ignored);
// unknown flags are ignored.  Denoising (Intel OIDN in the reference) is not
// available and is skipped with a notice.
#include <cerrno>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cctype>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/tinypt_cuda.h"

namespace {

int fail(const char* what) {
    std::fprintf(stderr, "%s: %s\n", what, tpt_last_error());
    return 1;
}

// usize / u64 parse: decimal digits with an optional '+', nothing else.
bool parse_ull(const char* s, unsigned long long& v) {
    const char* d = s[0] == '+' ? s + 1 : s;
    if (*d < '0' || *d > '9') return false;
    char* end = nullptr;
    errno = 0;
    v = std::strtoull(d, &end, 10);
    return end && *end == '\0' && errno != ERANGE;
}
// f64 parse: a decimal number, inf or nan with an optional sign; strtod
// would also take leading spaces and hex floats.
bool parse_d(const char* s, double& v) {
    const char* d = (s[0] == '+' || s[0] == '-') ? s + 1 : s;
    if (*d == '\0' || std::isspace((unsigned char)*d) || (d[0] == '0' && (d[1] == 'x' || d[1] == 'X'))) return false;
    char* end = nullptr;
    v = std::strtod(s, &end);
    return end && end != s && *end == '\0';
}
int clamp_int(unsigned long long u) { return (int)(u < 1 ? 1 : (u > (unsigned long long)INT_MAX ? INT_MAX : u)); }

}  // namespace

int main(int argc, char** argv) {
    tpt_render_config cfg{};  // RenderConfig::default (src/config.rs:69-92)
    cfg.width = 1920;
    cfg.height = 1080;
    cfg.spp = 512;
    cfg.max_bounces = 8;
    cfg.rr_start = 3;
    cfg.tile = 16;
    cfg.adaptive_enabled = 0;
    cfg.adaptive_min_spp = 8;
    cfg.adaptive_threshold = 0.02;
    cfg.morton_enabled = 1;
    cfg.mode = TPT_MODE_WAVEFRONT_FP32;
    cfg.seed = 0;
    std::string out = "out.ppm", scene_path, env_path;
    bool denoise = true;
    int tonemap = 1;  // aces
    double exposure = 0.0;
    long long spp_override = -1;
    bool dry_run = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> const char* { return i + 1 < argc ? argv[++i] : nullptr; };
        unsigned long long u;
        double d;
        if (a == "--spp") {
            if (const char* v = next())
                if (parse_ull(v, u)) { cfg.spp = clamp_int(u); spp_override = cfg.spp; }
        } else if (a == "--out" || a == "-o") {
            if (const char* v = next()) out = v;
        } else if (a == "--env") {
            if (const char* v = next()) env_path = v;
        } else if (a == "--scene") {
            if (const char* v = next()) scene_path = v;
        } else if (a == "--no-env") {
            env_path.clear();
        } else if (a == "--denoise") {
            denoise = true;
        } else if (a == "--no-denoise") {
            denoise = false;
        } else if (a == "--adaptive") {
            cfg.adaptive_enabled = 1;
        } else if (a == "--no-adaptive") {
            cfg.adaptive_enabled = 0;
        } else if (a == "--adaptive-min-spp") {
            if (const char* v = next())
                if (parse_ull(v, u)) cfg.adaptive_min_spp = clamp_int(u);
        } else if (a == "--adaptive-threshold") {
            if (const char* v = next())
                if (parse_d(v, d)) cfg.adaptive_threshold = d >= 0.0 ? d : 0.0;  // f64::max(d, 0.0), NaN -> 0
        } else if (a == "--seed") {
            if (const char* v = next())
                if (parse_ull(v, u)) cfg.seed = u;
        } else if (a == "--tonemap") {
            if (const char* v = next()) {
                if (std::strcmp(v, "none") == 0) tonemap = 0;
                else if (std::strcmp(v, "aces") == 0) tonemap = 1;
            }
        } else if (a == "--exposure") {
            if (const char* v = next())
                if (parse_d(v, d)) exposure = d;
        } else if (a == "--morton") {
            cfg.morton_enabled = 1;
        } else if (a == "--no-morton") {
            cfg.morton_enabled = 0;
        } else if (a == "--mode") {
            if (const char* v = next()) {
                if (std::strcmp(v, "plain") == 0) cfg.mode = TPT_MODE_PLAIN_F64;
                else if (std::strcmp(v, "wavefront") == 0) cfg.mode = TPT_MODE_WAVEFRONT_FP32;
            }
        } else if (a == "--dry-run") {
            dry_run = true;
        }
    }

    void* loaded = nullptr;
    if (!scene_path.empty()) {
        if (tpt_scene_load_xml(scene_path.c_str(), &cfg, &loaded) != TPT_OK) return fail("load scene");
        if (spp_override > 0) cfg.spp = (int)spp_override;
    } else {
        if (tpt_scene_default(&cfg, env_path.empty() ? nullptr : env_path.c_str(), &loaded) != TPT_OK)
            return fail("build scene");
    }
    for (int64_t k = 0; k < tpt_loaded_warning_count(loaded); ++k)
        std::fprintf(stderr, "[mitsuba] warning: %s\n", tpt_loaded_warning(loaded, k));
    if (dry_run) {
        std::printf("width=%d height=%d spp=%d max_bounces=%d rr_start=%d tile=%d adaptive=%d adaptive_min_spp=%d "
                    "adaptive_threshold=%.17g morton=%d seed=%llu mode=%s denoise=%d tonemap=%s exposure=%.17g "
                    "out=%s env=%s scene=%s\n",
                    cfg.width, cfg.height, cfg.spp, cfg.max_bounces, cfg.rr_start, cfg.tile, cfg.adaptive_enabled,
                    cfg.adaptive_min_spp, cfg.adaptive_threshold, cfg.morton_enabled, (unsigned long long)cfg.seed,
                    cfg.mode == TPT_MODE_PLAIN_F64 ? "plain" : "wavefront", denoise ? 1 : 0,
                    tonemap ? "aces" : "none", exposure, out.c_str(),
                    scene_path.empty() && !env_path.empty() ? env_path.c_str() : "-",
                    scene_path.empty() ? "-" : scene_path.c_str());
        tpt_loaded_destroy(loaded);
        return 0;
    }

    void* scene = nullptr;
    if (tpt_scene_create(tpt_loaded_desc(loaded), &scene) != TPT_OK) return fail("upload scene");
    const size_t n = (size_t)cfg.width * (size_t)cfg.height;
    std::vector<double> acc(3 * n), acc_w(n);
    std::fprintf(stderr, "Rendering %dx%d, %d spp, max depth %d (%s)\n", cfg.width, cfg.height, cfg.spp,
                 cfg.max_bounces, cfg.mode == TPT_MODE_PLAIN_F64 ? "plain f64" : "FP32 wavefront");
    const auto t0 = std::chrono::steady_clock::now();
    tpt_stats st{};
    const int rc = tpt_render(scene, &cfg, acc.data(), acc_w.data(), &st);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    tpt_scene_destroy(scene);
    tpt_loaded_destroy(loaded);
    if (rc != TPT_OK) return fail("render");
    std::fprintf(stderr, "Done in %.2fs\n", secs);

    std::vector<double> px(3 * n);  // resolve_pixels (src/output.rs:96-102)
    for (size_t i = 0; i < n; ++i) {
        const double w = acc_w[i] > 1.0 ? acc_w[i] : 1.0;
        for (int c = 0; c < 3; ++c) px[3 * i + c] = acc[3 * i + c] / w;
    }
    if (denoise) std::fprintf(stderr, "Denoising skipped: Intel OIDN is not available in this build\n");
    if (tpt_write_image(out.c_str(), cfg.width, cfg.height, px.data(), exposure, tonemap) != TPT_OK)
        return fail("write image");
    return 0;
}
