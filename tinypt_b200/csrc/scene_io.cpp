// Scene ingestion of the CLI drop-in (host code).  A small XML reader plus
// the Mitsuba subset rules of src/mitsuba.rs:137-595, the OBJ reader of
// src/obj_loader.rs:11-47 and the built-in scene of src/scene.rs:26-95.
// Transforms and camera inputs are computed in f64 in the reference's
// operation order, so instances and cameras match the reference bit for bit.
#include "scene_io.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>

#include "image_io.hpp"

namespace tpt {
namespace {

constexpr double kPi = 3.14159265358979323846;

// ---- XML ---------------------------------------------------------------------------
struct Element {
    std::string tag;
    std::map<std::string, std::string> attrs;
    std::vector<Element> children;
    const std::string* attr(const std::string& k) const {
        auto it = attrs.find(k);
        return it == attrs.end() ? nullptr : &it->second;
    }
    std::string type() const {
        const std::string* t = attr("type");
        return t ? *t : std::string();
    }
    const Element* child(const std::string& tag_) const {
        for (const Element& c : children)
            if (c.tag == tag_) return &c;
        return nullptr;
    }
    const Element* prop(const std::string& tag_, const std::string& name) const {
        for (const Element& c : children) {
            const std::string* n = c.attr("name");
            if (c.tag == tag_ && n && *n == name) return &c;
        }
        return nullptr;
    }
};

std::string unescape(const std::string& s) {
    std::string o;
    for (size_t i = 0; i < s.size(); ++i) {
        if (s[i] != '&') { o.push_back(s[i]); continue; }
        const size_t e = s.find(';', i);
        if (e == std::string::npos) throw std::runtime_error("bad XML entity");
        const std::string ent = s.substr(i + 1, e - i - 1);
        if (ent == "amp") o.push_back('&');
        else if (ent == "lt") o.push_back('<');
        else if (ent == "gt") o.push_back('>');
        else if (ent == "quot") o.push_back('"');
        else if (ent == "apos") o.push_back('\'');
        else if (!ent.empty() && ent[0] == '#') {
            const long v = ent.size() > 1 && ent[1] == 'x' ? std::strtol(ent.c_str() + 2, nullptr, 16)
                                                           : std::strtol(ent.c_str() + 1, nullptr, 10);
            if (v <= 0 || v > 127) throw std::runtime_error("unsupported XML character reference");
            o.push_back((char)v);
        } else {
            throw std::runtime_error("unknown XML entity &" + ent + ";");
        }
        i = e;
    }
    return o;
}

class XmlReader {
  public:
    explicit XmlReader(const std::string& s) : s_(s) {}
    Element parse() {
        std::vector<Element> stack;
        Element root;
        bool have_root = false;
        while (true) {
            const size_t lt = s_.find('<', p_);
            if (lt == std::string::npos) break;  // trailing text
            p_ = lt;
            if (s_.compare(p_, 4, "<!--") == 0) {
                const size_t e = s_.find("-->", p_);
                if (e == std::string::npos) throw std::runtime_error("unterminated XML comment");
                p_ = e + 3;
                continue;
            }
            if (s_.compare(p_, 2, "<?") == 0) {
                const size_t e = s_.find("?>", p_);
                if (e == std::string::npos) throw std::runtime_error("unterminated XML declaration");
                p_ = e + 2;
                continue;
            }
            if (s_.compare(p_, 9, "<![CDATA[") == 0) {
                const size_t e = s_.find("]]>", p_);
                if (e == std::string::npos) throw std::runtime_error("unterminated CDATA");
                p_ = e + 3;
                continue;
            }
            if (s_.compare(p_, 2, "<!") == 0) {  // DOCTYPE
                const size_t e = s_.find('>', p_);
                if (e == std::string::npos) throw std::runtime_error("unterminated XML markup");
                p_ = e + 1;
                continue;
            }
            if (s_.compare(p_, 2, "</") == 0) {
                const size_t e = s_.find('>', p_);
                if (e == std::string::npos) throw std::runtime_error("unterminated end tag");
                const std::string name = trim(s_.substr(p_ + 2, e - p_ - 2));
                p_ = e + 1;
                if (stack.empty() || stack.back().tag != name) throw std::runtime_error("unbalanced XML");
                Element el = std::move(stack.back());
                stack.pop_back();
                attach(stack, root, have_root, std::move(el));
                continue;
            }
            bool empty = false;
            Element el = read_start(empty);
            if (empty) attach(stack, root, have_root, std::move(el));
            else stack.push_back(std::move(el));
        }
        if (!stack.empty()) throw std::runtime_error("unbalanced XML");
        if (!have_root) throw std::runtime_error("empty XML");
        return root;
    }

  private:
    static std::string trim(const std::string& t) {
        const size_t a = t.find_first_not_of(" \t\r\n");
        if (a == std::string::npos) return "";
        const size_t b = t.find_last_not_of(" \t\r\n");
        return t.substr(a, b - a + 1);
    }
    static void attach(std::vector<Element>& stack, Element& root, bool& have_root, Element&& el) {
        if (!stack.empty()) stack.back().children.push_back(std::move(el));
        else { root = std::move(el); have_root = true; }
    }
    static bool name_char(char c) {
        return std::isalnum((unsigned char)c) || c == '_' || c == '-' || c == ':' || c == '.';
    }
    Element read_start(bool& empty) {
        ++p_;  // '<'
        Element el;
        while (p_ < s_.size() && name_char(s_[p_])) el.tag.push_back(s_[p_++]);
        if (el.tag.empty()) throw std::runtime_error("bad XML tag");
        while (true) {
            while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_;
            if (p_ >= s_.size()) throw std::runtime_error("unterminated start tag");
            if (s_[p_] == '/') {
                if (p_ + 1 >= s_.size() || s_[p_ + 1] != '>') throw std::runtime_error("bad empty tag");
                p_ += 2;
                empty = true;
                return el;
            }
            if (s_[p_] == '>') {
                ++p_;
                return el;
            }
            std::string key;
            while (p_ < s_.size() && name_char(s_[p_])) key.push_back(s_[p_++]);
            if (key.empty()) throw std::runtime_error("bad XML attribute");
            while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_;
            if (p_ >= s_.size() || s_[p_] != '=') throw std::runtime_error("XML attribute without value");
            ++p_;
            while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_;
            if (p_ >= s_.size() || (s_[p_] != '"' && s_[p_] != '\'')) throw std::runtime_error("unquoted XML attribute");
            const char q = s_[p_++];
            const size_t e = s_.find(q, p_);
            if (e == std::string::npos) throw std::runtime_error("unterminated XML attribute");
            el.attrs[key] = unescape(s_.substr(p_, e - p_));
            p_ = e + 1;
        }
    }
    const std::string& s_;
    size_t p_ = 0;
};

// ---- values (src/mitsuba.rs:46-122) ---------------------------------------------------
bool parse_f64(const std::string& s0, double& out) {
    const size_t a = s0.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return false;
    const size_t b = s0.find_last_not_of(" \t\r\n");
    const std::string s = s0.substr(a, b - a + 1);
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (end != s.c_str() + s.size()) return false;
    out = v;
    return true;
}
bool parse_usize(const std::string& s0, long long& out) {
    const size_t a = s0.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return false;
    const size_t b = s0.find_last_not_of(" \t\r\n");
    const std::string s = s0.substr(a, b - a + 1);
    if (s.empty() || s.find_first_not_of("0123456789+") != std::string::npos || s.find('+', 1) != std::string::npos)
        return false;
    out = std::atoll(s.c_str());
    return true;
}
struct V3 { double x, y, z; };
bool parse_vec3(const std::string& s, V3& v) {
    std::vector<double> parts;
    std::string tok;
    auto flush = [&]() -> bool {
        if (tok.find_first_not_of(" \t\r\n") == std::string::npos) { tok.clear(); return true; }
        double d;
        if (!parse_f64(tok, d)) return false;
        parts.push_back(d);
        tok.clear();
        return true;
    };
    for (char c : s) {
        if (c == ',' || c == ' ') { if (!flush()) return false; }
        else tok.push_back(c);
    }
    if (!flush()) return false;
    if (parts.size() == 3) { v = {parts[0], parts[1], parts[2]}; return true; }
    if (parts.size() == 1) { v = {parts[0], parts[0], parts[0]}; return true; }
    return false;
}
double srgb_to_linear(double c) { return c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4); }

bool el_float(const Element& e, const char* name, double& out) {
    const Element* p = e.prop("float", name);
    if (!p || !p->attr("value")) return false;
    return parse_f64(*p->attr("value"), out);
}
bool el_int(const Element& e, const char* name, long long& out) {
    const Element* p = e.prop("integer", name);
    if (!p || !p->attr("value")) return false;
    return parse_usize(*p->attr("value"), out);
}
const std::string* el_string(const Element& e, const char* name) {
    const Element* p = e.prop("string", name);
    return p ? p->attr("value") : nullptr;
}
bool el_point(const Element& e, const char* name, V3& v) {
    const Element* p = e.prop("point", name);
    if (!p) return false;
    const std::string *x = p->attr("x"), *y = p->attr("y"), *z = p->attr("z");
    if (x && y && z) return parse_f64(*x, v.x) && parse_f64(*y, v.y) && parse_f64(*z, v.z);
    return p->attr("value") && parse_vec3(*p->attr("value"), v);
}
bool el_color(const Element& e, const char* name, V3& c) {
    if (const Element* p = e.prop("rgb", name)) return p->attr("value") && parse_vec3(*p->attr("value"), c);
    if (const Element* p = e.prop("srgb", name)) {
        if (!p->attr("value") || !parse_vec3(*p->attr("value"), c)) return false;
        c = {srgb_to_linear(c.x), srgb_to_linear(c.y), srgb_to_linear(c.z)};
        return true;
    }
    return false;
}

// ---- transforms (src/transform.rs:24-111) --------------------------------------------
struct Xf {
    double a[3][3];
    double t[3];
};
Xf xf_identity() { return Xf{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, {0, 0, 0}}; }
Xf xf_compose(const Xf& s, const Xf& in) {  // s o in
    Xf r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.a[i][j] = s.a[i][0] * in.a[0][j] + s.a[i][1] * in.a[1][j] + s.a[i][2] * in.a[2][j];
    for (int i = 0; i < 3; ++i) r.t[i] = (s.a[i][0] * in.t[0] + s.a[i][1] * in.t[1] + s.a[i][2] * in.t[2]) + s.t[i];
    return r;
}
Xf xf_rotate(V3 axis, double deg) {  // Rodrigues (src/transform.rs:101-111)
    const double l = std::max(std::sqrt(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z), 1e-30);
    const double x = axis.x / l, y = axis.y / l, z = axis.z / l;
    const double r = deg * (kPi / 180.0);
    const double s = std::sin(r), c = std::cos(r), oc = 1.0 - c;
    return Xf{{{c + x * x * oc, x * y * oc - z * s, x * z * oc + y * s},
               {y * x * oc + z * s, c + y * y * oc, y * z * oc - x * s},
               {z * x * oc - y * s, z * y * oc + x * s, c + z * z * oc}},
              {0, 0, 0}};
}
V3 xyz_of(const Element& e, double dflt) {
    auto g = [&](const char* k) {
        double v;
        const std::string* s = e.attr(k);
        return (s && parse_f64(*s, v)) ? v : dflt;
    };
    return {g("x"), g("y"), g("z")};
}

// ---- shapes ---------------------------------------------------------------------------
void add_tri(LoadedMesh& m, const double* a, const double* b, const double* c, int32_t mat) {
    const int32_t base = (int32_t)(m.pos.size() / 3);
    for (const double* p : {a, b, c}) m.pos.insert(m.pos.end(), p, p + 3);
    m.idx.insert(m.idx.end(), {base, base + 1, base + 2});
    m.mat.push_back(mat);
}
LoadedMesh unit_rectangle(int32_t mat) {  // src/mitsuba.rs:414-424
    const double a[3] = {-1, -1, 0}, b[3] = {1, -1, 0}, c[3] = {1, 1, 0}, d[3] = {-1, 1, 0};
    LoadedMesh m;
    add_tri(m, a, b, c, mat);
    add_tri(m, a, c, d, mat);
    return m;
}
LoadedMesh unit_cube(int32_t mat) {  // src/mitsuba.rs:426-452
    const double v[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                            {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    const int q[6][4] = {{0, 1, 2, 3}, {4, 7, 6, 5}, {0, 4, 5, 1}, {1, 5, 6, 2}, {2, 6, 7, 3}, {3, 7, 4, 0}};
    LoadedMesh m;
    for (const auto& f : q) {
        add_tri(m, v[f[0]], v[f[1]], v[f[2]], mat);
        add_tri(m, v[f[0]], v[f[2]], v[f[3]], mat);
    }
    return m;
}
LoadedMesh unit_disk(int32_t mat) {  // src/mitsuba.rs:454-470
    const int n = 64;
    const double tau = 2.0 * kPi;
    LoadedMesh m;
    const double c[3] = {0, 0, 0};
    for (int i = 0; i < n; ++i) {
        const double a0 = tau * (double)i / (double)n, a1 = tau * (double)(i + 1) / (double)n;
        const double p0[3] = {std::cos(a0), std::sin(a0), 0.0}, p1[3] = {std::cos(a1), std::sin(a1), 0.0};
        add_tri(m, c, p0, p1, mat);
    }
    return m;
}

std::string dir_of(const std::string& path) {
    const size_t k = path.find_last_of('/');
    return k == std::string::npos ? std::string() : path.substr(0, k);
}
std::string resolve(const std::string& base, const std::string& f) {
    if (!f.empty() && f[0] == '/') return f;
    return base.empty() ? f : base + "/" + f;
}

tpt_material mk(int kind, V3 c, double p) {
    tpt_material m{};
    m.kind = kind;
    m.rgb[0] = c.x; m.rgb[1] = c.y; m.rgb[2] = c.z;
    m.param = p;
    return m;
}

tpt_material parse_bsdf(const Element& e, LoadedScene& out) {  // src/mitsuba.rs:558-597
    const std::string t = e.type();
    V3 c;
    double v;
    if (t == "twosided") {
        const Element* inner = e.child("bsdf");
        return inner ? parse_bsdf(*inner, out) : mk(TPT_MAT_LAMBERT, {0.5, 0.5, 0.5}, 0.0);
    }
    if (t == "diffuse") return mk(TPT_MAT_LAMBERT, el_color(e, "reflectance", c) ? c : V3{0.5, 0.5, 0.5}, 0.0);
    if (t == "conductor")
        return mk(TPT_MAT_METAL, el_color(e, "specular_reflectance", c) ? c : V3{1, 1, 1}, 0.0);
    if (t == "roughconductor") {
        const std::string* d = el_string(e, "distribution");
        if (d && *d != "ggx") out.warnings.push_back("roughconductor distribution '" + *d + "' unsupported; using ggx");
        return mk(TPT_MAT_GGX, el_color(e, "specular_reflectance", c) ? c : V3{1, 1, 1},
                  el_float(e, "alpha", v) ? v : 0.1);
    }
    if (t == "dielectric" || t == "thindielectric" || t == "roughdielectric") {
        double ii = 1.5, ei = 1.0;
        el_float(e, "int_ior", ii);
        el_float(e, "ext_ior", ei);
        return mk(TPT_MAT_DIELECTRIC, el_color(e, "absorption", c) ? c : V3{0, 0, 0}, ii / ei);
    }
    out.warnings.push_back("unsupported bsdf type '" + t + "'; defaulting to diffuse");
    return mk(TPT_MAT_LAMBERT, el_color(e, "reflectance", c) ? c : V3{0.5, 0.5, 0.5}, 0.0);
}

Xf parse_transform(const Element& e, LoadedScene& out) {  // src/mitsuba.rs:483-541
    Xf acc = xf_identity();
    for (const Element& op : e.children) {
        Xf x = xf_identity();
        bool have = true;
        if (op.tag == "translate") {
            const V3 t = xyz_of(op, 0.0);
            x.t[0] = t.x; x.t[1] = t.y; x.t[2] = t.z;
        } else if (op.tag == "scale") {
            double s;
            const V3 v = (op.attr("value") && parse_f64(*op.attr("value"), s)) ? V3{s, s, s} : xyz_of(op, 1.0);
            x.a[0][0] = v.x; x.a[1][1] = v.y; x.a[2][2] = v.z;
        } else if (op.tag == "rotate") {
            const V3 axis = xyz_of(op, 0.0);
            double ang = 0.0;
            if (op.attr("angle")) parse_f64(*op.attr("angle"), ang) || (ang = 0.0);
            if (std::sqrt(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z) < 1e-12) {
                out.warnings.push_back("rotate with zero axis; ignored");
                have = false;
            } else {
                x = xf_rotate(axis, ang);
            }
        } else if (op.tag == "matrix") {
            std::vector<double> vals;
            if (op.attr("value")) {
                std::string tok;
                auto flush = [&]() {
                    double d;
                    if (tok.find_first_not_of(" \t\r\n") != std::string::npos && parse_f64(tok, d)) vals.push_back(d);
                    tok.clear();
                };
                for (char c : *op.attr("value")) {
                    if (c == ',' || c == ' ') flush();
                    else tok.push_back(c);
                }
                flush();
            }
            if (vals.size() == 16) {
                for (int r = 0; r < 3; ++r) {
                    for (int c = 0; c < 3; ++c) x.a[r][c] = vals[(size_t)r * 4 + c];
                    x.t[r] = vals[(size_t)r * 4 + 3];
                }
            } else {
                out.warnings.push_back("matrix expects 16 values, got " + std::to_string(vals.size()) +
                                       "; ignored");
                have = false;
            }
        } else if (op.tag == "lookat") {
            have = false;
        } else {
            out.warnings.push_back("unsupported transform op <" + op.tag + ">, ignored");
            have = false;
        }
        if (have) acc = xf_compose(acc, x);
    }
    return acc;
}

void parse_shape(const Element& e, const std::string& base, LoadedScene& out) {  // src/mitsuba.rs:352-412
    tpt_material mat;
    V3 c;
    if (const Element* em = e.child("emitter")) {
        if (em->type() != "area") out.warnings.push_back("emitter type '" + em->type() + "' treated as area light");
        mat = mk(TPT_MAT_DIFFUSE_LIGHT, el_color(*em, "radiance", c) ? c : V3{1, 1, 1}, 0.0);
    } else if (const Element* b = e.child("bsdf")) {
        mat = parse_bsdf(*b, out);
    } else {
        out.warnings.push_back("shape type '" + e.type() + "' without bsdf or emitter; defaulting to diffuse");
        mat = mk(TPT_MAT_LAMBERT, {0.5, 0.5, 0.5}, 0.0);
    }
    const int32_t mat_id = (int32_t)out.mats.size();
    const std::string t = e.type();
    LoadedMesh mesh;
    if (t == "sphere") {
        V3 center{0, 0, 0};
        double r = 1.0;
        el_point(e, "center", center) || (center = V3{0, 0, 0}, true);
        el_float(e, "radius", r) || (r = 1.0, true);
        out.mats.push_back(mat);
        tpt_sphere s{};
        s.center[0] = center.x; s.center[1] = center.y; s.center[2] = center.z;
        s.radius = r;
        s.mat_id = mat_id;
        out.spheres.push_back(s);
        return;
    } else if (t == "rectangle") {
        mesh = unit_rectangle(mat_id);
    } else if (t == "cube") {
        mesh = unit_cube(mat_id);
    } else if (t == "disk") {
        mesh = unit_disk(mat_id);
    } else if (t == "obj") {
        const std::string* f = el_string(e, "filename");
        if (!f) {
            out.warnings.push_back("obj shape without filename; skipped");
            return;
        }
        try {
            load_obj(resolve(base, *f), mesh.pos, mesh.idx);
        } catch (const std::exception& ex) {
            out.warnings.push_back(std::string("failed to load obj '") + resolve(base, *f) + "': " + ex.what() +
                                   "; skipped");
            return;
        }
        mesh.mat.assign(mesh.idx.size() / 3, mat_id);
    } else {
        out.warnings.push_back("unsupported shape type '" + t + "', skipped");
        return;
    }
    const Element* te = e.child("transform");
    const Xf x = te ? parse_transform(*te, out) : xf_identity();
    out.mats.push_back(mat);
    tpt_instance_desc inst{};
    inst.mesh_id = (int64_t)out.meshes.size();
    for (int r = 0; r < 3; ++r) {
        for (int cc = 0; cc < 3; ++cc) inst.linear[r * 3 + cc] = x.a[r][cc];
        inst.translation[r] = x.t[r];
    }
    inst.mat_override = -1;
    out.meshes.push_back(std::move(mesh));
    out.instances.push_back(inst);
}

void set_env_pixels(LoadedScene& out, int w, int h, std::vector<double>&& px) {
    out.env_pixels = std::move(px);
    out.desc.env.kind = TPT_ENV_MAP;
    out.desc.env.width = w;
    out.desc.env.height = h;
}

}  // namespace

void LoadedScene::finalize() {
    mesh_descs.clear();
    for (const LoadedMesh& m : meshes) {
        tpt_mesh_desc d{};
        d.positions = m.pos.data();
        d.n_vertices = (int64_t)(m.pos.size() / 3);
        d.indices = m.idx.data();
        d.mat_ids = m.mat.data();
        d.n_tris = (int64_t)m.mat.size();
        mesh_descs.push_back(d);
    }
    desc.spheres = spheres.data();
    desc.n_spheres = (int64_t)spheres.size();
    desc.meshes = mesh_descs.data();
    desc.n_meshes = (int64_t)mesh_descs.size();
    desc.instances = instances.data();
    desc.n_instances = (int64_t)instances.size();
    desc.materials = mats.data();
    desc.n_materials = (int64_t)mats.size();
    desc.env.pixels = env_pixels.empty() ? nullptr : env_pixels.data();
}

void load_obj(const std::string& path, std::vector<double>& pos, std::vector<int32_t>& idx) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open " + path);
    pos.clear();
    idx.clear();
    std::string line;
    auto num = [](const std::string& t, double dflt) {
        double v;
        return parse_f64(t, v) ? v : dflt;
    };
    while (std::getline(in, line)) {
        const size_t a = line.find_first_not_of(" \t\r\n");
        if (a == std::string::npos) continue;
        const size_t b = line.find_last_not_of(" \t\r\n");
        const std::string l = line.substr(a, b - a + 1);
        if (l[0] == '#') continue;
        std::istringstream ss(l.size() > 2 ? l.substr(2) : std::string());
        if (l.rfind("v ", 0) == 0) {
            std::string x, y, z;
            ss >> x >> y >> z;
            pos.push_back(num(x, 0.0));
            pos.push_back(num(y, 0.0));
            pos.push_back(num(z, 0.0));
        } else if (l.rfind("f ", 0) == 0) {
            std::vector<int32_t> face;
            std::string tok;
            const long long n = (long long)(pos.size() / 3);
            while (ss >> tok) {
                const std::string first = tok.substr(0, tok.find('/'));
                char* end = nullptr;
                const long i = std::strtol(first.c_str(), &end, 10);
                const bool ok = !first.empty() && end == first.c_str() + first.size();
                const long v = ok ? i : 0;
                if (v > 0 && v - 1 < n) face.push_back((int32_t)(v - 1));  // 1-based
                else if (v < 0 && n + v >= 0) face.push_back((int32_t)(n + v));  // relative
            }
            for (size_t k = 1; k + 1 < face.size(); ++k) {  // fan
                idx.push_back(face[0]);
                idx.push_back(face[k]);
                idx.push_back(face[k + 1]);
            }
        }
    }
}

std::unique_ptr<LoadedScene> load_mitsuba(const std::string& path, tpt_render_config& cfg) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + path);
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string text = ss.str();
    XmlReader rd(text);
    const Element root = rd.parse();
    if (root.tag != "scene") throw std::runtime_error("root element is not <scene>");
    long long v;
    for (const Element& c : root.children) {
        if (c.tag == "film") {
            if (el_int(c, "width", v)) cfg.width = (int32_t)std::max(v, 1ll);
            if (el_int(c, "height", v)) cfg.height = (int32_t)std::max(v, 1ll);
        } else if (c.tag == "sampler") {
            if (el_int(c, "sample_count", v)) cfg.spp = (int32_t)std::max(v, 1ll);
        } else if (c.tag == "integrator") {
            if (el_int(c, "max_depth", v)) cfg.max_bounces = (int32_t)std::max(v, 1ll);
            if (el_int(c, "rr_depth", v)) cfg.rr_start = (int32_t)v;
        }
    }
    const std::string base = dir_of(path);
    const double aspect = (double)cfg.width / (double)cfg.height;
    auto out = std::make_unique<LoadedScene>();
    bool have_cam = false, have_env = false;
    for (const Element& c : root.children) {
        if (c.tag == "sensor") {
            if (c.type() != "perspective") {
                out->warnings.push_back("unsupported sensor type '" + c.type() + "', ignored");
                continue;
            }
            double fov = 40.0;  // src/mitsuba.rs:307-337
            el_float(c, "fov", fov);
            const std::string* axis = el_string(c, "fov_axis");
            double vfov = fov;
            if (!(axis && *axis == "y")) {
                const double hr = fov * (kPi / 180.0);
                vfov = (2.0 * std::atan(std::tan(hr * 0.5) / aspect)) * (180.0 / kPi);
            }
            V3 eye{0, 0, 4}, tgt{0, 0, 0}, up{0, 1, 0};
            const Element* t = c.child("transform");
            const Element* la = t ? t->child("lookat") : nullptr;
            if (la) {
                V3 o, g, u;
                if (la->attr("origin") && parse_vec3(*la->attr("origin"), o) && la->attr("target") &&
                    parse_vec3(*la->attr("target"), g)) {
                    eye = o;
                    tgt = g;
                    up = (la->attr("up") && parse_vec3(*la->attr("up"), u)) ? u : V3{0, 1, 0};
                }
            }
            double ap = 0.0;
            el_float(c, "aperture_radius", ap);
            const double dx = eye.x - tgt.x, dy = eye.y - tgt.y, dz = eye.z - tgt.z;
            double focus = std::sqrt(dx * dx + dy * dy + dz * dz);
            el_float(c, "focus_distance", focus);
            tpt_camera_desc& cd = out->desc.camera;
            cd.kind = TPT_CAMERA_LOOK_AT_DOF;
            cd.eye[0] = eye.x; cd.eye[1] = eye.y; cd.eye[2] = eye.z;
            cd.target[0] = tgt.x; cd.target[1] = tgt.y; cd.target[2] = tgt.z;
            cd.up[0] = up.x; cd.up[1] = up.y; cd.up[2] = up.z;
            cd.fov_y_deg = vfov;
            cd.aspect = aspect;
            cd.focus_dist = focus;
            cd.aperture = 2.0 * ap;
            have_cam = true;
        } else if (c.tag == "shape") {
            parse_shape(c, base, *out);
        } else if (c.tag == "emitter") {  // src/mitsuba.rs:226-253
            if (c.child("transform")) out->warnings.push_back("envmap to_world rotation is unsupported; ignored");
            double scale = 1.0;
            el_float(c, "scale", scale);
            if (c.type() == "envmap") {
                const std::string* f = el_string(c, "filename");
                if (!f) continue;
                try {
                    int w = 0, h = 0;
                    std::vector<double> px;
                    read_hdr(resolve(base, *f), w, h, px);
                    if (scale != 1.0)
                        for (double& p : px) p *= scale;
                    set_env_pixels(*out, w, h, std::move(px));
                    have_env = true;
                } catch (const std::exception& ex) {
                    out->warnings.push_back(std::string("failed to load envmap: ") + ex.what() + "; ignored");
                }
            } else if (c.type() == "constant") {
                V3 r{1, 1, 1};
                el_color(c, "radiance", r) || (r = V3{1, 1, 1}, true);
                std::vector<double> px = {r.x, r.y, r.z};
                if (scale != 1.0)
                    for (double& p : px) p *= scale;
                set_env_pixels(*out, 1, 1, std::move(px));
                have_env = true;
            } else {
                out->warnings.push_back("unsupported scene emitter type '" + c.type() + "', ignored");
            }
        } else if (c.tag == "integrator" || c.tag == "sampler" || c.tag == "film" || c.tag == "default" ||
                   c.tag == "rfilter") {
        } else {
            out->warnings.push_back("unsupported element <" + c.tag + ">, skipped");
        }
    }
    if (!have_cam) {
        out->warnings.push_back("no perspective sensor found; using a default camera");
        tpt_camera_desc& cd = out->desc.camera;
        cd.kind = TPT_CAMERA_LOOK_AT;
        cd.eye[2] = 4.0;
        cd.up[1] = 1.0;
        cd.fov_y_deg = 40.0;
        cd.aspect = aspect;
    }
    if (!have_env) set_env_pixels(*out, 1, 1, std::vector<double>{0.0, 0.0, 0.0});  // black, src/mitsuba.rs:218
    out->finalize();
    return out;
}

std::unique_ptr<LoadedScene> default_scene(const tpt_render_config& cfg, const std::string& env_path) {
    auto out = std::make_unique<LoadedScene>();
    tpt_camera_desc& cd = out->desc.camera;  // src/scene.rs:27-37
    cd.kind = TPT_CAMERA_LOOK_AT_DOF;
    const double eye[3] = {0.0, 1.2, 4.0}, tgt[3] = {0.0, 0.5, 0.0};
    for (int k = 0; k < 3; ++k) { cd.eye[k] = eye[k]; cd.target[k] = tgt[k]; }
    cd.up[1] = 1.0;
    cd.fov_y_deg = 40.0;
    cd.aspect = (double)cfg.width / (double)cfg.height;
    const double dx = eye[0] - tgt[0], dy = eye[1] - tgt[1], dz = eye[2] - tgt[2];
    cd.focus_dist = std::sqrt(dx * dx + dy * dy + dz * dz);
    cd.aperture = 0.0;
    auto srgb = [](double r, double g, double b) { return V3{srgb_to_linear(r), srgb_to_linear(g), srgb_to_linear(b)}; };
    out->mats = {mk(TPT_MAT_LAMBERT, srgb(0.5, 0.5, 0.5), 0.0), mk(TPT_MAT_LAMBERT, srgb(0.8, 0.3, 0.3), 0.0),
                 mk(TPT_MAT_METAL, srgb(0.8, 0.8, 0.8), 0.0), mk(TPT_MAT_GGX, srgb(0.95, 0.78, 0.35), 0.25),
                 mk(TPT_MAT_DIELECTRIC, {0.02, 0.05, 0.02}, 1.5), mk(TPT_MAT_DIFFUSE_LIGHT, {8.0, 7.0, 5.0}, 0.0)};
    const double sp[6][5] = {{0.0, -1000.0, 0.0, 1000.0, 0}, {-1.8, 0.5, 0.0, 0.5, 1}, {-0.6, 0.5, 0.0, 0.5, 2},
                             {0.6, 0.5, 0.0, 0.5, 3},        {1.8, 0.5, 0.0, 0.5, 4},  {0.0, 3.0, -1.0, 0.8, 5}};
    for (const auto& s : sp) {
        tpt_sphere o{};
        o.center[0] = s[0]; o.center[1] = s[1]; o.center[2] = s[2];
        o.radius = s[3];
        o.mat_id = (int64_t)s[4];
        out->spheres.push_back(o);
    }
    if (!env_path.empty()) {
        try {
            int w = 0, h = 0;
            std::vector<double> px;
            read_hdr(env_path, w, h, px);
            set_env_pixels(*out, w, h, std::move(px));
        } catch (const std::exception& ex) {
            out->warnings.push_back(std::string("env map load failed (") + env_path + "): " + ex.what());
        }
    }
    out->finalize();
    return out;
}

}  // namespace tpt
