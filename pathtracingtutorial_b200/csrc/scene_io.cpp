// scene_io.cpp -- the reference's JSON scene format, RGBE .hdr images and OBJ
// meshes, read into a HostScene.
//
// Scene format (Part_2/src/scene/scene_loader.cpp:34-276):
//   camera{position,lookAt,up,fov,aperture,focalDistance,resolution}
//   render{spp,samplePerFrame,maxDepth,output,sampler}
//   environment{file}
//   materials{name:{...}}   -- indexed in sorted key order, as the reference's
//                              JSON library stores objects in a sorted map
//   lights[{type,position,direction,color,intensity,range,innerCone,outerCone}]
//   objects[{type: quad|mesh, vertices|file, material, transform}]
// glTF objects are not supported (the glTF importer is outside this library);
// such a scene is rejected with an error instead of being rendered without them.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <stdexcept>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <unordered_map>

#include "engine.h"

namespace ptb {

// ---------------------------------------------------------------------------
// Minimal JSON value + recursive-descent parser.
// ---------------------------------------------------------------------------
namespace json {

struct Value;
using Object = std::map<std::string, Value>;
using Array  = std::vector<Value>;

struct Value {
    enum Kind { Null, Bool, Int, Real, String, Arr, Obj } kind = Null;
    bool b = false;
    long long i = 0;
    double d = 0.0;
    std::string s;
    std::shared_ptr<Array> a;
    std::shared_ptr<Object> o;

    bool is_number() const { return kind == Int || kind == Real; }
    bool has(const char* k) const { return kind == Obj && o->count(k) != 0; }
    const Value& operator[](const char* k) const { return o->at(k); }
    const Value& operator[](size_t idx) const { return a->at(idx); }
    const Value& operator[](int idx) const { return a->at(static_cast<size_t>(idx)); }
    size_t size() const { return kind == Arr ? a->size() : (kind == Obj ? o->size() : 0); }
};

struct Error { std::string msg; };

class Parser {
public:
    explicit Parser(const std::string& t) : t_(t) {}
    Value parse() {
        Value v = value();
        ws();
        if (p_ != t_.size()) fail("trailing characters");
        return v;
    }

private:
    [[noreturn]] void fail(const std::string& m) {
        throw Error{"JSON parse error at offset " + std::to_string(p_) + ": " + m};
    }
    void ws() { while (p_ < t_.size() && std::isspace(static_cast<unsigned char>(t_[p_]))) ++p_; }
    char peek() { ws(); return p_ < t_.size() ? t_[p_] : '\0'; }
    void expect(char c) { if (peek() != c) fail(std::string("expected '") + c + "'"); ++p_; }

    Value value() {
        const char c = peek();
        if (c == '{') return object();
        if (c == '[') return array();
        if (c == '"') { Value v; v.kind = Value::String; v.s = str(); return v; }
        if (c == 't' || c == 'f' || c == 'n') return literal();
        if (c == '-' || std::isdigit(static_cast<unsigned char>(c))) return number();
        fail("unexpected character");
    }
    Value object() {
        expect('{');
        Value v; v.kind = Value::Obj; v.o = std::make_shared<Object>();
        if (peek() == '}') { ++p_; return v; }
        for (;;) {
            if (peek() != '"') fail("expected key");
            std::string k = str();
            expect(':');
            (*v.o)[k] = value();
            const char c = peek();
            if (c == ',') { ++p_; continue; }
            if (c == '}') { ++p_; return v; }
            fail("expected ',' or '}'");
        }
    }
    Value array() {
        expect('[');
        Value v; v.kind = Value::Arr; v.a = std::make_shared<Array>();
        if (peek() == ']') { ++p_; return v; }
        for (;;) {
            v.a->push_back(value());
            const char c = peek();
            if (c == ',') { ++p_; continue; }
            if (c == ']') { ++p_; return v; }
            fail("expected ',' or ']'");
        }
    }
    std::string str() {
        expect('"');
        std::string out;
        while (p_ < t_.size() && t_[p_] != '"') {
            char c = t_[p_++];
            if (c == '\\') {
                if (p_ >= t_.size()) fail("bad escape");
                const char e = t_[p_++];
                switch (e) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case '/': out += '/'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'n': out += '\n'; break;
                    case 'r': out += '\r'; break;
                    case 't': out += '\t'; break;
                    case 'u': {
                        if (p_ + 4 > t_.size()) fail("bad \\u escape");
                        const unsigned cp = static_cast<unsigned>(std::stoul(t_.substr(p_, 4), nullptr, 16));
                        p_ += 4;
                        if (cp < 0x80) out += static_cast<char>(cp);
                        else if (cp < 0x800) { out += static_cast<char>(0xC0 | (cp >> 6)); out += static_cast<char>(0x80 | (cp & 0x3F)); }
                        else { out += static_cast<char>(0xE0 | (cp >> 12)); out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F)); out += static_cast<char>(0x80 | (cp & 0x3F)); }
                        break;
                    }
                    default: fail("bad escape");
                }
            } else {
                out += c;
            }
        }
        if (p_ >= t_.size()) fail("unterminated string");
        ++p_;
        return out;
    }
    Value literal() {
        Value v;
        if (t_.compare(p_, 4, "true") == 0) { v.kind = Value::Bool; v.b = true; p_ += 4; return v; }
        if (t_.compare(p_, 5, "false") == 0) { v.kind = Value::Bool; v.b = false; p_ += 5; return v; }
        if (t_.compare(p_, 4, "null") == 0) { p_ += 4; return v; }
        fail("bad literal");
    }
    Value number() {
        const size_t s = p_;
        bool real = false;
        if (t_[p_] == '-') ++p_;
        while (p_ < t_.size()) {
            const char c = t_[p_];
            if (std::isdigit(static_cast<unsigned char>(c))) { ++p_; continue; }
            if (c == '.' || c == 'e' || c == 'E' || c == '+' || c == '-') { real = true; ++p_; continue; }
            break;
        }
        const std::string tok = t_.substr(s, p_ - s);
        Value v;
        char* end = nullptr;
        if (!real) {
            errno = 0;
            const long long iv = std::strtoll(tok.c_str(), &end, 10);
            if (errno == 0 && end && *end == '\0') { v.kind = Value::Int; v.i = iv; v.d = static_cast<double>(iv); return v; }
        }
        v.kind = Value::Real;
        v.d = std::strtod(tok.c_str(), &end);
        if (!end || *end != '\0') fail("bad number");
        return v;
    }

    const std::string& t_;
    size_t p_ = 0;
};

// get<float>(): integers convert from the integer, reals from the double.
float as_float(const Value& v) {
    if (v.kind == Value::Int) return static_cast<float>(v.i);
    if (v.kind == Value::Real) return static_cast<float>(v.d);
    throw Error{"expected a number"};
}
int as_int(const Value& v) {
    if (v.kind == Value::Int) return static_cast<int>(v.i);
    if (v.kind == Value::Real) return static_cast<int>(v.d);
    throw Error{"expected an integer"};
}
bool as_bool(const Value& v) {
    if (v.kind == Value::Bool) return v.b;
    throw Error{"expected a boolean"};
}
const std::string& as_string(const Value& v) {
    if (v.kind == Value::String) return v.s;
    throw Error{"expected a string"};
}

}  // namespace json

// ---------------------------------------------------------------------------
// 4x4 transform (translation * rotation * uniform scale), row-major like
// Part_2/src/math/mat4.h.
// ---------------------------------------------------------------------------
namespace {

struct M4 { float m[16]; };

M4 m4_identity() { M4 r{}; for (int i = 0; i < 16; ++i) r.m[i] = (i % 5 == 0) ? 1.0f : 0.0f; return r; }
M4 m4_mul(const M4& a, const M4& b) {
    M4 r{};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            float s = 0.0f;
            for (int k = 0; k < 4; ++k) s += a.m[i * 4 + k] * b.m[k * 4 + j];
            r.m[i * 4 + j] = s;
        }
    return r;
}
M4 m4_translation(f3 t) { M4 r = m4_identity(); r.m[3] = t.x; r.m[7] = t.y; r.m[11] = t.z; return r; }
M4 m4_scaling(float s) { M4 r = m4_identity(); r.m[0] = s; r.m[5] = s; r.m[10] = s; return r; }
// Axis-angle rotation (Rodrigues).
M4 m4_rotation(float rad, f3 axis) {
    const float len = std::sqrt(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z);
    if (len < 1e-8f) return m4_identity();
    const float x = axis.x / len, y = axis.y / len, z = axis.z / len;
    const float c = cosf(rad), s = sinf(rad), omc = 1.0f - c;
    M4 r = m4_identity();
    r.m[0] = c + omc * x * x;     r.m[1] = omc * x * y - s * z; r.m[2] = omc * x * z + s * y;  r.m[3] = 0;
    r.m[4] = omc * y * x + s * z; r.m[5] = c + omc * y * y;     r.m[6] = omc * y * z - s * x;  r.m[7] = 0;
    r.m[8] = omc * z * x - s * y; r.m[9] = omc * z * y + s * x; r.m[10] = c + omc * z * z;     r.m[11] = 0;
    r.m[12] = 0; r.m[13] = 0; r.m[14] = 0; r.m[15] = 1;
    return r;
}
// Gauss-Jordan inverse with partial pivoting (identity when singular).
M4 m4_inverse(const M4& in) {
    M4 inv = m4_identity();
    M4 a = in;
    for (int i = 0; i < 4; ++i) {
        float pv = std::fabs(a.m[i * 4 + i]);
        int pr = i;
        for (int j = i + 1; j < 4; ++j) {
            const float c = std::fabs(a.m[j * 4 + i]);
            if (c > pv) { pv = c; pr = j; }
        }
        if (pv < 1e-8f) return m4_identity();
        if (pr != i)
            for (int k = 0; k < 4; ++k) {
                std::swap(a.m[i * 4 + k], a.m[pr * 4 + k]);
                std::swap(inv.m[i * 4 + k], inv.m[pr * 4 + k]);
            }
        const float p = a.m[i * 4 + i];
        for (int k = 0; k < 4; ++k) { a.m[i * 4 + k] /= p; inv.m[i * 4 + k] /= p; }
        for (int j = 0; j < 4; ++j) {
            if (j == i) continue;
            const float f = a.m[j * 4 + i];
            for (int k = 0; k < 4; ++k) { a.m[j * 4 + k] -= f * a.m[i * 4 + k]; inv.m[j * 4 + k] -= f * inv.m[i * 4 + k]; }
        }
    }
    return inv;
}
M4 m4_transpose(const M4& a) { M4 r{}; for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) r.m[j * 4 + i] = a.m[i * 4 + j]; return r; }
f3 m4_point(const M4& t, f3 v) {
    const float* m = t.m;
    return mk(m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3],
              m[4] * v.x + m[5] * v.y + m[6] * v.z + m[7],
              m[8] * v.x + m[9] * v.y + m[10] * v.z + m[11]);
}
f3 m4_vector(const M4& t, f3 v) {
    const float* m = t.m;
    return mk(m[0] * v.x + m[1] * v.y + m[2] * v.z,
              m[4] * v.x + m[5] * v.y + m[6] * v.z,
              m[8] * v.x + m[9] * v.y + m[10] * v.z);
}

f3 to_f3(const json::Value& v) {
    if (v.kind != json::Value::Arr || v.size() < 3) throw json::Error{"expected a 3-vector"};
    return mk(json::as_float(v[0]), json::as_float(v[1]), json::as_float(v[2]));
}
void st3(float* dst, f3 v) { dst[0] = v.x; dst[1] = v.y; dst[2] = v.z; }

std::string resolve_relative(const std::string& base, const std::string& rel) {
    if (!rel.empty() && rel[0] == '/') return rel;
    const size_t slash = base.find_last_of('/');
    if (slash == std::string::npos) return rel;
    return base.substr(0, slash + 1) + rel;
}

std::string lower_ext(const std::string& path) {
    const size_t dot = path.find_last_of('.');
    if (dot == std::string::npos) return "";
    std::string e = path.substr(dot);
    for (char& c : e) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    return e;
}

void apply_material_override(const json::Value& p, pt_material& m) {
    using json::as_float;
    if (p.has("baseColor"))          st3(m.base_color, to_f3(p["baseColor"]));
    if (p.has("metallic"))           m.metallic = as_float(p["metallic"]);
    if (p.has("roughness"))          m.roughness = as_float(p["roughness"]);
    if (p.has("specularTint"))       m.specular_tint = as_float(p["specularTint"]);
    if (p.has("anisotropic"))        m.anisotropic = as_float(p["anisotropic"]);
    if (p.has("sheen"))              m.sheen = as_float(p["sheen"]);
    if (p.has("sheenTint"))          m.sheen_tint = as_float(p["sheenTint"]);
    if (p.has("clearcoat"))          m.clearcoat = as_float(p["clearcoat"]);
    if (p.has("clearcoatRoughness")) m.clearcoat_roughness = as_float(p["clearcoatRoughness"]);
    if (p.has("specTrans"))          m.spec_trans = as_float(p["specTrans"]);
    if (p.has("ior"))                m.ior = as_float(p["ior"]);
    if (p.has("subsurface"))         m.subsurface = as_float(p["subsurface"]);
    if (p.has("emissive"))           st3(m.emissive, to_f3(p["emissive"]));
    if (p.has("emissiveStrength"))   m.emissive_strength = as_float(p["emissiveStrength"]);
    if (p.has("alphaCutoff"))        m.alpha_cutoff = as_float(p["alphaCutoff"]);
    if (p.has("alphaMode"))          m.alpha_mode = json::as_int(p["alphaMode"]);
    if (p.has("doubleSided"))        m.double_sided = json::as_bool(p["doubleSided"]) ? 1 : 0;
}

M4 parse_transform(const json::Value& obj) {
    if (!obj.has("transform")) return m4_identity();
    const json::Value& t = obj["transform"];
    f3 translate = mk(0.0f), axis = mk(0.0f, 1.0f, 0.0f);
    float angle = 0.0f, scale = 1.0f;
    if (t.has("translate")) translate = to_f3(t["translate"]);
    if (t.has("rotate")) { axis = to_f3(t["rotate"]["axis"]); angle = json::as_float(t["rotate"]["angle"]); }
    if (t.has("scale")) scale = json::as_float(t["scale"]);
    return m4_mul(m4_mul(m4_translation(translate), m4_rotation(angle * kPi / 180.0f, axis)), m4_scaling(scale));
}

// Camera placement from the geometry bounds when the scene has no camera.
void auto_fit_camera(const std::vector<pt_vertex>& verts, pt_camera& cam) {
    if (verts.empty()) return;
    f3 lo = mk(1e30f), hi = mk(-1e30f);
    for (const pt_vertex& v : verts) {
        lo = mk(std::fmin(lo.x, v.position[0]), std::fmin(lo.y, v.position[1]), std::fmin(lo.z, v.position[2]));
        hi = mk(std::fmax(hi.x, v.position[0]), std::fmax(hi.y, v.position[1]), std::fmax(hi.z, v.position[2]));
    }
    const f3 center = (lo + hi) * 0.5f;
    float radius = length(hi - lo) * 0.5f;
    if (radius < 1e-5f) radius = 1.0f;
    const float fov_rad = cam.fov * kPi / 180.0f;
    const float dist = radius / std::tan(fov_rad * 0.5f) * 1.2f;
    st3(cam.position, center + mk(0.0f, radius * 0.3f, dist));
    st3(cam.look_at, center);
    st3(cam.up, mk(0.0f, 1.0f, 0.0f));
}

}  // namespace

void add_quad(const float a_[3], const float b_[3], const float c_[3], const float d_[3], int mat,
              std::vector<pt_vertex>& verts, std::vector<pt_face>& faces) {
    const f3 a = ld3(a_), b = ld3(b_), c = ld3(c_), d = ld3(d_);
    const f3 n = normalize(cross(b - a, c - a));
    const f3 t = normalize(b - a);
    const uint32_t base = static_cast<uint32_t>(verts.size());
    const f3 pts[4] = {a, b, c, d};
    const float uvs[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
    for (int i = 0; i < 4; ++i) {
        pt_vertex v{};
        st3(v.position, pts[i]);
        st3(v.normal, n);
        v.uv[0] = uvs[i][0]; v.uv[1] = uvs[i][1];
        v.tangent[0] = t.x; v.tangent[1] = t.y; v.tangent[2] = t.z; v.tangent[3] = 1.0f;
        verts.push_back(v);
    }
    faces.push_back({base + 0, base + 1, base + 2, mat});
    faces.push_back({base + 0, base + 2, base + 3, mat});
}

// ---------------------------------------------------------------------------
// Radiance RGBE (.hdr): header lines, resolution "-Y H +X W", then scanlines
// either flat RGBE or new-style RLE.  Decoding m * 2^(e - 136) (zero exponent
// -> black), alpha forced to 1, as the reference's loader yields.
// ---------------------------------------------------------------------------
bool load_hdr(const std::string& path, std::vector<float>& rgba, int32_t& w, int32_t& h) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { set_error("cannot open " + path); return false; }
    std::unique_ptr<FILE, int (*)(FILE*)> guard(f, &std::fclose);
    char line[512];
    if (!std::fgets(line, sizeof(line), f) || std::strncmp(line, "#?", 2) != 0) { set_error(path + ": not a Radiance HDR file"); return false; }
    bool fmt_ok = false;
    for (;;) {
        if (!std::fgets(line, sizeof(line), f)) { set_error(path + ": truncated header"); return false; }
        if (line[0] == '\n' || line[0] == '\r') break;
        if (std::strncmp(line, "FORMAT=32-bit_rle_rgbe", 22) == 0) fmt_ok = true;
    }
    if (!fmt_ok) { set_error(path + ": unsupported HDR format (need 32-bit_rle_rgbe)"); return false; }
    if (!std::fgets(line, sizeof(line), f)) { set_error(path + ": missing resolution"); return false; }
    int hh = 0, ww = 0;
    if (std::sscanf(line, "-Y %d +X %d", &hh, &ww) != 2 || hh <= 0 || ww <= 0) { set_error(path + ": unsupported resolution line"); return false; }
    w = ww; h = hh;
    rgba.assign(static_cast<size_t>(w) * h * 4, 0.0f);
    std::vector<unsigned char> scan(static_cast<size_t>(w) * 4);
    auto decode = [&](int y) {
        for (int x = 0; x < w; ++x) {
            const unsigned char* p = &scan[static_cast<size_t>(x) * 4];
            float* o = &rgba[(static_cast<size_t>(y) * w + x) * 4];
            if (p[3] != 0) {
                const float s = static_cast<float>(std::ldexp(1.0f, p[3] - (128 + 8)));
                o[0] = p[0] * s; o[1] = p[1] * s; o[2] = p[2] * s;
            }
            o[3] = 1.0f;
        }
    };
    for (int y = 0; y < h; ++y) {
        unsigned char hdr4[4];
        if (std::fread(hdr4, 1, 4, f) != 4) { set_error(path + ": truncated pixel data"); return false; }
        const bool rle = (w >= 8 && w < 32768 && hdr4[0] == 2 && hdr4[1] == 2 && !(hdr4[2] & 0x80));
        if (!rle) {
            std::memcpy(&scan[0], hdr4, 4);
            if (w > 1 && std::fread(&scan[4], 1, static_cast<size_t>(w - 1) * 4, f) != static_cast<size_t>(w - 1) * 4) {
                set_error(path + ": truncated pixel data"); return false;
            }
            decode(y);
            continue;
        }
        if (((hdr4[2] << 8) | hdr4[3]) != w) { set_error(path + ": bad RLE scanline width"); return false; }
        for (int c = 0; c < 4; ++c) {
            int x = 0;
            while (x < w) {
                int cnt = std::fgetc(f);
                if (cnt == EOF) { set_error(path + ": truncated RLE data"); return false; }
                if (cnt > 128) {
                    cnt -= 128;
                    const int val = std::fgetc(f);
                    if (val == EOF || x + cnt > w) { set_error(path + ": bad RLE run"); return false; }
                    for (int k = 0; k < cnt; ++k) scan[static_cast<size_t>(x++) * 4 + c] = static_cast<unsigned char>(val);
                } else {
                    if (cnt == 0 || x + cnt > w) { set_error(path + ": bad RLE dump"); return false; }
                    for (int k = 0; k < cnt; ++k) {
                        const int val = std::fgetc(f);
                        if (val == EOF) { set_error(path + ": truncated RLE data"); return false; }
                        scan[static_cast<size_t>(x++) * 4 + c] = static_cast<unsigned char>(val);
                    }
                }
            }
        }
        decode(y);
    }
    return true;
}

// ---------------------------------------------------------------------------
// OBJ: v / vn / vt / f (1-based or negative indices).  Vertices are shared per
// distinct (v, vn, vt) triple in first-use order; positions by the transform,
// normals by its inverse transpose; a face whose first corner lacks a normal
// writes its face normal into its three vertices.  Polygons with more than
// three corners are fan-triangulated.
// ---------------------------------------------------------------------------
bool load_obj(const std::string& path, int mat, const float xform[16],
              std::vector<pt_vertex>& verts, std::vector<pt_face>& faces) {
    std::ifstream in(path);
    if (!in) { set_error("cannot open " + path); return false; }
    M4 T; std::memcpy(T.m, xform, sizeof(T.m));
    const M4 invT = m4_transpose(m4_inverse(T));
    std::vector<f3> vp, vn;
    std::vector<std::pair<float, float>> vt;
    struct Key { int v, n, t; bool operator==(const Key& o) const { return v == o.v && n == o.n && t == o.t; } };
    struct KeyHash { size_t operator()(const Key& k) const { return (size_t)k.v * 73856093u ^ (size_t)k.n * 19349663u ^ (size_t)k.t * 83492791u; } };
    std::unordered_map<Key, uint32_t, KeyHash> cache;
    auto fix = [](int idx, size_t n) { return idx < 0 ? static_cast<int>(n) + idx : idx - 1; };
    auto vertex_of = [&](const Key& k) -> uint32_t {
        auto it = cache.find(k);
        if (it != cache.end()) return it->second;
        pt_vertex v{};
        st3(v.position, m4_point(T, vp.at(k.v)));
        if (k.n >= 0) st3(v.normal, normalize(m4_vector(invT, vn.at(k.n))));
        if (k.t >= 0) { v.uv[0] = vt.at(k.t).first; v.uv[1] = vt.at(k.t).second; }
        const uint32_t id = static_cast<uint32_t>(verts.size());
        verts.push_back(v);
        cache.emplace(k, id);
        return id;
    };
    std::string ln;
    try {
        while (std::getline(in, ln)) {
            std::istringstream ss(ln);
            std::string tag;
            ss >> tag;
            if (tag == "v") { float x, y, z; ss >> x >> y >> z; vp.push_back(mk(x, y, z)); }
            else if (tag == "vn") { float x, y, z; ss >> x >> y >> z; vn.push_back(mk(x, y, z)); }
            else if (tag == "vt") { float u = 0, v = 0; ss >> u >> v; vt.emplace_back(u, v); }
            else if (tag == "f") {
                std::vector<Key> ks;
                std::string c;
                while (ss >> c) {
                    Key k{-1, -1, -1};
                    int a = 0, b = 0, d = 0;
                    if (std::sscanf(c.c_str(), "%d/%d/%d", &a, &b, &d) == 3) { k.v = fix(a, vp.size()); k.t = fix(b, vt.size()); k.n = fix(d, vn.size()); }
                    else if (std::sscanf(c.c_str(), "%d//%d", &a, &d) == 2) { k.v = fix(a, vp.size()); k.n = fix(d, vn.size()); }
                    else if (std::sscanf(c.c_str(), "%d/%d", &a, &b) == 2) { k.v = fix(a, vp.size()); k.t = fix(b, vt.size()); }
                    else if (std::sscanf(c.c_str(), "%d", &a) == 1) { k.v = fix(a, vp.size()); }
                    else throw std::runtime_error("bad face corner '" + c + "'");
                    ks.push_back(k);
                }
                for (size_t i = 1; i + 1 < ks.size(); ++i) {
                    const uint32_t i0 = vertex_of(ks[0]), i1 = vertex_of(ks[i]), i2 = vertex_of(ks[i + 1]);
                    if (ks[0].n < 0) {
                        const f3 fn = normalize(cross(ld3(verts[i1].position) - ld3(verts[i0].position),
                                                      ld3(verts[i2].position) - ld3(verts[i0].position)));
                        st3(verts[i0].normal, fn); st3(verts[i1].normal, fn); st3(verts[i2].normal, fn);
                    }
                    faces.push_back({i0, i1, i2, mat});
                }
            }
        }
    } catch (const std::exception& e) {
        set_error(path + ": " + e.what());
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Scene JSON.
// ---------------------------------------------------------------------------
bool load_json_scene(const std::string& path, HostScene& hs) {
    std::ifstream in(path, std::ios::binary);
    if (!in) { set_error("cannot open " + path); return false; }
    std::stringstream buf;
    buf << in.rdbuf();
    const std::string text = buf.str();
    try {
        const json::Value root = json::Parser(text).parse();
        if (root.kind != json::Value::Obj) throw json::Error{"scene root must be an object"};
        bool camera_set = false;
        if (root.has("camera")) {
            const json::Value& c = root["camera"];
            if (c.has("position")) st3(hs.camera.position, to_f3(c["position"]));
            if (c.has("lookAt")) st3(hs.camera.look_at, to_f3(c["lookAt"]));
            if (c.has("up")) st3(hs.camera.up, to_f3(c["up"]));
            if (c.has("fov")) hs.camera.fov = json::as_float(c["fov"]);
            if (c.has("aperture")) hs.camera.aperture = json::as_float(c["aperture"]);
            if (c.has("focalDistance")) hs.camera.focal_distance = json::as_float(c["focalDistance"]);
            if (c.has("resolution")) {
                hs.camera.width = json::as_int(c["resolution"][0]);
                hs.camera.height = json::as_int(c["resolution"][1]);
            }
            camera_set = true;
        }
        if (root.has("render")) {
            const json::Value& r = root["render"];
            if (r.has("spp")) hs.settings.spp = json::as_int(r["spp"]);
            if (r.has("samplePerFrame")) hs.settings.sample_per_frame = json::as_int(r["samplePerFrame"]);
            if (r.has("maxDepth")) hs.settings.max_depth = json::as_int(r["maxDepth"]);
            if (r.has("output")) hs.output_file = json::as_string(r["output"]);
            if (r.has("sampler")) {
                const std::string& s = json::as_string(r["sampler"]);
                if (s == "pcg") hs.settings.sampler_type = PT_SAMPLER_PCG;
                else if (s == "sobol") hs.settings.sampler_type = PT_SAMPLER_SOBOL;
            }
        }
        if (root.has("environment") && root["environment"].has("file")) {
            const std::string env = resolve_relative(path, json::as_string(root["environment"]["file"]));
            if (lower_ext(env) != ".hdr") throw json::Error{"environment '" + env + "': only .hdr maps are supported"};
            // The reference continues without an environment when the image
            // cannot be read (Part_2/src/scene/scene_loader.cpp:105-110).
            if (!load_hdr(env, hs.env_rgba, hs.env_w, hs.env_h)) { hs.env_rgba.clear(); hs.env_w = hs.env_h = 0; }
        }
        std::map<std::string, int> mat_index;
        if (root.has("materials")) {
            for (const auto& kv : *root["materials"].o) {
                pt_material m = default_material();
                apply_material_override(kv.second, m);
                mat_index[kv.first] = static_cast<int>(hs.materials.size());
                hs.materials.push_back(m);
            }
        }
        if (root.has("lights")) {
            const json::Value& ls = root["lights"];
            for (size_t i = 0; i < ls.size(); ++i) {
                const json::Value& jl = ls[i];
                pt_punctual_light L{};
                st3(L.position, mk(0.0f)); L.range = FLT_MAX; st3(L.color, mk(1.0f)); L.intensity = 1.0f;
                st3(L.direction, mk(0.0f, -1.0f, 0.0f)); L.inner_cone = 0.0f; L.outer_cone = 0.7071068f; L.type = 0;
                const std::string type = jl.has("type") ? json::as_string(jl["type"]) : std::string("point");
                L.type = type == "directional" ? 1 : (type == "spot" ? 2 : 0);
                if (jl.has("position")) st3(L.position, to_f3(jl["position"]));
                if (jl.has("direction")) st3(L.direction, normalize(to_f3(jl["direction"])));
                if (jl.has("color")) st3(L.color, to_f3(jl["color"]));
                if (jl.has("intensity")) L.intensity = json::as_float(jl["intensity"]);
                if (jl.has("range")) L.range = json::as_float(jl["range"]);
                if (jl.has("innerCone")) L.inner_cone = std::cos(json::as_float(jl["innerCone"]));
                if (jl.has("outerCone")) L.outer_cone = std::cos(json::as_float(jl["outerCone"]));
                hs.punctual.push_back(L);
            }
        }
        if (root.has("objects")) {
            const json::Value& objs = root["objects"];
            auto resolve_mat = [&](const json::Value& j) -> int {
                if (j.kind == json::Value::String) {
                    auto it = mat_index.find(j.s);
                    return it != mat_index.end() ? it->second : 0;
                }
                return json::as_int(j);
            };
            for (size_t i = 0; i < objs.size(); ++i) {
                const json::Value& o = objs[i];
                const std::string type = o.has("type") ? json::as_string(o["type"]) : std::string();
                if (type == "quad") {
                    const json::Value& v = o["vertices"];
                    float p[4][3];
                    for (int k = 0; k < 4; ++k) st3(p[k], to_f3(v[k]));
                    add_quad(p[0], p[1], p[2], p[3], resolve_mat(o["material"]), hs.vertices, hs.faces);
                } else if (type == "mesh") {
                    const std::string file = resolve_relative(path, json::as_string(o["file"]));
                    const int mid = resolve_mat(o["material"]);
                    const M4 T = parse_transform(o);
                    if (!load_obj(file, mid, T.m, hs.vertices, hs.faces)) return false;
                } else if (type == "gltf") {
                    throw json::Error{"glTF objects are not supported by this library"};
                }
            }
        }
        if (hs.materials.empty()) hs.materials.push_back(default_material());
        if (!camera_set) auto_fit_camera(hs.vertices, hs.camera);
    } catch (const json::Error& e) {
        set_error(path + ": " + e.msg);
        return false;
    } catch (const std::exception& e) {
        set_error(path + ": " + e.what());
        return false;
    }
    return true;
}

}  // namespace ptb
