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
//   objects[{type: quad|mesh|gltf, vertices|file, material, transform,
//            materialOverrides}]
// A path ending in .gltf / .glb is read as a glTF scene (see load_gltf).
#include <algorithm>
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
#include "image_decode.h"

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
// Radiance RGBE writer: ImageIO::write for .hdr (Part_2/src/io/image_io.cpp:
// 79-121: RGBA -> RGB, rows swapped when flip_y) through the reference's
// vendored stb_image_write v1.16 (stbi_write_hdr), restated from its
// published algorithm so that the files are byte for byte the same:
//   header "#?RADIANCE", "# Written by stb_image_write.h",
//     "FORMAT=32-bit_rle_rgbe", "EXPOSURE=          1.0000000000000", "",
//     "-Y <h> +X <w>";
//   pixel -> RGBE: m = max(r, max(g, b)); m < 1e-32 -> 0 0 0 0, else
//     s = frexp(m, e) * 256 / m, bytes (r s, g s, b s) truncated, e + 128;
//   scanline: width < 8 or >= 32768 -> flat RGBE; otherwise 2 2 w>>8 w&255
//     and each of the four byte planes run-length coded: literal stretches of
//     at most 128 bytes up to the next run of three equal bytes, runs of at
//     most 127 (length + 128, byte).
// ---------------------------------------------------------------------------
namespace {

void rgbe_of(const float* lin, unsigned char* out) {
    const float m12 = lin[1] > lin[2] ? lin[1] : lin[2];
    const float m = lin[0] > m12 ? lin[0] : m12;
    if (m < 1e-32f) { out[0] = out[1] = out[2] = out[3] = 0; return; }
    int e = 0;
    const float s = static_cast<float>(std::frexp(m, &e)) * 256.0f / m;
    for (int c = 0; c < 3; ++c) out[c] = static_cast<unsigned char>(static_cast<int>(lin[c] * s));
    out[3] = static_cast<unsigned char>(e + 128);
}

void hdr_scanline(std::string& o, int width, const float* rgb, std::vector<unsigned char>& plane) {
    if (width < 8 || width >= 32768) {
        unsigned char q[4];
        for (int x = 0; x < width; ++x) { rgbe_of(rgb + 3 * x, q); o.append(reinterpret_cast<char*>(q), 4); }
        return;
    }
    plane.resize(static_cast<size_t>(width) * 4);
    for (int x = 0; x < width; ++x) {
        unsigned char q[4];
        rgbe_of(rgb + 3 * x, q);
        for (int c = 0; c < 4; ++c) plane[static_cast<size_t>(c) * width + x] = q[c];
    }
    o.push_back(2); o.push_back(2);
    o.push_back(static_cast<char>((width & 0xff00) >> 8)); o.push_back(static_cast<char>(width & 0xff));
    for (int c = 0; c < 4; ++c) {
        const unsigned char* b = plane.data() + static_cast<size_t>(c) * width;
        int x = 0;
        while (x < width) {
            int r = x;   // start of the next run of three equal bytes, else width
            while (r + 2 < width && !(b[r] == b[r + 1] && b[r] == b[r + 2])) ++r;
            if (r + 2 >= width) r = width;
            while (x < r) {
                const int len = std::min(r - x, 128);
                o.push_back(static_cast<char>(len));
                o.append(reinterpret_cast<const char*>(b + x), len);
                x += len;
            }
            if (r + 2 < width) {
                while (r < width && b[r] == b[x]) ++r;
                while (x < r) {
                    const int len = std::min(r - x, 127);
                    o.push_back(static_cast<char>(len + 128));
                    o.push_back(static_cast<char>(b[x]));
                    x += len;
                }
            }
        }
    }
}

}  // namespace

bool write_hdr(const std::string& path, const float* rgba, int32_t w, int32_t h, bool flip_y) {
    if (!rgba || w <= 0 || h <= 0) { set_error("invalid image"); return false; }
    const size_t px = static_cast<size_t>(w) * h;
    std::vector<float> rgb(px * 3);
    for (size_t i = 0; i < px; ++i)
        for (int c = 0; c < 3; ++c) rgb[i * 3 + c] = rgba[i * 4 + c];
    if (flip_y) {
        const size_t row = static_cast<size_t>(w) * 3;
        for (int y = 0; y < h / 2; ++y)
            std::swap_ranges(rgb.begin() + y * row, rgb.begin() + (y + 1) * row, rgb.begin() + (h - 1 - y) * row);
    }
    std::string o = "#?RADIANCE\n# Written by stb_image_write.h\nFORMAT=32-bit_rle_rgbe\n";
    o += "EXPOSURE=          1.0000000000000\n\n-Y " + std::to_string(h) + " +X " + std::to_string(w) + "\n";
    std::vector<unsigned char> plane;
    for (int y = 0; y < h; ++y) hdr_scanline(o, w, rgb.data() + static_cast<size_t>(y) * w * 3, plane);
    std::FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) { set_error("cannot write " + path); return false; }
    const bool ok = std::fwrite(o.data(), 1, o.size(), fp) == o.size();
    std::fclose(fp);
    if (!ok) set_error("cannot write " + path);
    return ok;
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
// glTF 2.0 (GltfSceneLoader::load, Part_2/src/io/gltf_loader.cpp:588-734):
// .gltf (JSON with external or data-URI buffers) and .glb (JSON and BIN
// chunks).  The default scene's node tree is walked with world = parent *
// local (a node's matrix, else T * R * S); every triangle primitive adds its
// vertices (positions by the world transform, normals by its inverse
// transpose and normalised, tangents by the world transform; normals that
// are absent are the normalised sums of the primitive's face normals) and its
// faces (indexed by 8/16/32-bit indices, else consecutive triples), on
// material `offset + material` or 0 when it has none.  Materials: the metal-
// rough factors and the emissive, ior, transmission, clearcoat, sheen,
// specular, volume and anisotropy extensions and the alpha mode
// (loadMaterials, gltf_loader.cpp:172-347); KHR_lights_punctual lights sit at
// their node's origin looking down its -z.  Vertex attributes must be FLOAT
// (the reference reads them as floats).  Textures: the images (PNG or
// baseline JPEG, decoded by image_decode.cpp) with their samplers' wrap
// modes, and the materials' texture indices and KHR_texture_transform.
// ---------------------------------------------------------------------------
namespace {

std::string read_binary_file(const std::string& path) {
    std::FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) throw json::Error{"cannot open " + path};
    std::string out;
    if (std::fseek(fp, 0, SEEK_END) == 0) {
        const long len = std::ftell(fp);
        if (len > 0) {
            out.resize(static_cast<size_t>(len));
            std::fseek(fp, 0, SEEK_SET);
            if (std::fread(&out[0], 1, out.size(), fp) != out.size()) { std::fclose(fp); throw json::Error{"cannot read " + path}; }
        }
    }
    std::fclose(fp);
    return out;
}

std::string base64_decode(const std::string& s, size_t from) {
    auto val = [](char c) -> int {
        if (c >= 'A' && c <= 'Z') return c - 'A';
        if (c >= 'a' && c <= 'z') return c - 'a' + 26;
        if (c >= '0' && c <= '9') return c - '0' + 52;
        if (c == '+' || c == '-') return 62;
        if (c == '/' || c == '_') return 63;
        return -1;
    };
    std::string out;
    uint32_t acc = 0;
    int bits = 0;
    for (size_t i = from; i < s.size(); ++i) {
        if (s[i] == '=') break;
        const int v = val(s[i]);
        if (v < 0) continue;
        acc = (acc << 6) | static_cast<uint32_t>(v);
        bits += 6;
        if (bits >= 8) { bits -= 8; out.push_back(static_cast<char>((acc >> bits) & 0xffu)); }
    }
    return out;
}

struct GltfBuffer {
    const char* data = nullptr;
    size_t size = 0;
};

struct GltfDoc {
    json::Value root;
    std::string file;                 // the .glb (its BIN chunk is buffer 0)
    std::vector<std::string> owned;   // external and data-URI buffers
    std::vector<GltfBuffer> buffers;
};

GltfDoc read_gltf(const std::string& path) {
    GltfDoc d;
    d.file = read_binary_file(path);
    const std::string& bytes = d.file;
    std::string text;
    size_t bin_off = 0, bin_len = 0;
    bool have_bin = false;
    if (lower_ext(path) == ".glb") {
        auto u32 = [&](size_t o) {
            if (o + 4 > bytes.size()) throw json::Error{"truncated .glb"};
            uint32_t v;
            std::memcpy(&v, bytes.data() + o, 4);
            return v;
        };
        if (u32(0) != 0x46546C67u || u32(4) != 2u) throw json::Error{"not a glTF 2.0 binary"};
        size_t o = 12;
        while (o + 8 <= bytes.size()) {
            const uint32_t len = u32(o), type = u32(o + 4);
            if (o + 8 + static_cast<size_t>(len) > bytes.size()) throw json::Error{"truncated .glb chunk"};
            if (type == 0x4E4F534Au) text.assign(bytes, o + 8, len);
            else if (type == 0x004E4942u && !have_bin) { bin_off = o + 8; bin_len = len; have_bin = true; }
            o += 8 + ((static_cast<size_t>(len) + 3) & ~size_t(3));
        }
        if (text.empty()) throw json::Error{".glb without a JSON chunk"};
    } else {
        text = bytes;
    }
    d.root = json::Parser(text).parse();
    if (d.root.kind != json::Value::Obj) throw json::Error{"glTF root must be an object"};
    if (d.root.has("buffers")) {
        const json::Value& bs = d.root["buffers"];
        d.owned.reserve(bs.size());
        for (size_t i = 0; i < bs.size(); ++i) {
            const json::Value& b = bs[i];
            GltfBuffer buf;
            if (b.has("uri")) {
                const std::string& uri = json::as_string(b["uri"]);
                if (uri.compare(0, 5, "data:") == 0) {
                    const size_t comma = uri.find(',');
                    if (comma == std::string::npos) throw json::Error{"bad data URI"};
                    d.owned.push_back(base64_decode(uri, comma + 1));
                } else {
                    d.owned.push_back(read_binary_file(resolve_relative(path, uri)));
                }
                buf.data = d.owned.back().data();
                buf.size = d.owned.back().size();
            } else if (i == 0 && have_bin) {
                buf.data = bytes.data() + bin_off;
                buf.size = bin_len;
            } else {
                throw json::Error{"buffer " + std::to_string(i) + " has no data"};
            }
            if (b.has("byteLength") && buf.size < static_cast<size_t>(json::as_int(b["byteLength"])))
                throw json::Error{"buffer " + std::to_string(i) + " is shorter than its byteLength"};
            d.buffers.push_back(buf);
        }
    }
    return d;
}

int get_int(const json::Value& o, const char* k, int dflt) { return o.has(k) ? json::as_int(o[k]) : dflt; }
float get_num(const json::Value& o, const char* k, float dflt) { return o.has(k) ? json::as_float(o[k]) : dflt; }

struct GltfAccessor {
    const unsigned char* base = nullptr;
    size_t stride = 0, count = 0, elem = 0, avail = 0;   // avail: bytes from base to the buffer's end
    int comp = 0;
};

GltfAccessor gltf_accessor(const GltfDoc& d, int idx, size_t default_elem) {
    const json::Value& accs = d.root["accessors"];
    if (idx < 0 || static_cast<size_t>(idx) >= accs.size()) throw json::Error{"accessor index out of range"};
    const json::Value& a = accs[idx];
    if (!a.has("bufferView")) throw json::Error{"accessor without a bufferView (sparse accessors are not supported)"};
    const int bvi = json::as_int(a["bufferView"]);
    const json::Value& bvs = d.root["bufferViews"];
    if (bvi < 0 || static_cast<size_t>(bvi) >= bvs.size()) throw json::Error{"bufferView index out of range"};
    const json::Value& bv = bvs[bvi];
    const int bi = json::as_int(bv["buffer"]);
    if (bi < 0 || static_cast<size_t>(bi) >= d.buffers.size()) throw json::Error{"buffer index out of range"};
    const GltfBuffer& buf = d.buffers[bi];
    const size_t off = static_cast<size_t>(get_int(bv, "byteOffset", 0)) + static_cast<size_t>(get_int(a, "byteOffset", 0));
    if (off > buf.size) throw json::Error{"accessor offset outside its buffer"};
    GltfAccessor r;
    r.base = reinterpret_cast<const unsigned char*>(buf.data) + off;
    r.avail = buf.size - off;
    const int stride = get_int(bv, "byteStride", 0);
    r.stride = stride > 0 ? static_cast<size_t>(stride) : default_elem;
    r.count = static_cast<size_t>(json::as_int(a["count"]));
    r.comp = json::as_int(a["componentType"]);
    r.elem = default_elem;
    return r;
}

const float* acc_float(const GltfAccessor& a, size_t i, size_t nfloats) {
    const size_t at = i * a.stride;
    if (at + nfloats * 4 > a.avail) throw json::Error{"accessor reads past its buffer"};
    return reinterpret_cast<const float*>(a.base + at);
}

// glTF's column-major matrix or T * R * S (gltf_loader.cpp:53-88).
M4 gltf_node_transform(const json::Value& n) {
    if (n.has("matrix") && n["matrix"].size() == 16) {
        float m[16];
        for (int i = 0; i < 16; ++i) m[i] = json::as_float(n["matrix"][i]);
        M4 r;
        for (int row = 0; row < 4; ++row)
            for (int col = 0; col < 4; ++col) r.m[row * 4 + col] = m[col * 4 + row];
        return r;
    }
    M4 T = m4_identity(), R = m4_identity(), S = m4_identity();
    if (n.has("translation") && n["translation"].size() == 3)
        T = m4_translation(mk(json::as_float(n["translation"][0]), json::as_float(n["translation"][1]),
                              json::as_float(n["translation"][2])));
    if (n.has("rotation") && n["rotation"].size() == 4) {
        const float qx = json::as_float(n["rotation"][0]), qy = json::as_float(n["rotation"][1]);
        const float qz = json::as_float(n["rotation"][2]), qw = json::as_float(n["rotation"][3]);
        const float xx = qx * qx, yy = qy * qy, zz = qz * qz, xy = qx * qy, xz = qx * qz, yz = qy * qz;
        const float wx = qw * qx, wy = qw * qy, wz = qw * qz;
        const float r[16] = {1 - 2 * (yy + zz), 2 * (xy - wz), 2 * (xz + wy), 0,
                             2 * (xy + wz), 1 - 2 * (xx + zz), 2 * (yz - wx), 0,
                             2 * (xz - wy), 2 * (yz + wx), 1 - 2 * (xx + yy), 0,
                             0, 0, 0, 1};
        std::memcpy(R.m, r, sizeof(r));
    }
    if (n.has("scale") && n["scale"].size() == 3) {
        S.m[0] = json::as_float(n["scale"][0]);
        S.m[5] = json::as_float(n["scale"][1]);
        S.m[10] = json::as_float(n["scale"][2]);
    }
    return m4_mul(m4_mul(T, R), S);
}

// Texture index of a textureInfo object (index + the scene's texture offset), else -1.
int gltf_tex_index(const json::Value& o, const char* key, int tex_offset) {
    if (!o.has(key)) return -1;
    const json::Value& info = o[key];
    if (!info.has("index")) return -1;
    const int i = json::as_int(info["index"]);
    return i >= 0 ? i + tex_offset : -1;
}

// glTF textures (loadTextures, gltf_loader.cpp:112-147): each texture's image
// (a bufferView, a data: URI or a file beside the glTF) decoded to 8-bit RGBA
// and stored as value / 255, with its sampler's wrap modes; a texture without
// a source image stays empty.
void gltf_textures(const GltfDoc& d, const std::string& path, std::vector<HostTextureImage>& out) {
    if (!d.root.has("textures")) return;
    const json::Value& ts = d.root["textures"];
    const size_t n_images = d.root.has("images") ? d.root["images"].size() : 0;
    std::vector<DecodedImage> decoded(n_images);
    std::vector<bool> done(n_images, false);
    for (size_t i = 0; i < ts.size(); ++i) {
        const json::Value& t = ts[i];
        HostTextureImage img;
        const int src = get_int(t, "source", -1);
        if (src >= 0 && static_cast<size_t>(src) < n_images) {
            if (!done[src]) {
                const json::Value& im = d.root["images"][static_cast<size_t>(src)];
                std::string owned;
                const uint8_t* bytes = nullptr;
                size_t size = 0;
                if (im.has("bufferView")) {
                    const int bvi = json::as_int(im["bufferView"]);
                    const json::Value& bvs = d.root["bufferViews"];
                    if (bvi < 0 || static_cast<size_t>(bvi) >= bvs.size()) throw json::Error{"image bufferView out of range"};
                    const json::Value& bv = bvs[static_cast<size_t>(bvi)];
                    const int bi = json::as_int(bv["buffer"]);
                    if (bi < 0 || static_cast<size_t>(bi) >= d.buffers.size()) throw json::Error{"image buffer out of range"};
                    const size_t off = static_cast<size_t>(get_int(bv, "byteOffset", 0));
                    const size_t len = static_cast<size_t>(json::as_int(bv["byteLength"]));
                    if (off + len > d.buffers[bi].size) throw json::Error{"image bufferView beyond its buffer"};
                    bytes = reinterpret_cast<const uint8_t*>(d.buffers[bi].data) + off;
                    size = len;
                } else if (im.has("uri")) {
                    const std::string& uri = json::as_string(im["uri"]);
                    if (uri.compare(0, 5, "data:") == 0) {
                        const size_t comma = uri.find(',');
                        if (comma == std::string::npos) throw json::Error{"bad image data URI"};
                        owned = base64_decode(uri, comma + 1);
                    } else {
                        owned = read_binary_file(resolve_relative(path, uri));
                    }
                    bytes = reinterpret_cast<const uint8_t*>(owned.data());
                    size = owned.size();
                } else {
                    throw json::Error{"image " + std::to_string(src) + " has neither a bufferView nor a uri"};
                }
                std::string err;
                if (!decode_image(bytes, size, decoded[src], err))
                    throw json::Error{"image " + std::to_string(src) + ": " + err};
                done[src] = true;
            }
            const DecodedImage& di = decoded[src];
            img.width = di.width;
            img.height = di.height;
            img.rgba.resize(di.rgba.size());
            for (size_t k = 0; k < di.rgba.size(); ++k) img.rgba[k] = static_cast<float>(di.rgba[k]) / 255.0f;
        }
        const int smp = get_int(t, "sampler", -1);
        if (smp >= 0 && d.root.has("samplers") && static_cast<size_t>(smp) < d.root["samplers"].size()) {
            const json::Value& sm = d.root["samplers"][static_cast<size_t>(smp)];
            img.wrap_s = get_int(sm, "wrapS", 10497);
            img.wrap_t = get_int(sm, "wrapT", 10497);
        }
        out.push_back(std::move(img));
    }
}

void gltf_materials(const GltfDoc& d, std::vector<pt_material>& out, std::vector<std::string>& names,
                    int tex_offset) {
    if (!d.root.has("materials")) return;
    const json::Value& ms = d.root["materials"];
    for (size_t i = 0; i < ms.size(); ++i) {
        const json::Value& g = ms[i];
        pt_material m = default_material();
        names.push_back(g.has("name") ? json::as_string(g["name"]) : std::string());
        // glTF defaults: base colour (1, 1, 1, 1), metallic 1, roughness 1, no emission
        float bc[4] = {1.0f, 1.0f, 1.0f, 1.0f};
        float metallic = 1.0f, roughness = 1.0f;
        if (g.has("pbrMetallicRoughness")) {
            const json::Value& p = g["pbrMetallicRoughness"];
            if (p.has("baseColorFactor"))
                for (size_t k = 0; k < 4 && k < p["baseColorFactor"].size(); ++k) bc[k] = json::as_float(p["baseColorFactor"][k]);
            metallic = get_num(p, "metallicFactor", 1.0f);
            roughness = get_num(p, "roughnessFactor", 1.0f);
            m.base_color_tex = gltf_tex_index(p, "baseColorTexture", tex_offset);
            if (m.base_color_tex >= 0 && p["baseColorTexture"].has("extensions") &&
                p["baseColorTexture"]["extensions"].has("KHR_texture_transform")) {
                // readTextureTransform (gltf_loader.cpp:158-170)
                const json::Value& tt = p["baseColorTexture"]["extensions"]["KHR_texture_transform"];
                if (tt.has("offset") && tt["offset"].size() >= 2) {
                    m.uv_offset_x = json::as_float(tt["offset"][0]);
                    m.uv_offset_y = json::as_float(tt["offset"][1]);
                }
                if (tt.has("scale") && tt["scale"].size() >= 2) {
                    m.uv_scale_x = json::as_float(tt["scale"][0]);
                    m.uv_scale_y = json::as_float(tt["scale"][1]);
                }
                if (tt.has("rotation")) m.uv_rotation = json::as_float(tt["rotation"]);
            }
            m.metallic_roughness_tex = gltf_tex_index(p, "metallicRoughnessTexture", tex_offset);
        }
        m.normal_tex = gltf_tex_index(g, "normalTexture", tex_offset);
        if (m.normal_tex >= 0) m.normal_scale = get_num(g["normalTexture"], "scale", 1.0f);
        m.emissive_tex = gltf_tex_index(g, "emissiveTexture", tex_offset);
        m.occlusion_tex = gltf_tex_index(g, "occlusionTexture", tex_offset);
        if (m.occlusion_tex >= 0) m.occlusion_strength = get_num(g["occlusionTexture"], "strength", 1.0f);
        m.base_color[0] = bc[0]; m.base_color[1] = bc[1]; m.base_color[2] = bc[2];
        m.base_alpha = bc[3];
        m.metallic = metallic;
        m.roughness = roughness;
        float em[3] = {0.0f, 0.0f, 0.0f};
        if (g.has("emissiveFactor"))
            for (size_t k = 0; k < 3 && k < g["emissiveFactor"].size(); ++k) em[k] = json::as_float(g["emissiveFactor"][k]);
        m.emissive[0] = em[0]; m.emissive[1] = em[1]; m.emissive[2] = em[2];
        if (em[0] > 0 || em[1] > 0 || em[2] > 0) m.emissive_strength = 1.0f;
        m.double_sided = (g.has("doubleSided") && json::as_bool(g["doubleSided"])) ? 1 : 0;
        if (g.has("extensions")) {
            const json::Value& x = g["extensions"];
            auto ext = [&](const char* k) -> const json::Value* { return x.has(k) ? &x[k] : nullptr; };
            if (const json::Value* e = ext("KHR_materials_emissive_strength"))
                if (e->has("emissiveStrength")) m.emissive_strength = json::as_float((*e)["emissiveStrength"]);
            if (const json::Value* e = ext("KHR_materials_ior"))
                if (e->has("ior")) m.ior = json::as_float((*e)["ior"]);
            if (const json::Value* e = ext("KHR_materials_transmission")) {
                if (e->has("transmissionFactor")) m.spec_trans = json::as_float((*e)["transmissionFactor"]);
                m.transmission_tex = gltf_tex_index(*e, "transmissionTexture", tex_offset);
            }
            if (const json::Value* e = ext("KHR_materials_clearcoat")) {
                if (e->has("clearcoatFactor")) m.clearcoat = json::as_float((*e)["clearcoatFactor"]);
                if (e->has("clearcoatRoughnessFactor"))
                    m.clearcoat_roughness = json::as_float((*e)["clearcoatRoughnessFactor"]);
                m.clearcoat_tex = gltf_tex_index(*e, "clearcoatTexture", tex_offset);
                m.clearcoat_roughness_tex = gltf_tex_index(*e, "clearcoatRoughnessTexture", tex_offset);
                m.clearcoat_normal_tex = gltf_tex_index(*e, "clearcoatNormalTexture", tex_offset);
            }
            if (const json::Value* e = ext("KHR_materials_sheen")) {
                if (e->has("sheenRoughnessFactor")) m.sheen = json::as_float((*e)["sheenRoughnessFactor"]);
                if (e->has("sheenColorFactor") && (*e)["sheenColorFactor"].size() >= 3) {
                    const json::Value& c = (*e)["sheenColorFactor"];
                    m.sheen_color_r = json::as_float(c[0]); m.sheen_color_g = json::as_float(c[1]);
                    m.sheen_color_b = json::as_float(c[2]);
                }
                m.sheen_color_tex = gltf_tex_index(*e, "sheenColorTexture", tex_offset);
                m.sheen_roughness_tex = gltf_tex_index(*e, "sheenRoughnessTexture", tex_offset);
            }
            if (const json::Value* e = ext("KHR_materials_specular")) {
                if (e->has("specularFactor")) m.specular_factor = json::as_float((*e)["specularFactor"]);
                if (e->has("specularColorFactor") && (*e)["specularColorFactor"].size() >= 3) {
                    const json::Value& c = (*e)["specularColorFactor"];
                    m.specular_color_r = json::as_float(c[0]); m.specular_color_g = json::as_float(c[1]);
                    m.specular_color_b = json::as_float(c[2]);
                }
            }
            if (const json::Value* e = ext("KHR_materials_volume")) {
                if (e->has("thicknessFactor")) m.thickness_factor = json::as_float((*e)["thicknessFactor"]);
                if (e->has("attenuationDistance")) m.attenuation_distance = json::as_float((*e)["attenuationDistance"]);
                if (e->has("attenuationColor") && (*e)["attenuationColor"].size() >= 3) {
                    const json::Value& c = (*e)["attenuationColor"];
                    m.att_color_r = json::as_float(c[0]); m.att_color_g = json::as_float(c[1]);
                    m.att_color_b = json::as_float(c[2]);
                }
            }
            if (const json::Value* e = ext("KHR_materials_anisotropy")) {
                if (e->has("anisotropyStrength")) m.anisotropic = json::as_float((*e)["anisotropyStrength"]);
                if (e->has("anisotropyRotation")) m.anisotropy_rotation = json::as_float((*e)["anisotropyRotation"]);
            }
        }
        const std::string mode = g.has("alphaMode") ? json::as_string(g["alphaMode"]) : std::string("OPAQUE");
        if (mode == "MASK") { m.alpha_mode = 1; m.alpha_cutoff = get_num(g, "alphaCutoff", 0.5f); }
        else if (mode == "BLEND") m.alpha_mode = 2;
        out.push_back(m);
    }
}

void gltf_primitive(const GltfDoc& d, const json::Value& prim, const M4& world, int mat_offset,
                    std::vector<pt_vertex>& verts, std::vector<pt_face>& faces) {
    const int mode = get_int(prim, "mode", -1);
    if (mode != 4 && mode != -1) return;
    if (!prim.has("attributes") || !prim["attributes"].has("POSITION")) return;
    const json::Value& at = prim["attributes"];
    auto float_attr = [&](const char* name, size_t n) {
        GltfAccessor a = gltf_accessor(d, json::as_int(at[name]), n * 4);
        if (a.comp != 5126) throw json::Error{std::string("glTF attribute ") + name + " must be FLOAT"};
        return a;
    };
    const GltfAccessor pos = float_attr("POSITION", 3);
    const bool has_n = at.has("NORMAL"), has_uv = at.has("TEXCOORD_0"), has_t = at.has("TANGENT");
    GltfAccessor nrm, uv, tan;
    if (has_n) nrm = float_attr("NORMAL", 3);
    if (has_uv) uv = float_attr("TEXCOORD_0", 2);
    if (has_t) tan = float_attr("TANGENT", 4);
    const M4 nmat = m4_transpose(m4_inverse(world));
    const uint32_t base = static_cast<uint32_t>(verts.size());
    const size_t nv = pos.count;
    if (nv * pos.stride > pos.avail + pos.stride) throw json::Error{"POSITION accessor reads past its buffer"};
    verts.reserve(verts.size() + nv);
    for (size_t v = 0; v < nv; ++v) {
        pt_vertex o{};
        const float* p = acc_float(pos, v, 3);
        st3(o.position, m4_point(world, mk(p[0], p[1], p[2])));
        if (has_n) {
            const float* q = acc_float(nrm, v, 3);
            st3(o.normal, normalize(m4_vector(nmat, mk(q[0], q[1], q[2]))));
        }
        if (has_uv) {
            const float* q = acc_float(uv, v, 2);
            o.uv[0] = q[0]; o.uv[1] = q[1];
        }
        if (has_t) {
            const float* q = acc_float(tan, v, 4);
            const f3 t = normalize(m4_vector(world, mk(q[0], q[1], q[2])));
            o.tangent[0] = t.x; o.tangent[1] = t.y; o.tangent[2] = t.z; o.tangent[3] = q[3];
        }
        verts.push_back(o);
    }
    const int mat = prim.has("material") && json::as_int(prim["material"]) >= 0
                        ? json::as_int(prim["material"]) + mat_offset : 0;
    size_t expected;
    if (prim.has("indices") && json::as_int(prim["indices"]) >= 0) {
        const GltfAccessor ia = gltf_accessor(d, json::as_int(prim["indices"]), 1);
        const size_t tris = ia.count / 3;
        expected = tris;
        faces.reserve(faces.size() + tris);
        const size_t width = ia.comp == 5121 ? 1 : (ia.comp == 5123 ? 2 : (ia.comp == 5125 ? 4 : 0));
        if (width && tris * 3 * width > ia.avail) throw json::Error{"index accessor reads past its buffer"};
        for (size_t t = 0; t < tris; ++t) {
            uint32_t i[3];
            for (int k = 0; k < 3; ++k) {
                const unsigned char* src = ia.base + (t * 3 + k) * width;
                if (width == 1) i[k] = src[0];
                else if (width == 2) { uint16_t x; std::memcpy(&x, src, 2); i[k] = x; }
                else if (width == 4) std::memcpy(&i[k], src, 4);
            }
            if (!width) continue;   // other index types: no faces (as the reference)
            for (int k = 0; k < 3; ++k)
                if (i[k] >= nv) throw json::Error{"glTF index " + std::to_string(i[k]) + " out of range"};
            faces.push_back({base + i[0], base + i[1], base + i[2], mat});
        }
    } else {
        expected = nv / 3;
        for (size_t t = 0; t < nv / 3; ++t) {
            const uint32_t i = static_cast<uint32_t>(t * 3);
            faces.push_back({base + i, base + i + 1, base + i + 2, mat});
        }
    }
    if (!has_n) {
        for (size_t v = 0; v < nv; ++v) st3(verts[base + v].normal, mk(0.0f));
        const size_t first = faces.size() >= expected ? faces.size() - expected : 0;
        for (size_t fi = first; fi < faces.size(); ++fi) {
            const pt_face& f = faces[fi];
            const f3 fn = cross(ld3(verts[f.v1].position) - ld3(verts[f.v0].position),
                                ld3(verts[f.v2].position) - ld3(verts[f.v0].position));
            for (uint32_t vi : {f.v0, f.v1, f.v2}) st3(verts[vi].normal, ld3(verts[vi].normal) + fn);
        }
        for (size_t v = 0; v < nv; ++v) {
            const f3 n = ld3(verts[base + v].normal);
            const float len = length(n);
            if (len > 0.0f) st3(verts[base + v].normal, n / len);
        }
    }
}

struct GltfLight { int type = 0; f3 color = mk(1.0f); float intensity = 1.0f, range = 1e30f, inner = 0.0f, outer = 0.7853982f; };

struct GltfOptions {
    M4 transform = m4_identity();
    bool load_camera = true, auto_fit_camera = true, add_default_lights = true, load_environment = true;
};

// PunctualLight's defaults (Part_2/src/lights/punctual_light.h:14-25).
pt_punctual_light default_punctual() {
    pt_punctual_light L{};
    st3(L.position, mk(0.0f)); L.range = FLT_MAX; st3(L.color, mk(1.0f)); L.intensity = 1.0f;
    st3(L.direction, mk(0.0f, -1.0f, 0.0f)); L.inner_cone = 0.0f; L.outer_cone = 0.7071068f; L.type = 0;
    return L;
}

void gltf_nodes(const GltfDoc& d, int idx, const M4& parent, int mat_offset, const std::vector<GltfLight>& lights,
                HostScene& hs, bool& camera_set, int depth) {
    const json::Value& nodes = d.root["nodes"];
    if (idx < 0 || static_cast<size_t>(idx) >= nodes.size()) return;
    if (depth > 256) throw json::Error{"glTF node hierarchy too deep (a cycle?)"};
    const json::Value& n = nodes[idx];
    const M4 world = m4_mul(parent, gltf_node_transform(n));
    const int mesh = get_int(n, "mesh", -1);
    if (mesh >= 0 && d.root.has("meshes") && static_cast<size_t>(mesh) < d.root["meshes"].size()) {
        const json::Value& m = d.root["meshes"][mesh];
        if (m.has("primitives"))
            for (size_t p = 0; p < m["primitives"].size(); ++p)
                gltf_primitive(d, m["primitives"][p], world, mat_offset, hs.vertices, hs.faces);
    }
    const int cam = get_int(n, "camera", -1);
    if (!camera_set && cam >= 0 && d.root.has("cameras") && static_cast<size_t>(cam) < d.root["cameras"].size()) {
        const json::Value& c = d.root["cameras"][cam];
        if (c.has("type") && json::as_string(c["type"]) == "perspective" && c.has("perspective")) {
            const json::Value& p = c["perspective"];
            const f3 pos = m4_point(world, mk(0.0f));
            st3(hs.camera.position, pos);
            st3(hs.camera.look_at, pos + normalize(m4_vector(world, mk(0.0f, 0.0f, -1.0f))));
            st3(hs.camera.up, normalize(m4_vector(world, mk(0.0f, 1.0f, 0.0f))));
            const double yfov = p.has("yfov") ? (p["yfov"].kind == json::Value::Int ? double(p["yfov"].i) : p["yfov"].d) : 0.0;
            hs.camera.fov = static_cast<float>(yfov * 180.0 / 3.14159265358979323846);
            const double aspect = p.has("aspectRatio") ? (p["aspectRatio"].kind == json::Value::Int ? double(p["aspectRatio"].i) : p["aspectRatio"].d) : 0.0;
            if (aspect > 0.0) hs.camera.width = static_cast<int>(aspect * hs.camera.height);
            camera_set = true;
        }
    }
    if (n.has("extensions") && n["extensions"].has("KHR_lights_punctual") &&
        n["extensions"]["KHR_lights_punctual"].has("light")) {
        const int li = json::as_int(n["extensions"]["KHR_lights_punctual"]["light"]);
        if (li >= 0 && static_cast<size_t>(li) < lights.size()) {
            const GltfLight& g = lights[li];
            pt_punctual_light L = default_punctual();
            L.type = g.type;
            st3(L.color, g.color);
            L.intensity = g.intensity;
            L.range = g.range;
            st3(L.position, m4_point(world, mk(0.0f)));
            st3(L.direction, normalize(m4_vector(world, mk(0.0f, 0.0f, -1.0f))));
            L.inner_cone = std::cos(g.inner);
            L.outer_cone = std::cos(g.outer);
            hs.punctual.push_back(L);
        }
    }
    if (n.has("children"))
        for (size_t c = 0; c < n["children"].size(); ++c)
            gltf_nodes(d, json::as_int(n["children"][c]), world, mat_offset, lights, hs, camera_set, depth + 1);
}

// Appends one glTF file to `hs`; returns the names of its materials.
std::vector<std::string> load_gltf(const std::string& path, HostScene& hs, const GltfOptions& opt) {
    const GltfDoc d = read_gltf(path);
    const int mat_offset = static_cast<int>(hs.materials.size());
    const int tex_offset = static_cast<int>(hs.textures.size());
    gltf_textures(d, path, hs.textures);
    std::vector<std::string> names;
    gltf_materials(d, hs.materials, names, tex_offset);
    if (hs.materials.empty()) hs.materials.push_back(default_material());
    std::vector<GltfLight> lights;
    if (d.root.has("extensions") && d.root["extensions"].has("KHR_lights_punctual") &&
        d.root["extensions"]["KHR_lights_punctual"].has("lights")) {
        const json::Value& ls = d.root["extensions"]["KHR_lights_punctual"]["lights"];
        for (size_t i = 0; i < ls.size(); ++i) {
            const json::Value& l = ls[i];
            GltfLight g;
            if (l.has("type")) {
                const std::string& t = json::as_string(l["type"]);
                g.type = t == "directional" ? 1 : (t == "spot" ? 2 : 0);
            }
            if (l.has("color") && l["color"].size() >= 3) g.color = to_f3(l["color"]);
            g.intensity = get_num(l, "intensity", g.intensity);
            g.range = get_num(l, "range", g.range);
            if (l.has("spot")) {
                g.inner = get_num(l["spot"], "innerConeAngle", g.inner);
                g.outer = get_num(l["spot"], "outerConeAngle", g.outer);
            }
            lights.push_back(g);
        }
    }
    bool camera_set = !opt.load_camera;
    const int scene = get_int(d.root, "scene", 0) >= 0 ? get_int(d.root, "scene", 0) : 0;
    if (d.root.has("scenes") && static_cast<size_t>(scene) < d.root["scenes"].size() && d.root.has("nodes")) {
        const json::Value& s = d.root["scenes"][scene];
        if (s.has("nodes"))
            for (size_t i = 0; i < s["nodes"].size(); ++i)
                gltf_nodes(d, json::as_int(s["nodes"][i]), opt.transform, mat_offset, lights, hs, camera_set, 0);
    }
    if (opt.auto_fit_camera && !camera_set && !hs.vertices.empty()) auto_fit_camera(hs.vertices, hs.camera);
    if (opt.load_environment && hs.env_w <= 0 && hs.env_h <= 0) {
        // the reference looks upward from the file for models/<its default sky>
        std::string dir = path;
        for (int up = 0; up < 64; ++up) {
            const size_t slash = dir.find_last_of('/');
            if (slash == std::string::npos) break;
            dir = dir.substr(0, slash);
            const std::string cand = (dir.empty() ? std::string() : dir) + "/models/kloofendal_48d_partly_cloudy_puresky_4k.hdr";
            std::ifstream probe(cand, std::ios::binary);
            if (probe) {
                if (!load_hdr(cand, hs.env_rgba, hs.env_w, hs.env_h)) { hs.env_rgba.clear(); hs.env_w = hs.env_h = 0; }
                break;
            }
            if (dir.empty()) break;
        }
    }
    bool emissive = false;
    for (const pt_material& m : hs.materials)
        if (m.emissive_strength > 0.0f && (m.emissive[0] > 0.0f || m.emissive[1] > 0.0f || m.emissive[2] > 0.0f)) emissive = true;
    if (opt.add_default_lights && !(hs.env_w > 0 && hs.env_h > 0) && !emissive && hs.punctual.empty()) {
        pt_punctual_light key = default_punctual(), fill = default_punctual();
        key.type = 1; st3(key.direction, normalize(mk(-0.5f, -0.8f, -0.6f))); st3(key.color, mk(1.0f, 0.95f, 0.9f));
        key.intensity = 3.0f;
        fill.type = 1; st3(fill.direction, normalize(mk(0.6f, -0.3f, 0.5f))); st3(fill.color, mk(0.7f, 0.8f, 1.0f));
        fill.intensity = 1.0f;
        hs.punctual.push_back(key);
        hs.punctual.push_back(fill);
    }
    return names;
}

}  // namespace

// ---------------------------------------------------------------------------
// Scene JSON.
// ---------------------------------------------------------------------------
bool load_json_scene(const std::string& path, HostScene& hs) {
    const std::string ext = lower_ext(path);
    if (ext == ".gltf" || ext == ".glb") {   // SceneLoader::load (scene_loader.cpp:280-289)
        try {
            load_gltf(path, hs, GltfOptions{});
        } catch (const json::Error& e) {
            set_error(path + ": " + e.msg);
            return false;
        } catch (const std::exception& e) {
            set_error(path + ": " + e.what());
            return false;
        }
        return true;
    }
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
                    // SceneLoader's glTF objects (scene_loader.cpp:162-193): the object's
                    // transform, no camera / default lights / environment, then the
                    // object's materialOverrides applied by glTF material name
                    GltfOptions opt;
                    opt.transform = parse_transform(o);
                    opt.load_camera = opt.auto_fit_camera = opt.add_default_lights = opt.load_environment = false;
                    const int first = static_cast<int>(hs.materials.size());
                    const std::vector<std::string> names =
                        load_gltf(resolve_relative(path, json::as_string(o["file"])), hs, opt);
                    if (o.has("materialOverrides")) {
                        for (const auto& kv : *o["materialOverrides"].o)
                            for (size_t k = 0; k < names.size(); ++k)
                                if (names[k] == kv.first && first + k < hs.materials.size())
                                    apply_material_override(kv.second, hs.materials[first + k]);
                    }
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
