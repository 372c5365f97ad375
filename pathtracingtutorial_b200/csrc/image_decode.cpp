// image_decode.cpp -- PNG and baseline JPEG into 8-bit RGBA (see image_decode.h).
//
// PNG (W3C PNG specification, 2nd edition): the IDAT stream is inflated by
// zlib, each scanline's filter (None, Sub, Up, Average, Paeth) is undone, and
// Adam7-interlaced passes are scattered to their pixels.  Colour types grey,
// RGB, palette, grey + alpha and RGBA at every legal bit depth; tRNS keys and
// palette alphas give alpha 0..255; 16-bit samples keep their high byte and
// sub-byte grey samples are scaled to 0..255.
//
// JPEG (ITU-T T.81): baseline and extended sequential Huffman frames (SOF0,
// SOF1), 8-bit precision, one or three components with any integer sampling
// factors, interleaved and single-component scans, restart intervals.  Blocks
// are dequantised and inverse transformed by the separable 8 x 8 IDCT of the
// specification (A.3.3) in double precision, level-shifted and clamped;
// chroma planes at half resolution are upsampled with a triangle filter
// (3/4 near sample, 1/4 far sample) and other ratios by replication; colour
// is converted with the JFIF equations, or kept as RGB when an Adobe APP14
// transform of 0 (or component ids 'R', 'G', 'B') says so.  Progressive and
// arithmetic-coded files are rejected with an error.
#include "image_decode.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstring>

namespace ptb {

namespace {

uint32_t be32(const uint8_t* p) {
    return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | uint32_t(p[3]);
}
uint16_t be16(const uint8_t* p) { return static_cast<uint16_t>((p[0] << 8) | p[1]); }

// ---------------------------------------------------------------------------
// PNG
// ---------------------------------------------------------------------------
bool inflate_exact(const std::vector<uint8_t>& in, std::vector<uint8_t>& out, size_t expect, std::string& err) {
    out.assign(expect, 0);
    if (in.size() > 0xffffffffull || expect > 0xffffffffull) { err = "PNG: image data too large"; return false; }
    z_stream zs;
    std::memset(&zs, 0, sizeof(zs));
    if (inflateInit(&zs) != Z_OK) { err = "PNG: inflateInit failed"; return false; }
    zs.next_in = const_cast<Bytef*>(in.data());
    zs.avail_in = static_cast<uInt>(in.size());
    zs.next_out = out.data();
    zs.avail_out = static_cast<uInt>(expect);
    const int rc = inflate(&zs, Z_FINISH);
    const size_t got = expect - zs.avail_out;
    inflateEnd(&zs);
    if (got != expect) { err = "PNG: image data ends early"; return false; }
    if (rc != Z_STREAM_END && rc != Z_BUF_ERROR && rc != Z_OK) { err = "PNG: corrupt image data"; return false; }
    return true;
}

uint8_t paeth(int a, int b, int c) {
    const int p = a + b - c;
    const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return static_cast<uint8_t>(a);
    if (pb <= pc) return static_cast<uint8_t>(b);
    return static_cast<uint8_t>(c);
}

// Undo the filters of `rows` scanlines of `rowbytes` bytes (each preceded by
// its filter byte in `src`) into `dst` (rows * rowbytes).
bool unfilter(const uint8_t* src, int rows, size_t rowbytes, int bpp, uint8_t* dst, std::string& err) {
    std::vector<uint8_t> zero(rowbytes, 0);
    for (int y = 0; y < rows; ++y) {
        const uint8_t f = src[0];
        const uint8_t* cur = src + 1;
        uint8_t* out = dst + static_cast<size_t>(y) * rowbytes;
        const uint8_t* prev = y ? out - rowbytes : zero.data();
        for (size_t i = 0; i < rowbytes; ++i) {
            const int a = i >= static_cast<size_t>(bpp) ? out[i - bpp] : 0;
            const int b = prev[i];
            const int c = i >= static_cast<size_t>(bpp) ? prev[i - bpp] : 0;
            int v = cur[i];
            switch (f) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) >> 1; break;
                case 4: v += paeth(a, b, c); break;
                default: err = "PNG: unknown filter type " + std::to_string(f); return false;
            }
            out[i] = static_cast<uint8_t>(v);
        }
        src += 1 + rowbytes;
    }
    return true;
}

}  // namespace

bool decode_png(const uint8_t* p, size_t n, DecodedImage& out, std::string& err) {
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (n < 8 || std::memcmp(p, sig, 8) != 0) { err = "PNG: bad signature"; return false; }
    uint32_t w = 0, h = 0;
    int bd = 0, ct = -1, interlace = 0;
    std::vector<uint8_t> plte, trns, idat;
    bool have_ihdr = false;
    size_t o = 8;
    while (o + 12 <= n) {
        const uint32_t len = be32(p + o);
        if (len > n - o - 12) { err = "PNG: truncated chunk"; return false; }
        const uint8_t* type = p + o + 4;
        const uint8_t* d = p + o + 8;
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len < 13) { err = "PNG: short IHDR"; return false; }
            w = be32(d); h = be32(d + 4); bd = d[8]; ct = d[9]; interlace = d[12];
            if (d[10] != 0 || d[11] != 0) { err = "PNG: unknown compression or filter method"; return false; }
            have_ihdr = true;
        } else if (!std::memcmp(type, "PLTE", 4)) {
            plte.assign(d, d + len);
        } else if (!std::memcmp(type, "tRNS", 4)) {
            trns.assign(d, d + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), d, d + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        } else if (!(type[0] & 0x20)) {
            err = std::string("PNG: unknown critical chunk ") + std::string(reinterpret_cast<const char*>(type), 4);
            return false;
        }
        o += 12 + len;
    }
    if (!have_ihdr || idat.empty()) { err = "PNG: missing IHDR or image data"; return false; }
    int ch = 0;
    switch (ct) {
        case 0: ch = 1; break;
        case 2: ch = 3; break;
        case 3: ch = 1; break;
        case 4: ch = 2; break;
        case 6: ch = 4; break;
        default: err = "PNG: unknown colour type " + std::to_string(ct); return false;
    }
    const bool bd_ok = (ct == 0 && (bd == 1 || bd == 2 || bd == 4 || bd == 8 || bd == 16)) ||
                       (ct == 3 && (bd == 1 || bd == 2 || bd == 4 || bd == 8)) ||
                       ((ct == 2 || ct == 4 || ct == 6) && (bd == 8 || bd == 16));
    if (!bd_ok) { err = "PNG: invalid bit depth " + std::to_string(bd); return false; }
    if (w == 0 || h == 0 || w > (1u << 24) || h > (1u << 24) || uint64_t(w) * h > (uint64_t(1) << 30)) {
        err = "PNG: invalid size"; return false;
    }
    if (ct == 3 && (plte.empty() || plte.size() % 3)) { err = "PNG: missing or malformed palette"; return false; }
    if (interlace > 1) { err = "PNG: unknown interlace method"; return false; }
    const int bpp = std::max(1, ch * bd / 8);
    struct Pass { int x0, y0, dx, dy; };
    const Pass adam7[7] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4}, {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
    const Pass whole[1] = {{0, 0, 1, 1}};
    const Pass* passes = interlace ? adam7 : whole;
    const int npass = interlace ? 7 : 1;
    size_t expect = 0;
    for (int k = 0; k < npass; ++k) {
        if (passes[k].x0 >= static_cast<int>(w) || passes[k].y0 >= static_cast<int>(h)) continue;
        const uint32_t pw = (w - passes[k].x0 + passes[k].dx - 1) / passes[k].dx;
        const uint32_t ph = (h - passes[k].y0 + passes[k].dy - 1) / passes[k].dy;
        if (pw == 0 || ph == 0) continue;
        expect += static_cast<size_t>(ph) * (1 + (static_cast<size_t>(pw) * ch * bd + 7) / 8);
    }
    std::vector<uint8_t> raw;
    if (!inflate_exact(idat, raw, expect, err)) return false;
    out.width = static_cast<int>(w);
    out.height = static_cast<int>(h);
    out.rgba.assign(static_cast<size_t>(w) * h * 4, 255);
    int key[3] = {-1, -1, -1};   // tRNS keys of grey / RGB images
    if (!trns.empty() && (ct == 0 || ct == 2)) {
        const size_t need = ct == 0 ? 2 : 6;
        if (trns.size() >= need)
            for (int c = 0; c < (ct == 0 ? 1 : 3); ++c) key[c] = be16(trns.data() + 2 * c) & ((1 << bd) - 1);
    }
    const int gray_scale = bd == 1 ? 255 : bd == 2 ? 85 : bd == 4 ? 17 : 1;
    const uint8_t* src = raw.data();
    std::vector<uint8_t> rows;
    for (int k = 0; k < npass; ++k) {
        const Pass& ps = passes[k];
        if (ps.x0 >= static_cast<int>(w) || ps.y0 >= static_cast<int>(h)) continue;
        const uint32_t pw = (w - ps.x0 + ps.dx - 1) / ps.dx;
        const uint32_t ph = (h - ps.y0 + ps.dy - 1) / ps.dy;
        if (pw == 0 || ph == 0) continue;
        const size_t rowbytes = (static_cast<size_t>(pw) * ch * bd + 7) / 8;
        rows.resize(rowbytes * ph);
        if (!unfilter(src, static_cast<int>(ph), rowbytes, bpp, rows.data(), err)) return false;
        src += ph * (1 + rowbytes);
        for (uint32_t j = 0; j < ph; ++j) {
            const uint8_t* r = rows.data() + static_cast<size_t>(j) * rowbytes;
            const uint32_t y = ps.y0 + j * ps.dy;
            for (uint32_t i = 0; i < pw; ++i) {
                const uint32_t x = ps.x0 + i * ps.dx;
                int s[4] = {0, 0, 0, 0};
                for (int c = 0; c < ch; ++c) {
                    const size_t idx = static_cast<size_t>(i) * ch + c;
                    if (bd == 16) s[c] = (r[2 * idx] << 8) | r[2 * idx + 1];
                    else if (bd == 8) s[c] = r[idx];
                    else {
                        const size_t bit = idx * bd;
                        s[c] = (r[bit >> 3] >> (8 - bd - static_cast<int>(bit & 7))) & ((1 << bd) - 1);
                    }
                }
                auto to8 = [&](int v) { return static_cast<uint8_t>(bd == 16 ? (v >> 8) : bd == 8 ? v : v * gray_scale); };
                uint8_t* px = out.rgba.data() + (static_cast<size_t>(y) * w + x) * 4;
                switch (ct) {
                    case 0:
                        px[0] = px[1] = px[2] = to8(s[0]);
                        px[3] = s[0] == key[0] ? 0 : 255;
                        break;
                    case 2:
                        px[0] = to8(s[0]); px[1] = to8(s[1]); px[2] = to8(s[2]);
                        px[3] = (s[0] == key[0] && s[1] == key[1] && s[2] == key[2]) ? 0 : 255;
                        break;
                    case 3: {
                        const size_t e = static_cast<size_t>(s[0]);
                        if (3 * e + 2 < plte.size()) { px[0] = plte[3 * e]; px[1] = plte[3 * e + 1]; px[2] = plte[3 * e + 2]; }
                        else { px[0] = px[1] = px[2] = 0; }
                        px[3] = e < trns.size() ? trns[e] : 255;
                        break;
                    }
                    case 4:
                        px[0] = px[1] = px[2] = to8(s[0]);
                        px[3] = to8(s[1]);
                        break;
                    default:
                        px[0] = to8(s[0]); px[1] = to8(s[1]); px[2] = to8(s[2]); px[3] = to8(s[3]);
                        break;
                }
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// JPEG
// ---------------------------------------------------------------------------
namespace {

const uint8_t kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                             12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                             35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                             58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

struct Huff {
    bool present = false;
    int maxcode[18];
    int valptr[17];
    int mincode[17];
    uint8_t vals[256];
};

// Canonical code assignment (T.81 Annex C) and the decoding tables of F.2.2.3.
bool build_huff(const uint8_t* bits, const uint8_t* vals, int nvals, Huff& h) {
    int code = 0, k = 0;
    for (int l = 1; l <= 16; ++l) {
        h.valptr[l] = k;
        h.mincode[l] = code;
        code += bits[l - 1];
        k += bits[l - 1];
        h.maxcode[l] = bits[l - 1] ? code - 1 : -1;
        if (code > (1 << l)) return false;
        code <<= 1;
    }
    h.maxcode[17] = 0x7fffffff;
    if (k != nvals || k > 256) return false;
    std::memcpy(h.vals, vals, static_cast<size_t>(k));
    h.present = true;
    return true;
}

struct Bits {
    const uint8_t* p;
    const uint8_t* end;
    uint32_t acc = 0;
    int n = 0;
    bool at_marker = false;   // entropy-coded data ended at a marker (not consumed)

    int byte() {
        if (at_marker || p >= end) { at_marker = true; return 0; }
        const uint8_t b = *p;
        if (b == 0xFF) {
            if (p + 1 < end && p[1] == 0x00) { p += 2; return 0xFF; }
            at_marker = true;
            return 0;
        }
        ++p;
        return b;
    }
    int bit() {
        if (n == 0) { acc = static_cast<uint32_t>(byte()); n = 8; }
        --n;
        return static_cast<int>((acc >> n) & 1u);
    }
    int get(int s) {
        int v = 0;
        for (int i = 0; i < s; ++i) v = (v << 1) | bit();
        return v;
    }
    void reset() { n = 0; acc = 0; }
};

int decode_huff(Bits& b, const Huff& h) {
    int code = b.bit();
    int l = 1;
    while (code > h.maxcode[l]) {
        code = (code << 1) | b.bit();
        if (++l > 16) return -1;
    }
    return h.vals[h.valptr[l] + code - h.mincode[l]];
}

int extend(int v, int s) { return s == 0 ? 0 : (v < (1 << (s - 1)) ? v - (1 << s) + 1 : v); }

struct Comp {
    int id = 0, hs = 1, vs = 1, tq = 0;
    int td = 0, ta = 0;
    int pred = 0;
    int bw = 0, bh = 0;            // blocks per row / column in the plane (MCU padded)
    int cw = 0, ch = 0;            // component samples (unpadded)
    std::vector<uint8_t> plane;    // bw*8 x bh*8
};

struct IdctTable {
    double c[8][8];   // c[x][u] = s(u) cos((2x + 1) u pi / 16), s(0) = sqrt(1/8), s(u) = 1/2
    IdctTable() {
        const double pi = 3.14159265358979323846;
        for (int x = 0; x < 8; ++x)
            for (int u = 0; u < 8; ++u)
                c[x][u] = (u == 0 ? std::sqrt(0.125) : 0.5) * std::cos((2 * x + 1) * u * pi / 16.0);
    }
};

void idct_block(const int* coef, uint8_t* dst, int stride) {
    static const IdctTable T;
    double tmp[8][8];
    for (int v = 0; v < 8; ++v)
        for (int x = 0; x < 8; ++x) {
            double s = 0.0;
            for (int u = 0; u < 8; ++u) s += T.c[x][u] * coef[v * 8 + u];
            tmp[v][x] = s;
        }
    for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) {
            double s = 0.0;
            for (int v = 0; v < 8; ++v) s += T.c[y][v] * tmp[v][x];
            const long r = std::lround(s + 128.0);
            dst[y * stride + x] = static_cast<uint8_t>(std::min(255L, std::max(0L, r)));
        }
}

// Triangle-filter upsampling by 2 along one axis of a line of n samples
// (outputs scaled by 4).
void up2_line(const int* in, int n, int* out) {
    for (int i = 0; i < n; ++i) {
        const int l = in[std::max(i - 1, 0)], r = in[std::min(i + 1, n - 1)];
        out[2 * i] = 3 * in[i] + l;
        out[2 * i + 1] = 3 * in[i] + r;
    }
}

}  // namespace

bool decode_jpeg(const uint8_t* p, size_t n, DecodedImage& out, std::string& err) {
    if (n < 4 || p[0] != 0xFF || p[1] != 0xD8) { err = "JPEG: missing SOI"; return false; }
    Huff dc[4], ac[4];
    uint16_t qt[4][64];
    bool qt_present[4] = {false, false, false, false};
    std::vector<Comp> comps;
    int W = 0, H = 0, hmax = 1, vmax = 1, mcux = 0, mcuy = 0;
    int restart = 0;
    bool frame = false, adobe = false;
    int adobe_transform = -1;
    size_t o = 2;
    for (;;) {
        while (o < n && p[o] != 0xFF) ++o;          // tolerate garbage between segments
        while (o < n && p[o] == 0xFF) ++o;          // fill bytes
        if (o >= n) { err = "JPEG: missing EOI"; return false; }
        const uint8_t m = p[o++];
        if (m == 0xD9) break;                       // EOI
        if (m >= 0xD0 && m <= 0xD7) continue;       // stray RST
        if (o + 2 > n) { err = "JPEG: truncated segment"; return false; }
        const size_t len = be16(p + o);
        if (len < 2 || o + len > n) { err = "JPEG: truncated segment"; return false; }
        const uint8_t* d = p + o + 2;
        const size_t dl = len - 2;
        switch (m) {
            case 0xC0: case 0xC1: {
                if (dl < 6 || d[0] != 8) { err = "JPEG: only 8-bit precision is supported"; return false; }
                H = be16(d + 1);
                W = be16(d + 3);
                const int nc = d[5];
                if (W <= 0 || H <= 0) { err = "JPEG: invalid size (DNL not supported)"; return false; }
                if (nc != 1 && nc != 3) { err = "JPEG: " + std::to_string(nc) + " components (only 1 or 3)"; return false; }
                if (dl < 6 + 3 * static_cast<size_t>(nc)) { err = "JPEG: truncated frame header"; return false; }
                comps.assign(nc, Comp());
                for (int c = 0; c < nc; ++c) {
                    comps[c].id = d[6 + 3 * c];
                    comps[c].hs = d[7 + 3 * c] >> 4;
                    comps[c].vs = d[7 + 3 * c] & 15;
                    comps[c].tq = d[8 + 3 * c];
                    if (comps[c].hs < 1 || comps[c].hs > 4 || comps[c].vs < 1 || comps[c].vs > 4 || comps[c].tq > 3) {
                        err = "JPEG: invalid component parameters"; return false;
                    }
                    hmax = std::max(hmax, comps[c].hs);
                    vmax = std::max(vmax, comps[c].vs);
                }
                mcux = (W + 8 * hmax - 1) / (8 * hmax);
                mcuy = (H + 8 * vmax - 1) / (8 * vmax);
                for (Comp& c : comps) {
                    if (hmax % c.hs || vmax % c.vs) { err = "JPEG: non-integer sampling ratio"; return false; }
                    c.bw = mcux * c.hs;
                    c.bh = mcuy * c.vs;
                    c.cw = (W * c.hs + hmax - 1) / hmax;
                    c.ch = (H * c.vs + vmax - 1) / vmax;
                    c.plane.assign(static_cast<size_t>(c.bw) * 8 * c.bh * 8, 0);
                }
                frame = true;
                break;
            }
            case 0xC2: case 0xC6: case 0xCA: case 0xCE:
                err = "JPEG: progressive files are not supported"; return false;
            case 0xC3: case 0xC5: case 0xC7: case 0xC9: case 0xCB: case 0xCD: case 0xCF:
                err = "JPEG: lossless, hierarchical or arithmetic-coded files are not supported"; return false;
            case 0xC4: {
                size_t k = 0;
                while (k + 17 <= dl) {
                    const int tc = d[k] >> 4, th = d[k] & 15;
                    if (tc > 1 || th > 3) { err = "JPEG: bad Huffman table id"; return false; }
                    int total = 0;
                    for (int i = 0; i < 16; ++i) total += d[k + 1 + i];
                    if (k + 17 + static_cast<size_t>(total) > dl) { err = "JPEG: truncated Huffman table"; return false; }
                    if (!build_huff(d + k + 1, d + k + 17, total, tc ? ac[th] : dc[th])) {
                        err = "JPEG: malformed Huffman table"; return false;
                    }
                    k += 17 + static_cast<size_t>(total);
                }
                break;
            }
            case 0xDB: {
                size_t k = 0;
                while (k < dl) {
                    const int pq = d[k] >> 4, tq = d[k] & 15;
                    if (tq > 3 || pq > 1 || k + 1 + (pq ? 128u : 64u) > dl) { err = "JPEG: bad quantisation table"; return false; }
                    for (int i = 0; i < 64; ++i)
                        qt[tq][i] = pq ? be16(d + k + 1 + 2 * i) : d[k + 1 + i];
                    qt_present[tq] = true;
                    k += 1 + (pq ? 128 : 64);
                }
                break;
            }
            case 0xDD:
                if (dl < 2) { err = "JPEG: bad DRI"; return false; }
                restart = be16(d);
                break;
            case 0xEE:
                if (dl >= 12 && !std::memcmp(d, "Adobe", 5)) { adobe = true; adobe_transform = d[11]; }
                break;
            case 0xDA: {
                if (!frame) { err = "JPEG: scan before frame header"; return false; }
                const int ns = dl ? d[0] : 0;
                if (ns < 1 || ns > 4 || dl < 1 + 2 * static_cast<size_t>(ns) + 3) { err = "JPEG: bad scan header"; return false; }
                std::vector<Comp*> sc;
                for (int i = 0; i < ns; ++i) {
                    Comp* c = nullptr;
                    for (Comp& x : comps) if (x.id == d[1 + 2 * i]) c = &x;
                    if (!c) { err = "JPEG: scan names an unknown component"; return false; }
                    c->td = d[2 + 2 * i] >> 4;
                    c->ta = d[2 + 2 * i] & 15;
                    if (c->td > 3 || c->ta > 3 || !dc[c->td].present || !ac[c->ta].present || !qt_present[c->tq]) {
                        err = "JPEG: scan uses a missing table"; return false;
                    }
                    c->pred = 0;
                    sc.push_back(c);
                }
                Bits b{p + o + len, p + n};
                int coef[64];
                auto block = [&](Comp& c, int bx, int by) -> bool {
                    std::fill(coef, coef + 64, 0);
                    const int t = decode_huff(b, dc[c.td]);
                    if (t < 0 || t > 11) return false;
                    c.pred += extend(b.get(t), t);
                    coef[0] = c.pred * qt[c.tq][0];
                    for (int k = 1; k < 64;) {
                        const int rs = decode_huff(b, ac[c.ta]);
                        if (rs < 0) return false;
                        const int r = rs >> 4, s = rs & 15;
                        if (s == 0) {
                            if (r != 15) break;
                            k += 16;
                            continue;
                        }
                        k += r;
                        if (k > 63) return false;
                        coef[kZigzag[k]] = extend(b.get(s), s) * qt[c.tq][k];
                        ++k;
                    }
                    const int stride = c.bw * 8;
                    idct_block(coef, c.plane.data() + static_cast<size_t>(by) * 8 * stride + static_cast<size_t>(bx) * 8, stride);
                    return true;
                };
                // MCUs of this scan: a single component's scan walks its own blocks
                int units_x, units_y;
                if (ns == 1) {
                    units_x = (sc[0]->cw + 7) / 8;
                    units_y = (sc[0]->ch + 7) / 8;
                } else {
                    units_x = mcux;
                    units_y = mcuy;
                }
                const long total = static_cast<long>(units_x) * units_y;
                for (long u = 0; u < total; ++u) {
                    if (restart && u > 0 && u % restart == 0) {
                        // expect RSTn: drop the partial byte, step over the marker, reset predictors
                        b.reset();
                        while (b.p + 1 < b.end && !(b.p[0] == 0xFF && b.p[1] >= 0xD0 && b.p[1] <= 0xD7)) ++b.p;
                        if (b.p + 1 < b.end) b.p += 2;
                        b.at_marker = false;
                        for (Comp* c : sc) c->pred = 0;
                    }
                    const int ux = static_cast<int>(u % units_x), uy = static_cast<int>(u / units_x);
                    if (ns == 1) {
                        if (!block(*sc[0], ux, uy)) { err = "JPEG: corrupt entropy-coded data"; return false; }
                    } else {
                        for (Comp* c : sc)
                            for (int v = 0; v < c->vs; ++v)
                                for (int h = 0; h < c->hs; ++h)
                                    if (!block(*c, ux * c->hs + h, uy * c->vs + v)) {
                                        err = "JPEG: corrupt entropy-coded data"; return false;
                                    }
                    }
                }
                // continue at the marker that ends the entropy-coded segment
                const uint8_t* q = b.p;
                while (q + 1 < p + n && !(q[0] == 0xFF && q[1] != 0x00 && !(q[1] >= 0xD0 && q[1] <= 0xD7))) ++q;
                o = static_cast<size_t>(q - p);
                continue;
            }
            default:
                break;   // APPn, COM and other segments are skipped
        }
        o += len;
    }
    if (!frame || comps.empty()) { err = "JPEG: no frame"; return false; }
    out.width = W;
    out.height = H;
    out.rgba.assign(static_cast<size_t>(W) * H * 4, 255);
    // full-resolution planes (scaled by 16 where upsampled by the triangle filter)
    std::vector<std::vector<int>> full(comps.size());
    std::vector<int> scale(comps.size(), 1);
    for (size_t k = 0; k < comps.size(); ++k) {
        const Comp& c = comps[k];
        const int fx = hmax / c.hs, fy = vmax / c.vs;
        const int stride = c.bw * 8;
        std::vector<int>& f = full[k];
        f.assign(static_cast<size_t>(W) * H, 0);
        if (fx == 1 && fy == 1) {
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x) f[static_cast<size_t>(y) * W + x] = c.plane[static_cast<size_t>(y) * stride + x];
        } else if ((fx == 1 || fx == 2) && (fy == 1 || fy == 2)) {
            const int cw = c.cw, chh = c.ch;
            std::vector<int> rows(static_cast<size_t>(cw) * chh * fy);
            std::vector<int> col(chh), upc(2 * chh);
            for (int x = 0; x < cw; ++x) {
                for (int y = 0; y < chh; ++y) col[y] = c.plane[static_cast<size_t>(y) * stride + x];
                if (fy == 2) up2_line(col.data(), chh, upc.data());
                for (int y = 0; y < chh * fy; ++y) rows[static_cast<size_t>(y) * cw + x] = fy == 2 ? upc[y] : 4 * col[y];
            }
            const int rh = chh * fy;
            std::vector<int> line(cw), up(2 * cw);
            for (int y = 0; y < std::min(rh, H); ++y) {
                for (int x = 0; x < cw; ++x) line[x] = rows[static_cast<size_t>(y) * cw + x];
                if (fx == 2) up2_line(line.data(), cw, up.data());
                for (int x = 0; x < W; ++x)
                    f[static_cast<size_t>(y) * W + x] = fx == 2 ? up[std::min(x, 2 * cw - 1)] : 4 * line[std::min(x, cw - 1)];
            }
            scale[k] = 16;
        } else {
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x)
                    f[static_cast<size_t>(y) * W + x] = c.plane[static_cast<size_t>(y / fy) * stride + x / fx];
        }
    }
    auto sample = [&](size_t k, size_t i) -> double {
        return scale[k] == 1 ? static_cast<double>(full[k][i]) : std::floor((full[k][i] + 8) / 16.0);
    };
    auto clamp8 = [](double v) { return static_cast<uint8_t>(std::min(255.0, std::max(0.0, std::floor(v + 0.5)))); };
    const bool rgb = comps.size() == 3 &&
                     ((adobe && adobe_transform == 0) || (comps[0].id == 'R' && comps[1].id == 'G' && comps[2].id == 'B'));
    for (size_t i = 0; i < static_cast<size_t>(W) * H; ++i) {
        uint8_t* px = out.rgba.data() + 4 * i;
        if (comps.size() == 1) {
            px[0] = px[1] = px[2] = clamp8(sample(0, i));
        } else if (rgb) {
            px[0] = clamp8(sample(0, i)); px[1] = clamp8(sample(1, i)); px[2] = clamp8(sample(2, i));
        } else {
            const double y = sample(0, i), cb = sample(1, i) - 128.0, cr = sample(2, i) - 128.0;
            px[0] = clamp8(y + 1.402 * cr);
            px[1] = clamp8(y - 0.344136 * cb - 0.714136 * cr);
            px[2] = clamp8(y + 1.772 * cb);
        }
    }
    return true;
}

bool decode_image(const uint8_t* data, size_t size, DecodedImage& out, std::string& err) {
    if (size >= 8 && data[0] == 0x89 && data[1] == 'P' && data[2] == 'N' && data[3] == 'G') return decode_png(data, size, out, err);
    if (size >= 2 && data[0] == 0xFF && data[1] == 0xD8) return decode_jpeg(data, size, out, err);
    err = "unknown image format (PNG and JPEG are supported)";
    return false;
}

}  // namespace ptb
