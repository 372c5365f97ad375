// bsdf.h -- Disney principled BSDF: material resolve, evaluation, sampling.
//
// Restates the reference's shading model so that the GPU estimator has the
// same expectation as Part_2's (parity is statistical, within the tolerances
// the tests state):
//   fetchMaterial            Part_2/src/materials/disney_bsdf.cuh:53-122
//   computeAlpha             disney_bsdf.cuh:126-131
//   evalDisneyDiffuse/Sheen  disney_bsdf.cuh:135-171
//   computeF0/LobeWeights    disney_bsdf.cuh:175-205
//   evalDisneyBsdf           disney_bsdf.cuh:209-321
//   sampleDisneyBsdf         disney_bsdf.cuh:325-410
//   GGX/Smith/Fresnel/VNDF   Part_2/src/materials/microfacet.cuh:10-113
// The tangent argument of the reference's eval/sample is never read (both
// build their frame from N alone), so it is not carried here.  Texture lookups
// (fetchMaterial's textured parameters) happen before this, in the shading
// kernels (resolve_material_textured in integrator.cu); MatEval holds the
// resolved values.
#pragma once

#include "pt_internal.h"
#include "sampler.h"

namespace ptb {

struct MatEval {
    f3    base;
    float metallic, roughness, spec_trans, ior;
    float clearcoat, cc_roughness;
    float sheen, sheen_tint, subsurface;
    float anisotropic, spec_tint, spec_factor;
    f3    spec_color;
    f3    sheen_color;
    float thickness, att_distance;
    f3    att_color;
};

PT_HD float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

PT_HD MatEval resolve_material(const pt_material& m) {
    MatEval e;
    e.base         = ld3(m.base_color);
    e.metallic     = clampf(m.metallic, 0.0f, 1.0f);
    e.roughness    = clampf(m.roughness, 0.001f, 1.0f);
    e.spec_trans   = m.spec_trans;
    e.ior          = m.ior;
    e.clearcoat    = m.clearcoat;
    e.cc_roughness = clampf(m.clearcoat_roughness, 0.001f, 1.0f);
    e.sheen        = m.sheen;
    e.sheen_tint   = m.sheen_tint;
    e.subsurface   = m.subsurface;
    e.anisotropic  = m.anisotropic;
    e.spec_tint    = m.specular_tint;
    e.spec_factor  = m.specular_factor;
    e.spec_color   = mk(m.specular_color_r, m.specular_color_g, m.specular_color_b);
    e.sheen_color  = mk(m.sheen_color_r, m.sheen_color_g, m.sheen_color_b);
    e.thickness    = m.thickness_factor;
    e.att_distance = m.attenuation_distance;
    e.att_color    = mk(m.att_color_r, m.att_color_g, m.att_color_b);
    return e;
}

PT_HD bool material_emits(const pt_material& m) {
    return m.emissive_strength > 0.0f &&
           (m.emissive[0] > 0.0f || m.emissive[1] > 0.0f || m.emissive[2] > 0.0f);
}
PT_HD f3 material_emission(const pt_material& m) { return ld3(m.emissive) * m.emissive_strength; }

// ---- microfacet pieces ----
PT_HD float ggx_d(float noh, float a) {
    const float a2 = a * a;
    const float d = noh * noh * (a2 - 1.0f) + 1.0f;
    return a2 / (kPi * d * d + 1e-7f);
}
PT_HD float ggx_d_aniso(float noh, float hx, float hy, float ax, float ay) {
    const float sx = hx / ax, sy = hy / ay;
    const float d = sx * sx + sy * sy + noh * noh;
    return 1.0f / (kPi * ax * ay * d * d + 1e-7f);
}
PT_HD float smith_g1(float nov, float a) {
    const float a2 = a * a;
    return 2.0f * nov / (nov + sqrtf(a2 + (1.0f - a2) * nov * nov) + 1e-7f);
}
PT_HD float smith_g2(float nol, float nov, float a) {
    const float a2 = a * a;
    const float gv = nol * sqrtf(a2 + (1.0f - a2) * nov * nov);
    const float gl = nov * sqrtf(a2 + (1.0f - a2) * nol * nol);
    return 2.0f * nol * nov / (gv + gl + 1e-7f);
}
PT_HD float schlick_weight(float c) {
    const float t = clampf(1.0f - c, 0.0f, 1.0f);
    const float t2 = t * t;
    return t2 * t2 * t;
}
PT_HD float schlick(float c, float f0) { return f0 + (1.0f - f0) * schlick_weight(c); }
PT_HD f3 schlick3(float c, f3 f0) { return f0 + (mk(1.0f) - f0) * schlick_weight(c); }
PT_HD float fresnel_dielectric(float cos_i, float eta) {
    const float sin2t = eta * eta * (1.0f - cos_i * cos_i);
    if (sin2t >= 1.0f) return 1.0f;
    const float cos_t = sqrtf(fmaxf(0.0f, 1.0f - sin2t));
    const float ci = fabsf(cos_i);
    const float rs = (ci - eta * cos_t) / (ci + eta * cos_t + 1e-7f);
    const float rp = (eta * ci - cos_t) / (eta * ci + cos_t + 1e-7f);
    return 0.5f * (rs * rs + rp * rp);
}
// Visible-normal sampling of an (anisotropic) GGX lobe, Heitz 2018.
PT_HD f3 sample_vndf(f3 wo, float ax, float ay, float u1, float u2) {
    f3 wh = normalize(mk(ax * wo.x, ay * wo.y, wo.z));
    if (wh.z < 0.0f) wh = -wh;
    const f3 t1v = (wh.z < 0.9999f) ? normalize(cross(mk(0.0f, 0.0f, 1.0f), wh)) : mk(1.0f, 0.0f, 0.0f);
    const f3 t2v = cross(wh, t1v);
    const float r = sqrtf(u1);
    const float phi = kTwoPi * u2;
    const float p1 = r * cosf(phi);
    float p2 = r * sinf(phi);
    const float s = 0.5f * (1.0f + wh.z);
    p2 = (1.0f - s) * sqrtf(fmaxf(0.0f, 1.0f - p1 * p1)) + s * p2;
    const f3 nh = p1 * t1v + p2 * t2v + sqrtf(fmaxf(0.0f, 1.0f - p1 * p1 - p2 * p2)) * wh;
    return normalize(mk(ax * nh.x, ay * nh.y, fmaxf(0.0f, nh.z)));
}
PT_HD float pdf_vndf(f3 wo, f3 h, float ax, float ay) {
    const float nov = fmaxf(wo.z, 1e-5f);
    const float noh = fmaxf(h.z, 0.0f);
    const float voh = fmaxf(dot(wo, h), 0.0f);
    return ggx_d_aniso(noh, h.x, h.y, ax, ay) * smith_g1(nov, sqrtf(ax * ay)) * voh / (nov + 1e-7f);
}
PT_HD bool refract_dir(f3 wi, f3 n, float eta, f3& wt) {
    const float ci = dot(wi, n);
    const float s2i = fmaxf(0.0f, 1.0f - ci * ci);
    const float s2t = eta * eta * s2i;
    if (s2t >= 1.0f) return false;
    const float ct = sqrtf(1.0f - s2t);
    wt = eta * (-wi) + (eta * ci - ct) * n;
    return true;
}

// ---- Disney lobes ----
PT_HD void aniso_alpha(float roughness, float anisotropic, float& ax, float& ay) {
    const float aspect = sqrtf(1.0f - 0.9f * anisotropic);
    const float a = roughness * roughness;
    ax = fmaxf(a / aspect, 0.001f);
    ay = fmaxf(a * aspect, 0.001f);
}
PT_HD f3 tint_of(f3 base) {
    const float lum = luminance(base);
    return lum > 0.0f ? base / lum : mk(1.0f);
}
PT_HD f3 disney_diffuse(const MatEval& m, float nol, float nov, float hol) {
    const float fd90 = 0.5f + 2.0f * hol * hol * m.roughness;
    const float fl = 1.0f + (fd90 - 1.0f) * powf(1.0f - nol, 5.0f);
    const float fv = 1.0f + (fd90 - 1.0f) * powf(1.0f - nov, 5.0f);
    f3 d = m.base * (kInvPi * fl * fv);
    if (m.subsurface > 0.0f) {
        const float fss90 = hol * hol * m.roughness;
        const float sl = 1.0f + (fss90 - 1.0f) * powf(1.0f - nol, 5.0f);
        const float sv = 1.0f + (fss90 - 1.0f) * powf(1.0f - nov, 5.0f);
        const float ss = 1.25f * (sl * sv * (1.0f / (nol + nov + 1e-5f) - 0.5f) + 0.5f);
        d = (1.0f - m.subsurface) * d + m.subsurface * (m.base * (kInvPi * ss));
    }
    return d;
}
PT_HD f3 disney_sheen(const MatEval& m, float hol) {
    if (m.sheen <= 0.0f) return mk(0.0f);
    const f3 c = ((1.0f - m.sheen_tint) * mk(1.0f) + m.sheen_tint * tint_of(m.base)) * m.sheen_color;
    return m.sheen * c * powf(1.0f - hol, 5.0f);
}
PT_HD f3 disney_f0(const MatEval& m) {
    const float eta = m.ior;
    const float r0 = ((eta - 1.0f) * (eta - 1.0f)) / ((eta + 1.0f) * (eta + 1.0f));
    f3 spec = r0 * ((1.0f - m.spec_tint) * mk(1.0f) + m.spec_tint * tint_of(m.base));
    spec = spec * m.spec_factor * m.spec_color;
    return (1.0f - m.metallic) * spec + m.metallic * m.base;
}
struct LobeWeights { float diff, spec, cc, trans, sheen; };
PT_HD LobeWeights lobe_weights(const MatEval& m) {
    const float wd = (1.0f - m.metallic) * (1.0f - m.spec_trans);
    const float ws = 1.0f;
    const float wt = (1.0f - m.metallic) * m.spec_trans;
    const float wc = 0.25f * m.clearcoat;
    const float wsh = (1.0f - m.metallic) * m.sheen * 0.1f;
    const float total = wd + ws + wc + wt + wsh;
    LobeWeights w;
    if (total <= 0.0f) { w.diff = w.spec = w.cc = w.trans = w.sheen = 0.0f; return w; }
    const float inv = 1.0f / total;
    w.diff = wd * inv; w.spec = ws * inv; w.cc = wc * inv; w.trans = wt * inv; w.sheen = wsh * inv;
    return w;
}

struct BsdfEval { f3 f; float pdf; };

// f * |N.L| and the lobe-mixture pdf for (wo, wi).
PT_HD BsdfEval disney_eval(const MatEval& m, f3 wo, f3 wi, f3 n, bool entering) {
    BsdfEval r; r.f = mk(0.0f); r.pdf = 0.0f;
    const float nol = dot(n, wi);
    const float nov = dot(n, wo);
    const bool refl = nol > 0.0f;
    if (!refl && m.spec_trans <= 0.0f) return r;
    if (!refl) {
        const float anol = fabsf(nol), anov = fabsf(nov);
        if (anol < 1e-5f || anov < 1e-5f) return r;
        const float eta = entering ? (1.0f / m.ior) : m.ior;
        const f3 ht = -normalize(wo * eta + wi);
        const float hov = fabsf(dot(ht, wo));
        float ax, ay; aniso_alpha(m.roughness, m.anisotropic, ax, ay);
        const Frame fr = make_frame(n);
        const f3 hl = to_local(fr, ht);
        const float D = ggx_d_aniso(fabsf(hl.z), hl.x, hl.y, ax, ay);
        const float G = smith_g2(anol, anov, sqrtf(ax * ay));
        const float F = fresnel_dielectric(hov, eta);
        const float sd = dot(wo, ht) * eta + dot(wi, ht);
        const float factor = fabsf(dot(wo, ht)) * fabsf(dot(wi, ht)) / (anov * anol * sd * sd + 1e-7f);
        const float tw = (1.0f - m.metallic) * m.spec_trans;
        r.f = m.base * tw * D * G * (1.0f - F) * factor;
        const LobeWeights w = lobe_weights(m);
        const float jac = eta * eta * fabsf(dot(wi, ht)) / (sd * sd + 1e-7f);
        const float tpdf = D * smith_g1(anov, sqrtf(ax * ay)) * hov / (anov + 1e-7f) * jac;
        r.pdf = w.trans * tpdf;
        return r;
    }
    if (nol < 1e-5f || nov < 1e-5f) return r;
    const f3 h = normalize(wo + wi);
    const float noh = fmaxf(dot(n, h), 0.0f);
    const float hol = fmaxf(dot(h, wi), 0.0f);
    const Frame fr = make_frame(n);
    const f3 hl = to_local(fr, h);
    float ax, ay; aniso_alpha(m.roughness, m.anisotropic, ax, ay);
    const LobeWeights w = lobe_weights(m);
    f3 ft = mk(0.0f);
    float pt = 0.0f;
    const float dw = (1.0f - m.metallic) * (1.0f - m.spec_trans);
    if (dw > 0.0f) {
        ft += dw * disney_diffuse(m, nol, nov, hol);
        pt += w.diff * (nol * kInvPi);
    }
    if (m.sheen > 0.0f && m.metallic < 1.0f) {
        ft += (1.0f - m.metallic) * disney_sheen(m, hol);
        pt += w.sheen * (nol * kInvPi);
    }
    {
        const float D = ggx_d_aniso(noh, hl.x, hl.y, ax, ay);
        const float G = smith_g2(nol, nov, sqrtf(ax * ay));
        const f3 F = schlick3(hol, disney_f0(m));
        ft += D * G * F / (4.0f * nol * nov + 1e-7f);
        const f3 wol = to_local(fr, wo);
        pt += w.spec * (pdf_vndf(wol, hl, ax, ay) / (4.0f * hol + 1e-7f));
    }
    if (m.clearcoat > 0.0f) {
        const float ca = fmaxf(m.cc_roughness * m.cc_roughness, 0.001f);
        const float Dc = ggx_d(noh, ca);
        const float Gc = smith_g2(nol, nov, ca);
        const float Fc = schlick(hol, 0.04f);
        ft += mk(0.25f * m.clearcoat * Dc * Gc * Fc / (4.0f * nol * nov + 1e-7f));
        pt += w.cc * (Dc * noh / (4.0f * hol + 1e-7f));
    }
    r.f = ft * nol;
    r.pdf = pt;
    return r;
}

// Density with which disney_sample draws wi, given disney_eval's pdf of it.
// The two differ in the clearcoat lobe: it is sampled from the visible
// normals of its GGX distribution, while the eval pdf counts it with the
// distribution of normals (D noh / (4 hol)); this swaps that term.  (The
// reflections that total internal reflection gives the transmission branch
// are not counted either way.)  The plain integrator only ever uses the eval
// pdf, as the reference does; the guided mixture needs the sampler's own
// density to keep the plain integrator's expectation.
PT_HD float disney_sample_density(const MatEval& m, f3 wo, f3 wi, f3 n, float eval_pdf) {
    if (m.clearcoat <= 0.0f) return eval_pdf;
    const float nol = dot(n, wi);
    const float nov = dot(n, wo);
    if (nol < 1e-5f || nov < 1e-5f) return eval_pdf;
    const f3 h = normalize(wo + wi);
    const float noh = fmaxf(dot(n, h), 0.0f);
    const float hol = fmaxf(dot(h, wi), 0.0f);
    const Frame fr = make_frame(n);
    const float ca = fmaxf(m.cc_roughness * m.cc_roughness, 0.001f);
    const LobeWeights w = lobe_weights(m);
    const float ndf = ggx_d(noh, ca) * noh / (4.0f * hol + 1e-7f);
    const float vis = pdf_vndf(to_local(fr, wo), to_local(fr, h), ca, ca) / (4.0f * hol + 1e-7f);
    return fmaxf(eval_pdf + w.cc * (vis - ndf), 0.0f);
}

struct BsdfSample { f3 wi; f3 weight; float pdf; bool delta; bool valid; };

#if defined(__CUDA_ARCH__)
// Device code calls the BSDF through one out-of-line copy: inlined at every
// call site (NEE per light type, BSDF sampling, guided MIS) the shading kernel
// outgrows the instruction cache.
__device__ __noinline__ BsdfEval disney_eval_call(const MatEval& m, f3 wo, f3 wi, f3 n, bool entering) {
    return disney_eval(m, wo, wi, n, entering);
}
#  define PT_BSDF_EVAL disney_eval_call
#else
#  define PT_BSDF_EVAL disney_eval
#endif

// The direction of disney_sample: draws 1 + 2 dimensions, none when N.V <
// 1e-5 (the reference returns before its first draw, disney_bsdf.cuh:332-333);
// false when the sample is rejected (below the surface).
PT_HD bool disney_sample_dir(const MatEval& m, f3 wo, f3 n, PathRng& rng, int rtl, bool entering, f3& wi_out,
                             bool& delta_out) {
    const float nov = dot(n, wo);
    if (nov < 1e-5f) return false;
    const LobeWeights w = lobe_weights(m);
    const float choice = rng_next(rng);
    const Frame fr = make_frame(n);
    const f3 wol = to_local(fr, wo);
    float ax, ay; aniso_alpha(m.roughness, m.anisotropic, ax, ay);
    f3 wi;
    bool delta = false;
    float u1, u2;
    rng_pair(rng, rtl, u1, u2);
    if (choice < w.diff + w.sheen) {
        // cosine hemisphere (Malley)
        const float rr = sqrtf(u1);
        const float phi = kTwoPi * u2;
        wi = to_world(fr, mk(rr * cosf(phi), rr * sinf(phi), sqrtf(fmaxf(0.0f, 1.0f - u1))));
    } else if (choice < w.diff + w.sheen + w.spec) {
        const f3 h = to_world(fr, sample_vndf(wol, ax, ay, u1, u2));
        wi = reflect(-wo, h);
        if (dot(wi, n) <= 0.0f) return false;
        delta = m.roughness < 0.01f;
    } else if (choice < w.diff + w.sheen + w.spec + w.cc) {
        const float ca = fmaxf(m.cc_roughness * m.cc_roughness, 0.001f);
        const f3 h = to_world(fr, sample_vndf(wol, ca, ca, u1, u2));
        wi = reflect(-wo, h);
        if (dot(wi, n) <= 0.0f) return false;
    } else {
        const f3 h = to_world(fr, sample_vndf(wol, ax, ay, u1, u2));
        const float eta = entering ? (1.0f / m.ior) : m.ior;
        f3 wt;
        if (!refract_dir(wo, h, eta, wt)) {
            wi = reflect(-wo, h);
            if (dot(wi, n) <= 0.0f) return false;
        } else {
            wi = normalize(wt);
            delta = m.roughness < 0.01f;
        }
    }
    wi_out = wi;
    delta_out = delta;
    return true;
}

// One-lobe importance sample (disney_bsdf.cuh:325-410): the direction, then
// the full BSDF there.
PT_HD BsdfSample disney_sample(const MatEval& m, f3 wo, f3 n, PathRng& rng, int rtl, bool entering) {
    BsdfSample r; r.wi = mk(0.0f); r.weight = mk(0.0f); r.pdf = 0.0f; r.delta = false; r.valid = false;
    f3 wi;
    bool delta = false;
    if (!disney_sample_dir(m, wo, n, rng, rtl, entering, wi, delta)) return r;
    const BsdfEval ev = PT_BSDF_EVAL(m, wo, wi, n, entering);
    if (ev.pdf <= 0.0f) return r;
    r.wi = wi; r.pdf = ev.pdf; r.delta = delta; r.valid = true;
    if (delta) {
        if (dot(n, wi) < 0.0f) {
            r.weight = m.base;
        } else {
            const f3 h = normalize(wo + wi);
            r.weight = schlick3(fmaxf(dot(h, wi), 0.0f), disney_f0(m));
        }
    } else {
        r.weight = ev.f / (ev.pdf + 1e-7f);
    }
    return r;
}

#if defined(__CUDA_ARCH__)
__device__ __noinline__ BsdfSample disney_sample_call(const MatEval& m, f3 wo, f3 n, PathRng& rng, int rtl,
                                                      bool entering) {
    return disney_sample(m, wo, n, rng, rtl, entering);
}
#  define PT_BSDF_SAMPLE disney_sample_call
#else
#  define PT_BSDF_SAMPLE disney_sample
#endif

PT_HD float power_heuristic(float a, float b) {
    const float a2 = a * a, b2 = b * b, s = a2 + b2;
    return s > 0.0f ? a2 / s : 0.0f;
}

}  // namespace ptb
