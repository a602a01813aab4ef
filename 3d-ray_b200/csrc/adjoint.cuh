// Path-replay adjoint of the sample radiance (rt_adjoint).
//
// Each camera sample is traced twice from its Sobol indices. The primal pass
// gives the forward-form state (lp, la, pre, att0); from it and the pixel's
// loss gradient the adjoints of the resolve (the two luminance clamps and the
// per-frame sanitize) are formed. The replay runs the same shade_vertex with a
// sink whose hooks turn every factor and term of the path into parameter
// gradients:
//   - a term x added at a vertex (emission, NEE) contributes g . dx/dtheta;
//   - a factor f multiplying the weight of everything after it contributes
//     g . (S * df/dtheta / f), with S the radiance still to come in the same
//     accumulator (the primal total minus what the replay has added so far),
//     as in path replay backpropagation (Vicini et al. 2021).
// Sampling decisions are detached: sampled directions, lobe choices, light
// samples, the MIS weights and the Russian-roulette probability are held
// fixed, so f/pdf is differentiated through f only. That is exact for an
// estimator linear in its terms; the luminance clamps are not, and for the
// medium's free-flight and Russian-roulette decisions the replay adds their
// score terms (free_flight, roulette_score). The local derivatives of
// the Disney BSDF come from forward-mode dual numbers run once per parameter
// direction over the material constructor and the BSDF formulas. Geometry
// and visibility (edges) are not differentiated.
#pragma once

#include "integrator.cuh"

namespace rt {

constexpr int kAdjPerMat = 16;    // RT_ADJ_PARAMS_PER_MATERIAL
constexpr int kAdjBsdfDirs = 12;  // slots 0..11 enter the BSDF
constexpr int kAdjLocal = 128;    // per-thread accumulators when the vector fits (7 materials)

// The dual-number BSDF code is large and reached from several hooks; one
// out-of-line copy of each function keeps the kernel within the instruction
// cache (inlined at every call site it thrashed it).
#define RT_NI __device__ __noinline__

// ---------------------------------------------------------------------------
// Forward-mode dual numbers: a value and one directional derivative.
// ---------------------------------------------------------------------------
struct Df {
    float v, d;
};
RT_D Df dconst(float v) { return Df{v, 0.0f}; }
RT_D Df operator+(Df a, Df b) { return Df{a.v + b.v, a.d + b.d}; }
RT_D Df operator-(Df a, Df b) { return Df{a.v - b.v, a.d - b.d}; }
RT_D Df operator*(Df a, Df b) { return Df{a.v * b.v, a.d * b.v + a.v * b.d}; }
RT_D Df operator/(Df a, Df b) {
    float q = a.v / b.v;
    return Df{q, (a.d - q * b.d) / b.v};
}
RT_D Df operator+(Df a, float b) { return Df{a.v + b, a.d}; }
RT_D Df operator+(float a, Df b) { return Df{a + b.v, b.d}; }
RT_D Df operator-(Df a, float b) { return Df{a.v - b, a.d}; }
RT_D Df operator-(float a, Df b) { return Df{a - b.v, -b.d}; }
RT_D Df operator*(Df a, float b) { return Df{a.v * b, a.d * b}; }
RT_D Df operator*(float a, Df b) { return Df{a * b.v, a * b.d}; }
RT_D Df operator/(Df a, float b) { return Df{a.v / b, a.d / b}; }
RT_D Df operator/(float a, Df b) {
    float q = a / b.v;
    return Df{q, -q * b.d / b.v};
}
RT_D Df dsqrt(Df a) {
    float s = sqrtf(a.v);
    return Df{s, s > 0.0f ? 0.5f * a.d / s : 0.0f};
}
RT_D Df dmax(Df a, float b) { return a.v > b ? a : Df{b, 0.0f}; }   // fmaxf(a, b)
RT_D Df dclamp(Df a, float lo, float hi) { return a.v < lo ? Df{lo, 0.0f} : (a.v > hi ? Df{hi, 0.0f} : a); }
RT_D bool live(Df a) { return a.v > 0.0f || a.d != 0.0f; }
RT_D float dlog(Df a) { return a.v > 0.0f ? a.d / a.v : 0.0f; }

struct D3 {
    Df x, y, z;
};
RT_D D3 d3(V3 a) { return D3{dconst(a.x), dconst(a.y), dconst(a.z)}; }
RT_D D3 d3(Df a) { return D3{a, a, a}; }
RT_D D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
RT_D D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
RT_D D3 operator*(D3 a, D3 b) { return D3{a.x * b.x, a.y * b.y, a.z * b.z}; }
RT_D D3 operator/(D3 a, D3 b) { return D3{a.x / b.x, a.y / b.y, a.z / b.z}; }
RT_D D3 operator*(D3 a, Df b) { return D3{a.x * b, a.y * b, a.z * b}; }
RT_D D3 operator*(Df b, D3 a) { return D3{a.x * b, a.y * b, a.z * b}; }
RT_D D3 operator/(D3 a, Df b) { return D3{a.x / b, a.y / b, a.z / b}; }
RT_D D3 operator*(D3 a, float b) { return D3{a.x * b, a.y * b, a.z * b}; }
RT_D D3 operator/(D3 a, float b) { return D3{a.x / b, a.y / b, a.z / b}; }
RT_D D3 operator-(float a, D3 b) { return D3{a - b.x, a - b.y, a - b.z}; }
RT_D D3 dlerp(D3 a, D3 b, Df t) { return a * (1.0f - t) + b * t; }   // lerp(a, b, t) = a(1-t) + bt
RT_D D3 dmax3(D3 a, float b) { return D3{dmax(a.x, b), dmax(a.y, b), dmax(a.z, b)}; }
RT_D V3 dpart(D3 a) { return v3(a.x.d, a.y.d, a.z.d); }

// ---------------------------------------------------------------------------
// Material constants as duals of one raw parameter (make_material,
// DisneyBsdf.cs:237-291, 1943-1959, 1016-1049, 1104-1139). p holds the
// material's 16 raw slots; k is the seeded slot. Values are those of the
// float Material; only the derivatives are new. The lobe selection
// probabilities (pl, in LOBE_* order) are carried for the score terms of the
// few discrete events whose probability the estimator does not divide out.
// ---------------------------------------------------------------------------
struct DMat {
    D3 base, f0, sheen_col, trans_tint;
    Df roughness, sheen, clearcoat, alpha_x, alpha_y, alpha_iso, e_avg, diffuse_w, diff_all;
    Df pl[7];
};

// EnergyCompensationLut.SampleEavg (:167-175), linear in alpha between bins.
RT_D Df eavg_dual(const float* eavg, Df alpha) {
    alpha = dclamp(alpha, 0.001f, 1.0f);
    float fal = alpha.v * 32.0f - 0.5f;
    int a0 = min(max((int)floorf(fal), 0), 31);
    int a1 = min(a0 + 1, 31);
    float fr = fal - (float)a0;
    float ta = clampf(fr, 0.0f, 1.0f);
    float dta = (fr > 0.0f && fr < 1.0f) ? 32.0f * alpha.d : 0.0f;
    float e0 = __ldg(eavg + a0), e1 = __ldg(eavg + a1);
    return Df{e0 + (e1 - e0) * ta, (e1 - e0) * dta};
}

// lut_e with a dual roughness (bilinear in mu and alpha).
RT_D Df lut_e_dual(const float* e, float mu, Df alpha) {
    mu = clampf(mu, 0.0f, 1.0f);
    alpha = dclamp(alpha, 0.001f, 1.0f);
    float fmu = mu * 32.0f - 0.5f;
    float fal = alpha.v * 32.0f - 0.5f;
    int m0 = min(max((int)floorf(fmu), 0), 31);
    int a0 = min(max((int)floorf(fal), 0), 31);
    int m1 = min(m0 + 1, 31);
    int a1 = min(a0 + 1, 31);
    float tu = clampf(fmu - (float)m0, 0.0f, 1.0f);
    float fr = fal - (float)a0;
    float ta = clampf(fr, 0.0f, 1.0f);
    float dta = (fr > 0.0f && fr < 1.0f) ? 32.0f * alpha.d : 0.0f;
    float e00 = __ldg(e + m0 * 32 + a0), e01 = __ldg(e + m0 * 32 + a1);
    float e10 = __ldg(e + m1 * 32 + a0), e11 = __ldg(e + m1 * 32 + a1);
    float x0 = e00 + (e01 - e00) * ta, dx0 = (e01 - e00) * dta;
    float x1 = e10 + (e11 - e10) * ta, dx1 = (e11 - e10) * dta;
    return Df{x0 + (x1 - x0) * tu, dx0 + (dx1 - dx0) * tu};
}

RT_NI DMat dual_material(const SceneView& s, const Material& m, const float* p, int k) {
    auto seed = [&](int i) { return Df{p[i], i == k ? 1.0f : 0.0f}; };
    DMat r;
    D3 bc = D3{seed(0), seed(1), seed(2)};
    Df roughness = dclamp(seed(3), 0.0f, 1.0f);
    Df metallic = dclamp(seed(4), 0.0f, 1.0f);
    Df specular = dclamp(seed(5), 0.0f, 2.0f);
    Df spec_tint = dclamp(seed(6), 0.0f, 1.0f);
    Df sheen = dclamp(seed(7), 0.0f, 1.0f);
    Df sheen_tint = dclamp(seed(8), 0.0f, 1.0f);
    Df clearcoat = dclamp(seed(9), 0.0f, 1.0f);
    Df spec_trans = dclamp(seed(10), 0.0f, 1.0f);
    Df aniso = dclamp(seed(11), 0.0f, 1.0f);
    Df alpha = dmax(roughness * roughness, 0.001f);
    Df aspect = dsqrt(1.0f - 0.9f * aniso);
    r.alpha_x = dmax(alpha / aspect, 0.001f);
    r.alpha_y = dmax(alpha * aspect, 0.001f);
    float rr = (m.ior - 1.0f) / (m.ior + 1.0f);
    Df scaled = (rr * rr * 2.0f) * specular;
    Df lum = 0.2126f * bc.x + 0.7152f * bc.y + 0.0722f * bc.z;
    D3 tint = lum.v > 0.0f ? bc / lum : d3(v3(1.0f));
    D3 diel = dlerp(d3(scaled), tint * scaled, spec_tint);
    r.f0 = dlerp(diel, bc, metallic);
    r.sheen_col = dlerp(d3(v3(1.0f)), tint, sheen_tint);
    if (m.has_tc) {
        r.trans_tint = d3(m.trans_tint);
    } else {
        D3 pb = dmax3(bc, 0.0f);
        r.trans_tint = D3{dsqrt(pb.x), dsqrt(pb.y), dsqrt(pb.z)};
    }
    r.diff_all = (1.0f - metallic) * (1.0f - spec_trans);
    r.diffuse_w = r.diff_all * (1.0f - m.diff_trans);
    r.alpha_iso = dsqrt(r.alpha_x * r.alpha_y);
    r.e_avg = eavg_dual(s.lut_eavg, r.alpha_iso);
    // ComputeLobeWeights (:1104-1139) and LobeWeights (:1094-1101)
    Df dt_w = r.diff_all * m.diff_trans;
    Df spec_f0 = metallic.v > 0.5f ? lum : (rr * rr * 2.0f) * specular;
    Df spec_floor = 0.1f * (1.0f - spec_trans * 0.9f);
    Df spec_lerp = spec_f0 + (1.0f - spec_f0) * metallic;
    Df spec_w = spec_floor.v > spec_lerp.v ? spec_floor : spec_lerp;
    Df trans_w = (1.0f - metallic) * spec_trans;
    Df clear_w = clearcoat * 0.04f;
    Df sheen_w = sheen * 0.25f * r.diff_all;
    Df ms_w = spec_w * (1.0f - r.e_avg);
    Df sum = r.diffuse_w + spec_w + trans_w + clear_w + sheen_w + ms_w + dt_w;
    Df total = sum.v < 1e-6f ? dconst(1.0f) : sum;
    r.pl[LOBE_DIFFUSE] = r.diffuse_w / total;
    r.pl[LOBE_SPECULAR] = spec_w / total;
    r.pl[LOBE_TRANSMISSION] = trans_w / total;
    r.pl[LOBE_SHEEN] = sheen_w / total;
    r.pl[LOBE_MULTISCATTER] = ms_w / total;
    r.pl[LOBE_DIFFTRANS] = dt_w / total;
    r.pl[LOBE_CLEARCOAT] = clear_w / total;
    r.base = bc;
    r.roughness = roughness;
    r.sheen = sheen;
    r.clearcoat = clearcoat;
    return r;
}

// ---------------------------------------------------------------------------
// Dual forms of the BSDF formulas in device.cuh. Discrete gates use the float
// material except where the gated lobe is scaled by the gating value itself
// (diffuse by diffuse_w, sheen by sheen, clearcoat by clearcoat): there the
// lobe is evaluated whenever its derivative can be non-zero, which gives the
// one-sided derivative at the clamp boundary.
// ---------------------------------------------------------------------------
RT_D Df ggx_d_dual(V3 h, Df ax, Df ay) {   // Microfacet.cs:43-49
    Df hx = h.x / ax;
    Df hy = h.y / ay;
    Df d = hx * hx + hy * hy + h.z * h.z;
    Df den = kPi * ax * ay * d * d;
    return 1.0f / dmax(den, 1e-20f);
}
RT_D Df ggx_g1_dual(V3 w, Df ax, Df ay) {   // :55-69
    float c2 = w.z * w.z;
    if (c2 < 1e-14f) return dconst(1.0f / (1.0f + 1e10f));
    Df num = (ax * w.x) * (ax * w.x) + (ay * w.y) * (ay * w.y);
    Df lam = 0.5f * (-1.0f + dsqrt(1.0f + num / c2));
    return 1.0f / (1.0f + lam);
}
RT_D D3 fresnel_schlick_dual(float c, D3 f0) {
    float w = schlick_weight(c);
    return f0 + (1.0f - f0) * w;
}
RT_NI D3 multiscatter_dual(const SceneView& s, const DMat& dm, float ndv, float ndl) {   // :1906-1926
    Df e_out = lut_e_dual(s.lut_e, ndv, dm.alpha_iso);
    Df e_in = lut_e_dual(s.lut_e, ndl, dm.alpha_iso);
    Df one_m = dmax(1.0f - dm.e_avg, 1e-6f);
    D3 f_avg = dm.f0 + (1.0f - dm.f0) * (1.0f / 21.0f);
    D3 den = dmax3(1.0f - f_avg * (1.0f - dm.e_avg), 1e-6f);
    D3 f_ms = f_avg * f_avg * dm.e_avg / den;
    return f_ms * ((1.0f - e_out) * (1.0f - e_in) / one_m);
}
RT_D Df diffuse_fd_dual(const DMat& dm, float ndv, float ndl, float ldh) {
    Df fd90 = 0.5f + 2.0f * dm.roughness * ldh * ldh;
    float fi = schlick_weight(ndv), fo = schlick_weight(ndl);
    return (1.0f + (fd90 - 1.0f) * fi) * (1.0f + (fd90 - 1.0f) * fo);
}
RT_D float clearcoat_shape(const Material& m, float cndv, float cndl, float cndh, float cvdh) {
    float ca2 = m.cc_alpha * m.cc_alpha;
    float cden = cndh * cndh * (ca2 - 1.0f) + 1.0f;
    float cD = ca2 / (kPi * cden * cden);
    float cG = smith_g1(cndv, m.cc_alpha) * smith_g1(cndl, m.cc_alpha);
    float cF = m.cc_f0 + (1.0f - m.cc_f0) * schlick_weight(cvdh);
    return 0.25f * cD * cG * cF;
}

// EvaluateDirect (bsdf_eval_direct).
RT_NI D3 eval_direct_dual(const SceneView& s, const Material& m, const DMat& dm, const Surface& rec, V3 L, V3 V) {
    V3 N = rec.n;
    D3 r = d3(v3(0.0f));
    float ndl = fmaxf(dot(N, L), 0.0f);
    if (ndl <= 0.0f) return r;
    float ndv = fmaxf(dot(N, V), 0.001f);
    V3 H = normalize(L + V);
    float ndh = fmaxf(dot(N, H), 0.0f);
    float vdh = fmaxf(dot(V, H), 0.0f);
    float ldh = fmaxf(dot(L, H), 0.0f);
    if (live(dm.diffuse_w)) r = r + dm.base * diffuse_fd_dual(dm, ndv, ndl, ldh) * (dm.diffuse_w * ndl / kPi);
    if (m.alpha > kDeltaAlpha) {
        Frame fr = shading_frame(rec, m);
        V3 vl = fr.to_local(V), ll = fr.to_local(L), hl = fr.to_local(H);
        Df D = ggx_d_dual(hl, dm.alpha_x, dm.alpha_y);
        Df G = ggx_g1_dual(vl, dm.alpha_x, dm.alpha_y) * ggx_g1_dual(ll, dm.alpha_x, dm.alpha_y);
        r = r + fresnel_schlick_dual(vdh, dm.f0) * (D * G / fmaxf(4.0f * ndv, 1e-6f));
    }
    if (live(dm.clearcoat) && m.cc_alpha > kDeltaAlpha) {
        float cndv = fmaxf(dot(N, V), 0.001f);
        float cndl = dot(N, L);
        if (cndl > 0.0f) {
            float cc = clearcoat_shape(m, cndv, cndl, fmaxf(dot(N, H), 0.0f), fmaxf(dot(V, H), 0.0f));
            r = r + d3(dm.clearcoat * (cc / fmaxf(4.0f * cndv, 1e-6f)));
        }
    }
    if (live(dm.sheen) && m.diffuse_w > 0.0f) {
        float sb = sheen_brdf(ndv, ndl, ndh, m.sheen_roughness);
        r = r + dm.sheen_col * (dm.sheen * (sb * ndl));
    }
    return r + multiscatter_dual(s, dm, ndv, ndl) * (ndl / kPi);
}

// Evaluate (bsdf_eval), without the cosine.
RT_NI D3 eval_dual(const SceneView& s, const Material& m, const DMat& dm, const Surface& rec, V3 V, V3 L) {
    V3 N = rec.n;
    D3 r = d3(v3(0.0f));
    float ndl = dot(N, L);
    float ndv = dot(N, V);
    if (ndv <= 0.0f) return r;
    if (ndl <= 0.0f) {
        if (!live(dm.diff_all) || m.diff_trans <= 0.0f) return r;
        return dm.base * (dm.diff_all * (m.diff_trans / kPi));
    }
    V3 hraw = V + L;
    float hl2 = length_sq(hraw);
    if (hl2 < 1e-14f) return r;
    V3 H = hraw / sqrtf(hl2);
    float ndh = fmaxf(dot(N, H), 0.0f);
    float vdh = fmaxf(dot(V, H), 0.0f);
    float ldh = fmaxf(dot(L, H), 0.0f);
    if (live(dm.diffuse_w)) r = r + dm.base * diffuse_fd_dual(dm, ndv, ndl, ldh) * (dm.diffuse_w / kPi);
    if (live(dm.sheen) && m.diffuse_w > 0.0f) {
        float sb = sheen_brdf(ndv, ndl, ndh, m.sheen_roughness);
        r = r + dm.sheen_col * (dm.sheen * sb);
    }
    Frame fr = shading_frame(rec, m);
    V3 vl = fr.to_local(V), ll = fr.to_local(L), hl = fr.to_local(H);
    Df D = ggx_d_dual(hl, dm.alpha_x, dm.alpha_y);
    Df G = ggx_g1_dual(vl, dm.alpha_x, dm.alpha_y) * ggx_g1_dual(ll, dm.alpha_x, dm.alpha_y);
    r = r + fresnel_schlick_dual(vdh, dm.f0) * (D * G / fmaxf(4.0f * ndv * ndl, 1e-7f));
    if (live(dm.clearcoat)) {
        float cndv = dot(N, V), cndl = dot(N, L);
        if (cndv > 0.0f && cndl > 0.0f) {
            float cc = clearcoat_shape(m, cndv, cndl, fmaxf(dot(N, H), 0.0f), fmaxf(dot(V, H), 0.0f));
            r = r + d3(dm.clearcoat * (cc / fmaxf(4.0f * cndv * cndl, 1e-7f)));
        }
    }
    return r + multiscatter_dual(s, dm, ndv, ndl) * (1.0f / kPi);
}

// The attenuation formula of one lobe of ScatterInternal (bsdf_scatter) for a
// direction already drawn: delta samples of Sample and the legacy Scatter
// path. The lobe selection probability in the divisor stays detached.
RT_NI D3 lobe_att_dual(const SceneView& s, const Material& m, const DMat& dm, const Surface& rec, V3 V, V3 dir,
                       int lobe) {
    V3 N = rec.n;
    switch (lobe) {
    case LOBE_DIFFUSE: {
        float ndv = fmaxf(dot(N, V), 0.001f);
        float ndl = fmaxf(dot(N, dir), 0.001f);
        V3 hraw = V + dir;
        float hl2 = length_sq(hraw);
        V3 H = hl2 > 1e-7f ? hraw / sqrtf(hl2) : N;
        float ldh = fmaxf(dot(dir, H), 0.0f);
        return dm.base * diffuse_fd_dual(dm, ndv, ndl, ldh) * ((1.0f - m.diff_trans) / fmaxf(m.p_d, 0.1f));
    }
    case LOBE_SPECULAR: {
        Frame fr = shading_frame(rec, m);
        V3 H = normalize(V + dir);
        float vdh = fmaxf(dot(V, H), 1e-4f);
        Df g1l = ggx_g1_dual(fr.to_local(dir), dm.alpha_x, dm.alpha_y);
        return fresnel_schlick_dual(vdh, dm.f0) * g1l / fmaxf(m.p_s, 0.1f);
    }
    case LOBE_TRANSMISSION: {
        D3 a = dot(dir, N) > 0.0f ? d3(v3(1.0f)) : dm.trans_tint;
        if (m.roughness > 0.01f) {
            Frame fr = shading_frame(rec, m);
            V3 ll = fr.to_local(dir);
            ll.z = fabsf(ll.z);
            a = a * ggx_g1_dual(ll, dm.alpha_x, dm.alpha_y);
        }
        return a / fmaxf(m.p_t, 0.1f);
    }
    case LOBE_SHEEN: {
        float ndv = fmaxf(dot(N, V), 1e-4f);
        float ndl = fmaxf(dot(N, dir), 1e-4f);
        V3 hraw = V + dir;
        float hl2 = length_sq(hraw);
        V3 H = hl2 > 1e-7f ? hraw / sqrtf(hl2) : N;
        float sb = sheen_brdf(ndv, ndl, fmaxf(dot(N, H), 0.0f), m.sheen_roughness);
        return dm.sheen_col * (dm.sheen * (kPi * sb / fmaxf(m.p_sh, 0.1f)));
    }
    case LOBE_MULTISCATTER: {
        float ndv = fmaxf(dot(N, V), 1e-3f);
        float ndl = fmaxf(dot(N, dir), 1e-3f);
        return multiscatter_dual(s, dm, ndv, ndl) / fmaxf(m.p_ms, 0.05f);
    }
    case LOBE_DIFFTRANS:
        return dm.base * (m.diff_trans / fmaxf(m.p_dt, 0.05f));
    default:   // clearcoat: no differentiated parameter enters its weight
        return d3(v3(0.0f));
    }
}

// Score terms. The estimator divides most sampling probabilities out, so they
// need no derivative, except in two places where the reference's estimator
// keeps them:
//   - a lobe whose weight is divided by max(p, floor) rather than p (delta
//     lobes and the legacy Scatter path): below the floor its expected
//     contribution is p * w / floor, so the chosen lobe adds d log p;
//   - a null Sample (the reflection lobe drew a direction below the surface),
//     after which the legacy Scatter path draws again: the probability of that
//     event, p_lobe times the lobe's density of the drawn direction, adds its
//     log-derivative.
RT_D float lobe_floor(int lobe) { return (lobe == LOBE_MULTISCATTER || lobe == LOBE_DIFFTRANS) ? 0.05f : 0.1f; }

RT_NI float null_sample_score(const Material& m, const DMat& dm, const Surface& rec, V3 V, int lobe, V3 tried) {
    if (lobe < 0 || lobe > LOBE_CLEARCOAT) return 0.0f;
    float sc = dlog(dm.pl[lobe]);
    if (lobe == LOBE_SPECULAR) {   // VNDF density of the drawn L: G1(V) D(H) / (4 N.V)
        V3 hraw = V + tried;
        float hl2 = length_sq(hraw);
        if (hl2 > 1e-14f) {
            Frame fr = shading_frame(rec, m);
            V3 hl = fr.to_local(hraw / sqrtf(hl2));
            sc += dlog(ggx_g1_dual(fr.to_local(V), dm.alpha_x, dm.alpha_y)) + dlog(ggx_d_dual(hl, dm.alpha_x, dm.alpha_y));
        }
    }
    return sc;
}

// Vector-Jacobian product of clamp_lum (sanitize, then scale to luminance mx).
RT_D V3 clamp_lum_vjp(V3 cin, float mx, V3 g) {
    V3 c = sanitize(cin);
    V3 keep = v3(isfinite(cin.x) && cin.x > 0.0f ? 1.0f : 0.0f, isfinite(cin.y) && cin.y > 0.0f ? 1.0f : 0.0f,
                 isfinite(cin.z) && cin.z > 0.0f ? 1.0f : 0.0f);
    float lum = luminance(c);
    V3 r = g;
    if (lum > mx && lum > 0.0f) {
        float k = mx / lum;
        float cg = dot(c, g) / lum;
        r = k * (g - cg * v3(0.2126f, 0.7152f, 0.0722f));
    }
    return r * keep;
}

// The adjoints of the resolve (path_resolve) for one primal end state (lp,
// la, pre, att0, clamp_mode) and the sample's film gradient delta: the primal
// total A, the raw la, and the adjoints of A, la and att0 through the two
// luminance clamps and the per-frame sanitize.
struct AdjResolve {
    V3 tot_a, tot_la, g_a, g_la, g_att0;
    V3 delta;    // the sample's film gradient
    float val;   // delta . the sample's clamped radiance
};
RT_D AdjResolve adjoint_resolve(const RenderConst& rc, V3 lp, V3 la, V3 pre, V3 att0, int clamp_mode, V3 delta) {
    AdjResolve r;
    V3 A = lp, X = v3(0.0f);
    if (clamp_mode) {
        X = att0 * sanitize(la);
        A = A + pre * clamp_lum(X, rc.ind_max);
    }
    r.tot_a = A;
    r.tot_la = la;
    r.delta = delta;
    r.val = dot(delta, clamp_lum(A, rc.max_rad));
    r.g_a = clamp_lum_vjp(A, rc.max_rad, delta);
    r.g_la = v3(0.0f);
    r.g_att0 = v3(0.0f);
    if (clamp_mode) {
        V3 gx = clamp_lum_vjp(X, rc.ind_max, r.g_a * pre);
        V3 sl = sanitize(la);
        r.g_att0 = gx * sl;
        V3 pos = v3(sl.x > 0.0f ? 1.0f : 0.0f, sl.y > 0.0f ? 1.0f : 0.0f, sl.z > 0.0f ? 1.0f : 0.0f);
        r.g_la = gx * att0 * pos;
    }
    return r;
}

// What the out-of-line hooks read of the path state, passed by value: handing
// them the PathState itself by reference would take its address and move the
// whole state out of registers into local memory for the entire replay loop.
struct PathView {
    V3 lp, la, mask;
    int clamp_mode, first;
};
RT_D PathView path_view(const PathState& ps) { return PathView{ps.lp, ps.la, ps.mask, ps.clamp_mode, ps.first}; }

// Per-thread adjoint state of one replayed sample, and the replay sink.
struct AdjointSink {
    const SceneView* s;
    const float* params;   // raw parameter vector (device), 16 per material
    const unsigned* mmask; // per material: bit k = slot k is differentiated
    unsigned gmask;        // the 6 global (medium) slots
    float* loc;            // per-thread accumulators (kAdjLocal), or null
    float* acc;            // block accumulators in shared memory, or null
    double* gacc;          // global accumulators
    int medium_base;       // first global slot (medium sigma_a, sigma_s)
    int opaque;
    int any4;              // opaque shadow rays walk the four-wide records in any order (stack bound fits)
    int* err;
    V3 tot_a, tot_la;      // primal A = lp + pre * clamp(att0 * S(la)) and la
    V3 g_a, g_la, g_att0;  // their adjoints
    int abs_mat;           // material of the current interior absorption (-1: none)
    V3 delta;              // the sample's film gradient
    float val;             // delta . the sample's clamped radiance
    float max_rad, ind_max;   // the two clamps (RenderConst)
    // d log beta_c / d theta_k of the path throughput Russian roulette reads,
    // for the medium's six slots (sigma_a, then sigma_s), kept while a medium
    // slot is differentiated
    float dlb[3][6];
    RT_D void set_resolve(const AdjResolve& r) {
        tot_a = r.tot_a;
        tot_la = r.tot_la;
        g_a = r.g_a;
        g_la = r.g_la;
        g_att0 = r.g_att0;
        delta = r.delta;
        val = r.val;
    }
    // the last shadow ray
    int sh_added;
    V3 sh_x;               // the term it added
    V3 sh_tr;              // its transmittance
    int sh_n;
    int sh_mat[8];
    float sh_len[8];       // >= 0: absorption length inside sh_mat; < 0: a crossing of sh_mat's surface

    RT_D void add(int i, float v) {
        if (v == 0.0f || !isfinite(v)) return;
        if (i >= medium_base ? !((gmask >> (i - medium_base)) & 1u) : !((mmask[i >> 4] >> (i & 15)) & 1u)) return;
        if (loc) loc[i] += v;
        else if (acc) atomicAdd(acc + i, v);
        else atomicAdd(gacc + i, (double)v);
    }
    RT_D V3 gain(const PathView& ps, int to_la) const {   // adjoint of a term added now
        if (!to_la) return g_a;
        return g_la * ps.mask;
    }
    RT_D void target(const PathView& ps, V3& g, V3& S) const {   // adjoint and radiance still to come
        if (ps.clamp_mode) {
            g = g_la;
            S = tot_la - ps.la;
        } else {
            g = g_a;
            S = tot_a - ps.lp;
        }
    }
    RT_D bool medium_ok() const {
        return s->has_medium && s->sigma_t.x > 0.0f && s->sigma_t.y > 0.0f && s->sigma_t.z > 0.0f;
    }

    // The transparent walk of shadow_transmittance, recording the absorption
    // lengths and surface crossings that the gradient needs.
    template <int STACK>
    RT_D V3 walk(V3 o, V3 d, float tmin, float tmax) {
        sh_n = 0;
        Hit h;
        if (opaque) {
            if (any4) traverse4_any<STACK>(*s, o, d, tmin, tmax, h, err);
            else traverse<true, STACK>(*s, o, d, tmin, tmax, h, nullptr, err);
            return h.kind == HIT_NONE ? v3(1.0f) : v3(0.0f);
        }
        V3 thr = v3(1.0f);
        float remaining = tmax;
        V3 sigma = v3(0.0f), entry = v3(0.0f);
        int ent_mat = -1;
        bool in_med = false;
        for (int i = 0; i < 8; i++) {
            traverse<false, STACK>(*s, o, d, tmin, remaining, h, nullptr, err);
            if (h.kind == HIT_NONE) return thr;
            Surface rec = make_surface(*s, h, o, d);
            const Material& m = s->materials[rec.material];
            if (in_med) {
                float dd = length(rec.p - entry);
                thr = v3(thr.x * expf(-sigma.x * dd), thr.y * expf(-sigma.y * dd), thr.z * expf(-sigma.z * dd));
                in_med = false;
                if (sh_n < 8) {
                    sh_mat[sh_n] = ent_mat;
                    sh_len[sh_n++] = dd;
                }
                if (near_zero(thr)) return v3(0.0f);
            }
            V3 t = bsdf_shadow_transmittance(m, d, rec);
            if (near_zero(t)) return v3(0.0f);
            thr = thr * t;
            if (sh_n < 8) {
                sh_mat[sh_n] = rec.material;
                sh_len[sh_n++] = -1.0f;
            }
            if (near_zero(thr)) return v3(0.0f);
            if (rec.front && m.type == 0) {
                V3 sg = m.trans_sigma;
                if (!near_zero(sg)) {
                    in_med = true;
                    entry = rec.p;
                    sigma = sg;
                    ent_mat = rec.material;
                }
            }
            V3 on = dot(d, rec.n) >= 0.0f ? rec.n : -rec.n;
            o = offset_origin(rec.p, on);
            remaining -= rec.t + 2.0f * kEps;
            if (remaining <= tmin) return thr;
        }
        return v3(0.0f);
    }

    // Gradients shared by the surface and medium NEE terms: the emitter's
    // radiance, the medium transmittance over the light distance and the
    // shadow ray's absorption and surface crossings.
    RT_NI void nee_common(PathView ps, int li, float dist, int to_la) {
        V3 gx = gain(ps, to_la) * sh_x;
        if (is_zero(gx)) return;
        const Light& l = s->lights[li];
        if ((l.type == LIGHT_GEOM_QUAD || l.type == LIGHT_GEOM_MESH || l.type == LIGHT_GEOM_SPHERE) &&
            l.emissive_material >= 0) {
            int b = l.emissive_material * kAdjPerMat;
            if (l.emission.x > 0.0f) add(b + 0, gx.x / l.emission.x);
            if (l.emission.y > 0.0f) add(b + 1, gx.y / l.emission.y);
            if (l.emission.z > 0.0f) add(b + 2, gx.z / l.emission.z);
        }
        if (medium_ok() && dist < kInf) {
            float v[3] = {-dist * gx.x, -dist * gx.y, -dist * gx.z};
            for (int c = 0; c < 3; c++) {
                add(medium_base + c, v[c]);
                add(medium_base + 3 + c, v[c]);
            }
        }
        for (int i = 0; i < sh_n; i++) {
            int mi = sh_mat[i];
            const Material& m = s->materials[mi];
            int b = mi * kAdjPerMat;
            if (sh_len[i] >= 0.0f) {
                float L = sh_len[i];
                if (m.trans_sigma.x > 0.0f) add(b + 12, -L * gx.x);
                if (m.trans_sigma.y > 0.0f) add(b + 13, -L * gx.y);
                if (m.trans_sigma.z > 0.0f) add(b + 14, -L * gx.z);
            } else {
                const float* p = params + b;
                if (!m.has_tc) {   // trans_tint = sqrt(baseColor)
                    if (p[0] > 0.0f) add(b + 0, 0.5f * gx.x / p[0]);
                    if (p[1] > 0.0f) add(b + 1, 0.5f * gx.y / p[1]);
                    if (p[2] > 0.0f) add(b + 2, 0.5f * gx.z / p[2]);
                }
                if (m.spec_trans_raw > 0.0f) add(b + 10, (gx.x + gx.y + gx.z) / m.spec_trans_raw);
            }
        }
    }

    // ---- the hooks of shade_vertex
    template <int STACK>
    RT_D void shadow_impl(PathState& ps, V3 o, V3 d, float tmax, V3 c, int to_la) {
        V3 tr = walk<STACK>(o, d, kEps, tmax);
        sh_added = !near_zero(tr);
        if (!sh_added) return;
        sh_tr = tr;
        sh_x = c * tr;
        ps.add(sh_x, to_la);
    }
    RT_D void skipped(V3, V3, float) {}
    RT_D void interior(int mat) { abs_mat = mat; }

    // Score terms under the clamps. The clamps make the sample value a
    // nonlinear function F of its terms, each term divided by the density of
    // the decisions before it, so the derivative of E[F] holds, besides the
    // detached terms, E[dlog p_j/dtheta * B_j] for every decision j whose
    // density depends on theta, with B_j = F - sum over the terms after j of
    // dF/dterm . term - b_j and any baseline b_j that depends on the path
    // before j alone. b_j = F of the terms before j (the sample's value had
    // the path ended there) makes B_j exactly 0 when F is linear (no clamp
    // saturates), so unclamped samples gain no variance. The terms after j are
    // the replay's suffix (target), except at the first surface vertex's
    // roulette, after which every term goes to la through att0.
    RT_D float score_weight(const PathView& v, V3 pre, V3 att0, bool first_surface) const {
        V3 now = v.lp;
        if (v.clamp_mode) now = now + pre * clamp_lum(att0 * sanitize(v.la), ind_max);
        float after;
        if (first_surface) {
            after = dot(g_la, tot_la);
        } else {
            V3 g, S;
            target(v, g, S);
            after = dot(g, S);
        }
        return val - after - dot(delta, clamp_lum(now, max_rad));
    }

    // A free-flight decision of the medium: its score, and its factor's log
    // derivatives in the throughput. medium_sample draws from the channel
    // mixture (1/3) sum_c sigma_t,c exp(-sigma_t,c t) for a scattering at t,
    // (1/3) sum_c exp(-sigma_t,c t) for passing a segment of length t, and
    // puts tr_c sigma_s,c / p or tr_c / p into the throughput; sigma_t =
    // sigma_a + sigma_s.
    RT_NI void free_flight(PathView v, V3 pre, V3 att0, float t, int mode) {
        bool sc = mode == SEG_MEDIUM_SCATTER;
        V3 st = s->sigma_t, tr = medium_tr(*s, t);
        V3 dens = sc ? st * tr : tr;
        float p = (dens.x + dens.y + dens.z) / 3.0f;
        if (!(p >= 1e-20f)) return;
        float stc[3] = {st.x, st.y, st.z}, trc[3] = {tr.x, tr.y, tr.z};
        float ssc[3] = {s->sigma_s.x, s->sigma_s.y, s->sigma_s.z};
        float dl[3];   // d log p / d sigma_t,k
        for (int k = 0; k < 3; k++) dl[k] = (sc ? trc[k] * (1.0f - stc[k] * t) : -t * trc[k]) / (3.0f * p);
        float b = score_weight(v, pre, att0, false);
        if (b != 0.0f && isfinite(b))
            for (int k = 0; k < 3; k++) {
                add(medium_base + k, b * dl[k]);
                add(medium_base + 3 + k, b * dl[k]);
            }
        for (int c = 0; c < 3; c++)
            for (int k = 0; k < 3; k++) {
                float own = c == k ? -t : 0.0f;
                dlb[c][k] += own - dl[k];
                dlb[c][3 + k] += own + ((c == k && sc && ssc[c] > 0.0f) ? 1.0f / ssc[c] : 0.0f) - dl[k];
            }
    }

    // Russian roulette: a survivor was drawn against q = clamp(max_c thr_c,
    // min survival, 0.95), which moves with theta only strictly between the
    // bounds, as the largest channel of the throughput. Channels tied for the
    // largest (a grey medium keeps all three equal until a coloured surface)
    // make the max a kink: its slope is the largest of their derivatives for
    // a rising theta and the smallest for a falling one, and the central
    // derivative, which central differences measure, is the mean of the two.
    // The survivor's throughput then carries 1/q. A path the roulette ends
    // has no terms after the decision, so its score weight is 0.
    RT_NI void roulette_score(PathView v, V3 pre, V3 att0, V3 thr, float q, int first_surface) {
        float m = fmaxf(thr.x, fmaxf(thr.y, thr.z));
        if (q != m) return;
        float thc[3] = {thr.x, thr.y, thr.z};
        float lo[6], hi[6];
        int tied = 0;
        for (int c = 0; c < 3; c++) {
            if (thc[c] != m) continue;
            for (int k = 0; k < 6; k++) {
                lo[k] = tied ? fminf(lo[k], dlb[c][k]) : dlb[c][k];
                hi[k] = tied ? fmaxf(hi[k], dlb[c][k]) : dlb[c][k];
            }
            tied++;
        }
        if (!tied) return;
        float dq[6];
        for (int k = 0; k < 6; k++) dq[k] = 0.5f * (lo[k] + hi[k]);
        float b = score_weight(v, pre, att0, first_surface != 0);
        if (b != 0.0f && isfinite(b))
            for (int k = 0; k < 6; k++) add(medium_base + k, b * dq[k]);
        for (int c = 0; c < 3; c++)
            for (int k = 0; k < 6; k++) dlb[c][k] -= dq[k];
    }
    RT_D bool medium_scores() const { return (gmask & 0x3Fu) && medium_ok(); }
    RT_D void roulette(const PathState& ps, V3 thr, float q, int first_surface) {
        if (medium_scores()) roulette_score(path_view(ps), ps.pre, ps.att0, thr, q, first_surface);
    }
    RT_D void clear_log_beta() {
        for (int c = 0; c < 3; c++)
            for (int k = 0; k < 6; k++) dlb[c][k] = 0.0f;
    }

    RT_D void segment(const PathState& ps, float t, int mode) {
        V3 g, S;
        target(path_view(ps), g, S);
        V3 gs = g * S;
        if (mode != SEG_ABSORPTION && medium_scores()) free_flight(path_view(ps), ps.pre, ps.att0, t, mode);
        if (is_zero(gs)) return;
        if (mode != SEG_MEDIUM_PASS && abs_mat >= 0) {
            const Material& m = s->materials[abs_mat];
            int b = abs_mat * kAdjPerMat + 12;
            if (m.trans_sigma.x > 0.0f) add(b + 0, -t * gs.x);
            if (m.trans_sigma.y > 0.0f) add(b + 1, -t * gs.y);
            if (m.trans_sigma.z > 0.0f) add(b + 2, -t * gs.z);
        }
        if (mode != SEG_ABSORPTION && medium_ok()) {
            float gsc[3] = {gs.x, gs.y, gs.z};
            float ss[3] = {s->sigma_s.x, s->sigma_s.y, s->sigma_s.z};
            for (int c = 0; c < 3; c++) {
                add(medium_base + c, -t * gsc[c]);
                float rs = -t;
                if (mode == SEG_MEDIUM_SCATTER) rs = ss[c] > 0.0f ? 1.0f / ss[c] - t : 0.0f;
                add(medium_base + 3 + c, rs * gsc[c]);
            }
        }
    }

    RT_D void emission(const PathState& ps, int mat, V3 we, int to_la) {
        V3 g = gain(path_view(ps), to_la) * ps.w * we;
        const Material& m = s->materials[mat];
        int b = mat * kAdjPerMat;
        if (m.emission.x > 0.0f) add(b + 0, g.x / m.emission.x);
        if (m.emission.y > 0.0f) add(b + 1, g.y / m.emission.y);
        if (m.emission.z > 0.0f) add(b + 2, g.z / m.emission.z);
    }

    RT_D void nee_surface(const PathState& ps, int li, const Material& m, const Surface& rec, V3 L, V3 V,
                          float term, V3 coef, float dist, V3 tr_m, int to_la) {
        if (sh_added) nee_surface_impl(path_view(ps), li, m, rec, L, V, term, coef, dist, tr_m, to_la);
    }
    RT_NI void nee_surface_impl(PathView ps, int li, const Material& m, const Surface& rec, V3 L, V3 V,
                                float term, V3 coef, float dist, V3 tr_m, int to_la) {
        nee_common(ps, li, dist, to_la);
        // the term is coef * (f_direct * term) * tr_m * tr: differentiate f_direct
        unsigned bits = mmask[rec.material] & ((1u << kAdjBsdfDirs) - 1u);
        if (!bits) return;
        V3 w = gain(ps, to_la) * coef * tr_m * sh_tr * term;
        if (is_zero(w)) return;
        const float* p = params + rec.material * kAdjPerMat;
        for (; bits; bits &= bits - 1u) {
            int k = __ffs(bits) - 1;
            DMat dm = dual_material(*s, m, p, k);
            add(rec.material * kAdjPerMat + k, dot(w, dpart(eval_direct_dual(*s, m, dm, rec, L, V))));
        }
    }
    RT_D void nee_medium(const PathState& ps, int li, float dist, int to_la) {
        if (sh_added) nee_common(path_view(ps), li, dist, to_la);
    }

    RT_D void scatter(const PathState& ps, const Material& m, const Surface& rec, V3 V, V3 dir, int lobe, int mode,
                      float pdf, V3 att_pre, V3 att, int null_lobe, V3 null_dir) {
        if (mmask[rec.material] & ((1u << kAdjBsdfDirs) - 1u))
            scatter_impl(path_view(ps), m, rec, V, dir, lobe, mode, pdf, att_pre, att, null_lobe, null_dir);
    }
    RT_NI void scatter_impl(PathView ps, const Material& m, const Surface& rec, V3 V, V3 dir, int lobe, int mode,
                            float pdf, V3 att_pre, V3 att, int null_lobe, V3 null_dir) {
        unsigned bits = mmask[rec.material] & ((1u << kAdjBsdfDirs) - 1u);
        if (!bits) return;
        V3 coef;
        if (ps.first) {   // att0: its own adjoint (times the Russian-roulette scale)
            float q = att_pre.x != 0.0f ? att.x / att_pre.x
                                        : (att_pre.y != 0.0f ? att.y / att_pre.y
                                                             : (att_pre.z != 0.0f ? att.z / att_pre.z : 0.0f));
            coef = g_att0 * q;
        } else {          // a factor of everything after this vertex
            V3 g, S;
            target(ps, g, S);
            V3 gs = g * S;
            coef = v3(att_pre.x != 0.0f ? gs.x / att_pre.x : 0.0f, att_pre.y != 0.0f ? gs.y / att_pre.y : 0.0f,
                      att_pre.z != 0.0f ? gs.z / att_pre.z : 0.0f);
        }
        if (is_zero(coef)) return;
        float cw = 1.0f;
        if (mode == SCATTER_SAMPLED) cw = fabsf(dot(rec.n, dir)) / pdf;
        const float* p = params + rec.material * kAdjPerMat;
        for (; bits; bits &= bits - 1u) {
            int k = __ffs(bits) - 1;
            DMat dm = dual_material(*s, m, p, k);
            V3 da = mode == SCATTER_SAMPLED ? dpart(eval_dual(*s, m, dm, rec, V, dir)) * cw
                                            : dpart(lobe_att_dual(*s, m, dm, rec, V, dir, lobe));
            if (mode != SCATTER_SAMPLED) {
                float sc = 0.0f;
                if (lobe >= 0 && lobe <= LOBE_CLEARCOAT && dm.pl[lobe].v < lobe_floor(lobe)) sc += dlog(dm.pl[lobe]);
                if (mode == SCATTER_LEGACY) sc += null_sample_score(m, dm, rec, V, null_lobe, null_dir);
                da = da + att_pre * sc;
            }
            add(rec.material * kAdjPerMat + k, dot(coef, da));
        }
    }
};

template <int STACK>
struct AdjointReplay : AdjointSink {
    // the adjoint captures no AOVs
    RT_D void aov_ray(const Hit&, V3) {}
    RT_D void aov_medium(float, V3) {}
    RT_D void aov_miss(V3) {}
    RT_D void aov_surface(V3, const Material&) {}
    RT_D void aov_bounce(bool, V3) {}
    RT_D void shadow(PathState& ps, V3 o, V3 d, float tmax, V3 c, int to_la) {
        shadow_impl<STACK>(ps, o, d, tmax, c, to_la);
    }
};

}  // namespace rt
