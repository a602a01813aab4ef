// One camera sample, traced to the end in forward (loop) form.
//
// Renderer.TraceRay (Rendering/Renderer.cs:1581-1783) is recursive; the value
// it returns for the camera ray is
//     L0 = W0 * (e0 + d0 + clampInd(att0 * S(L1)))     (first vertex on a surface)
//     Lk = Wk * (ek + dk + attk * S(L(k+1)))             (deeper vertices)
// with W the segment factors (medium beta, interior Beer-Lambert), S the
// per-frame sanitize and clampInd the primary-surface indirect clamp
// (Renderer.cs:1378-1381). The loop below accumulates the same sum front to
// back: terms of the first vertex go to Lp, deeper terms to La weighted by the
// product of the attenuations after the first vertex, and the clamp is applied
// to att0 * La at the end. The RNG dimension sequence, the throughput used by
// Russian roulette and every branch decision are those of the recursion; only
// the order of the final additions differs.
#pragma once

#include "device.cuh"

namespace rt {

struct RenderConst {
    Camera cam;
    int width, height;
    int max_depth;
    float max_rad, ind_max;
    int mis_power;
    int rr_min_bounces;
    float rr_min_survival;
    int opaque;        // no material transmits shadow rays: any-hit shadows
    int dielectrics;   // a solid dielectric exists: keep the IOR stack
};

struct IorStackD {   // Volumetrics/IorStack.cs (capacity 8)
    float slot[8];
    int n;
    RT_D float top() const { return n == 0 ? 1.0f : slot[n - 1]; }
    RT_D float enclosing() const { return n >= 2 ? slot[n - 2] : 1.0f; }
    RT_D void push(float v) {
        if (n >= 8) {
            for (int i = 0; i < 7; i++) slot[i] = slot[i + 1];
            slot[7] = v;
            return;
        }
        slot[n++] = v;
    }
    RT_D void pop() {
        if (n > 0) n--;
    }
};

RT_D float shadow_terminator(V3 ng, V3 ns, V3 w) {   // Core/MathUtils.cs:44-61
    float ng_w = dot(ng, w);
    if (ng_w <= 0.0f) return 0.0f;
    float ns_w = dot(ns, w);
    if (ns_w <= 0.0f) return 0.0f;
    float ng_ns = dot(ng, ns);
    if (ng_ns >= 0.9999f) return 1.0f;
    float g = ng_w / (ns_w * fmaxf(ng_ns, 1e-4f));
    if (g >= 1.0f) return 1.0f;
    if (g <= 0.0f) return 0.0f;
    float g2 = g * g;
    return (-g2 * g) + g2 + g;
}

// Renderer.WeightEmission (:1549-1565)
RT_D V3 weight_emission(const SceneView& s, const RenderConst& rc, V3 raw, int mat, V3 o, V3 d, float prev_pdf,
                        int prev_delta) {
    if (prev_delta) return raw;
    int li = s.emitter_light[mat];
    if (li >= 0) {
        float pl = light_pdf(s, s.lights[li], o, d);
        if (prev_pdf + pl <= 1e-20f) return v3(0.0f);
        return raw * mis_weight(prev_pdf, pl, rc.mis_power);
    }
    return raw;
}

// ComputeDirectLighting, strategy All (Renderer.cs:1894-2036). The BSDF
// integrand and MIS weight are evaluated before the shadow ray, and the ray is
// skipped when they are zero: the reference casts it first, which changes
// nothing but the cost (all draws happen in the light sampler).
template <int STACK>
__device__ __forceinline__ V3 direct_lighting(const SceneView& s, const RenderConst& rc, const Surface& rec,
                                              const Material& m, V3 view, Sampler& rng, Counters* cnt, int* err) {
    V3 result = v3(0.0f);
    float view_term = shadow_terminator(rec.n, rec.n, view);
    for (int li = 0; li < s.num_lights; li++) {
        const Light& l = s.lights[li];
        V3 acc = v3(0.0f);
        for (int si = 0; si < l.shadow_samples; si++) {
            LightSample ls = light_sample(s, l, rec.p, rec.n, si, rng);
            if (ls.occluded) continue;
            V3 brdf = bsdf_eval_direct(s, m, rec, ls.dir, view, rec.n);
            brdf = brdf * (view_term * shadow_terminator(rec.n, rec.n, ls.dir));
            if (is_zero(brdf)) continue;
            V3 color = ls.color;
            if (ls.has_ray) {
                V3 tr = shadow_transmittance<STACK>(s, rc.opaque, ls.ray_o, ls.dir, kEps, ls.ray_tmax, cnt, err);
                if (near_zero(tr)) continue;
                color = color * tr;
            }
            V3 tr_m = v3(1.0f);
            if (s.has_medium) tr_m = medium_tr(s, ls.dist >= kInf ? 1e30f : ls.dist);
            float w = 1.0f;
            if (!l.is_delta) {
                float pb = bsdf_pdf(m, rec, view, ls.dir);
                if (pb > 0.0f) {
                    float pl = light_pdf(s, l, rec.p, ls.dir);
                    w = (pl + pb > 0.0f) ? mis_weight(pl, pb, rc.mis_power) : 1.0f;
                }
            }
            acc = acc + w * color * brdf * tr_m;
        }
        result = result + acc;
    }
    return result;
}

// ComputeDirectLightingMedium, strategy All (Renderer.cs:2162-2203)
template <int STACK>
__device__ __forceinline__ V3 direct_lighting_medium(const SceneView& s, const RenderConst& rc, V3 p, V3 wo,
                                                     Sampler& rng, Counters* cnt, int* err) {
    V3 result = v3(0.0f);
    for (int li = 0; li < s.num_lights; li++) {
        const Light& l = s.lights[li];
        V3 acc = v3(0.0f);
        for (int si = 0; si < l.shadow_samples; si++) {
            LightSample ls = light_sample(s, l, p, v3(0.0f), si, rng);
            if (ls.occluded) continue;
            V3 color = ls.color;
            if (ls.has_ray) {
                V3 tr = shadow_transmittance<STACK>(s, rc.opaque, ls.ray_o, ls.dir, kEps, ls.ray_tmax, cnt, err);
                if (near_zero(tr)) continue;
                color = color * tr;
            }
            float ph = hg_eval(s.hg_g, wo, ls.dir);
            V3 tr_m = medium_tr(s, ls.dist >= kInf ? 1e30f : ls.dist);
            float w = 1.0f;
            if (!l.is_delta && ph > 0.0f) {
                float pl = light_pdf(s, l, p, ls.dir);
                if (pl + ph > 0.0f) w = mis_weight(pl, ph, rc.mis_power);
            }
            acc = acc + w * color * ph * tr_m;
        }
        result = result + acc;
    }
    return result;
}

// Russian roulette on the projected throughput (Renderer.cs:1283-1294).
RT_D bool russian_roulette(const RenderConst& rc, int depth, V3& att, V3& next_beta, Sampler& rng) {
    int used = rc.max_depth - depth;
    if (used >= rc.rr_min_bounces) {
        float q = fmaxf(next_beta.x, fmaxf(next_beta.y, next_beta.z));
        q = fmaxf(q, rc.rr_min_survival);
        q = fminf(q, 0.95f);
        if (rng.next() > q) return false;
        float inv = 1.0f / q;
        att = att * inv;
        next_beta = next_beta * inv;
    }
    return true;
}

struct Accum {
    V3 lp, la;       // first-vertex terms; deeper terms (relative to att0)
    V3 mask;         // channels still live in la (per-frame sanitize)
    int after;       // 1 once the first vertex has scattered
    RT_D void add(V3 x) {
        if (!after) {
            lp = lp + x;
            return;
        }
        if (!isfinite(x.x)) mask.x = 0.0f;
        if (!isfinite(x.y)) mask.y = 0.0f;
        if (!isfinite(x.z)) mask.z = 0.0f;
        la = la + v3(mask.x != 0.0f ? x.x : 0.0f, mask.y != 0.0f ? x.y : 0.0f, mask.z != 0.0f ? x.z : 0.0f);
    }
};

RT_D V3 bl_factor(V3 sigma, float t) { return beer_lambert(v3(1.0f), sigma, t); }

// Traces one camera sample of pixel (px, py) and returns the clamped sample
// radiance (ClampRadiance applied, Renderer.cs:670). cnt (counting builds
// only) accumulates the traversal work.
template <int STACK, bool COUNT>
__device__ V3 trace_sample(const SceneView& s, const RenderConst& rc, int px, int py, uint32_t sample_index,
                           Counters* cnt, int* err) {
    if (!COUNT) cnt = nullptr;
    uint32_t seed = ((uint32_t)px * 73856093u) ^ ((uint32_t)py * 19349663u);   // Renderer.cs:615
    Sampler rng{seed, sample_index, 0u};
    float ju = rng.next();
    float jv = rng.next();
    float u = ((float)px + ju) / (float)rc.width;
    float v = ((float)(rc.height - py - 1) + jv) / (float)rc.height;
    V3 target = rc.cam.llc + u * rc.cam.horizontal + v * rc.cam.vertical;   // Camera.cs:127-139
    V3 o = rc.cam.origin;
    V3 d = target - rc.cam.origin;
    V3 beta = v3(1.0f);
    float prev_pdf = 0.0f;
    int prev_delta = 1;
    V3 cur_abs = v3(0.0f);
    IorStackD iors;
    iors.n = 0;
    Accum acc{v3(0.0f), v3(0.0f), v3(1.0f), 0};
    V3 W = v3(1.0f), pre = v3(1.0f), att0 = v3(0.0f);
    int clamp_mode = 0;
    int first = 1;
    for (int depth = rc.max_depth; depth > 0; --depth) {
        if (max3(beta) < 1e-4f) break;   // dead path (Renderer.cs:1600-1603)
        Hit h;
        if (COUNT) cnt->closest_rays++;
        traverse<false, STACK>(s, o, d, kEps, kInf, h, cnt, err);
        bool hit = h.kind != HIT_NONE;
        V3 beta_s = beta;
        if (s.has_medium) {   // volumetric branch (Renderer.cs:1704-1782)
            float tmax = hit ? h.t : 1e30f;
            float tmed;
            V3 mb;
            bool sc = medium_sample(s, tmax, rng, tmed, mb);
            if (sc) {
                V3 p = o + d * tmed;
                W = W * bl_factor(cur_abs, tmed) * mb;
                V3 lnee = direct_lighting_medium<STACK>(s, rc, p, d, rng, cnt, err);
                acc.add(W * lnee);
                V3 mthr = beta * mb;
                int used = rc.max_depth - depth;
                float scale = 1.0f;
                if (used >= rc.rr_min_bounces) {
                    float q = fmaxf(mthr.x, fmaxf(mthr.y, mthr.z));
                    q = fmaxf(q, rc.rr_min_survival);
                    q = fminf(q, 0.95f);
                    if (rng.next() > q) break;
                    scale = 1.0f / q;
                }
                float ppdf;
                V3 wi = hg_sample(s.hg_g, d, rng, ppdf);
                float pv = hg_eval(s.hg_g, d, wi);
                float pw = ppdf > 1e-20f ? pv / ppdf : 0.0f;
                beta = mthr * (pw * scale);
                W = W * (pw * scale);
                o = p;
                d = wi;
                prev_pdf = ppdf;
                prev_delta = 0;
                if (first) {
                    first = 0;
                    acc.after = 0;   // a medium first vertex: no primary clamp, keep summing into lp
                }
                continue;
            }
            W = W * mb;
            beta_s = beta * mb;
        }
        if (!hit) break;   // black flat sky: SampleSky returns 0
        W = W * bl_factor(cur_abs, h.t);
        Surface rec = make_surface(s, h, o, d);
        const Material& m = s.materials[rec.material];
        if (m.type != 0) {   // Emissive: Emit (front face only), no NEE, no scatter
            if (rec.front && (m.emission.x > 0.0f || m.emission.y > 0.0f || m.emission.z > 0.0f))
                acc.add(W * weight_emission(s, rc, m.emission, rec.material, o, d, prev_pdf, prev_delta));
            break;
        }
        V3 view = normalize(-d);
        float rel_eta = 0.0f;
        bool dielectric = !m.thin_walled && m.spec_trans_raw > 0.0f;
        if (dielectric) rel_eta = rec.front ? (iors.top() / m.ior_raw) : (m.ior_raw / iors.enclosing());
        V3 direct = direct_lighting<STACK>(s, rc, rec, m, view, rng, cnt, err);
        acc.add(W * direct);
        BsdfSample bs;
        V3 att, next_o, next_d;
        float next_pdf;
        int next_delta;
        V3 next_beta;
        if (bsdf_sample(s, m, rec, view, rel_eta, rng, bs)) {   // ShadeSampleBounce (:1235-1383)
            if (bs.is_delta) {
                att = bs.f;
            } else {
                float a = fabsf(dot(rec.n, bs.wo));
                if (a <= 0.0f || bs.pdf <= 0.0f) break;
                att = bs.f * a / bs.pdf;
            }
            next_beta = beta_s * att;
            if (!russian_roulette(rc, depth, att, next_beta, rng)) break;
            V3 off = dot(bs.wo, rec.n) >= 0.0f ? rec.n : -rec.n;
            next_o = offset_origin(rec.p, off);
            next_d = bs.wo;
            next_pdf = bs.is_delta ? 0.0f : bs.pdf;
            next_delta = bs.is_delta;
            if (bs.has_next_absorption) cur_abs = bs.next_absorption;
            if (rc.dielectrics && bs.transition == 1) iors.push(dielectric ? m.ior_raw : iors.top());
            if (rc.dielectrics && bs.transition == 2) iors.pop();
        } else {   // Sample returned null: the legacy Scatter path (:1127-1225)
            V3 sdir;
            int lobe;
            if (!bsdf_scatter(s, m, rec, d, rel_eta, rng, att, sdir, lobe)) break;
            next_beta = beta_s * att;
            if (!russian_roulette(rc, depth, att, next_beta, rng)) break;
            next_o = rec.p;
            next_d = sdir;
            next_pdf = 0.0f;
            next_delta = 0;
            if (rc.dielectrics && dielectric && dot(sdir, rec.n) < 0.0f) {
                if (rec.front) iors.push(m.ior_raw);
                else iors.pop();
            }
        }
        if (first) {   // primary surface: later terms are clamped as one (:1380-1381)
            first = 0;
            clamp_mode = 1;
            pre = W;
            att0 = att;
            W = v3(1.0f);
            acc.after = 1;
        } else {
            W = W * att;
        }
        beta = next_beta;
        o = next_o;
        d = next_d;
        prev_pdf = next_pdf;
        prev_delta = next_delta;
    }
    V3 L = acc.lp;
    if (clamp_mode) L = L + pre * clamp_lum(att0 * sanitize(acc.la), rc.ind_max);
    return clamp_lum(L, rc.max_rad);
}

}  // namespace rt
