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
    int light_pick;    // RT_LIGHTS_*: 0 every light, 1 / 2 one light by power / uniformly
};

// LightDistribution.Sample (LightDistribution.cs:104-122): the light whose CDF
// entry is the first not below xi, and its pick probability.
RT_D int pick_light(const SceneView& s, int mode, float xi, float& pdf) {
    int n = s.num_lights;
    const float* cdf = s.pick_cdf + (size_t)(mode - 1) * n;
    const float* pp = s.pick_pdf + (size_t)(mode - 1) * n;
    if (n == 1) {
        pdf = pp[0];
        return 0;
    }
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (cdf[mid] < xi) lo = mid + 1;
        else hi = mid;
    }
    pdf = pp[lo];
    return lo;
}

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

// Renderer.WeightEmission (:1549-1565). Out of line: it runs only when a ray
// hits an emitter, and keeping it out of the shading code that every vertex
// runs eases the instruction cache (wavefront shade -1.7%, megakernel -6.8%
// per frame on the icosphere field).
__device__ __noinline__ V3 weight_emission(const SceneView& s, const RenderConst& rc, V3 raw, int mat, V3 o, V3 d, float prev_pdf,
                        int prev_delta) {
    if (prev_delta) return raw;
    int li = s.emitter_light[RT_IX(mat, s.n_materials)];
    if (li >= 0) {
        float pl = light_pdf(s, s.lights[RT_IX(li, s.num_lights)], o, d);
        if (prev_pdf + pl <= 1e-20f) return v3(0.0f);
        return raw * mis_weight(prev_pdf, pl, rc.mis_power);
    }
    return raw;
}

// SampleSky (Renderer.cs:1820-1861) for a flat sky: its radiance, MIS-weighted
// against the EnvironmentLight's uniform-sphere pdf unless the bounce before
// was delta (or no EnvironmentLight samples the sky).
RT_D V3 weight_sky(const SceneView& s, const RenderConst& rc, float prev_pdf, int prev_delta) {
    if (prev_delta || s.env_light < 0) return s.sky;
    float pl = 1.0f / (4.0f * kPi);   // EnvironmentLight.PdfSolidAngle -> FlatSky.Pdf
    if (prev_pdf + pl <= 1e-20f) return v3(0.0f);
    return s.sky * mis_weight(prev_pdf, pl, rc.mis_power);
}

// Path state carried from vertex to vertex. The megakernel keeps it in
// registers; the wavefront stores it in SoA arrays between kernels.
struct PathState {
    V3 o, d;          // current ray
    V3 beta;          // path throughput used by RR and the dead-path test
    V3 w;             // weight of the next vertex's terms (segment factors x attenuations)
    V3 lp, la;        // first-vertex terms; deeper terms relative to att0
    V3 pre, att0;     // first-vertex weight and attenuation (primary clamp)
    V3 cur_abs;       // interior Beer-Lambert sigma_a of the current segment
    V3 mask;          // channels still live in la (per-frame sanitize)
    float prev_pdf;
    int prev_delta;
    int first;        // no scattering vertex yet
    int clamp_mode;   // the first vertex was a surface
    int depth;        // TraceRay depth of the next segment
    Sampler rng;
    IorStackD iors;

    // Adds a term of the current vertex (already weighted) to lp or la.
    RT_D void add(V3 x, int to_la) {
        if (!to_la) {
            lp = lp + x;
            return;
        }
        if (!isfinite(x.x)) mask.x = 0.0f;
        if (!isfinite(x.y)) mask.y = 0.0f;
        if (!isfinite(x.z)) mask.z = 0.0f;
        la = la + v3(mask.x != 0.0f ? x.x : 0.0f, mask.y != 0.0f ? x.y : 0.0f, mask.z != 0.0f ? x.z : 0.0f);
    }
};

// Camera sample setup (Renderer.cs:615-653): pixel seed, 2 jitter draws,
// pinhole ray (Camera.cs:127-139).
RT_D void path_init(PathState& ps, const RenderConst& rc, int px, int py, uint32_t sample_index) {
    uint32_t seed = ((uint32_t)px * 73856093u) ^ ((uint32_t)py * 19349663u);
    ps.rng = Sampler{seed, sample_index, 0u};
    float ju = ps.rng.next();
    float jv = ps.rng.next();
    float u = ((float)px + ju) / (float)rc.width;
    float v = ((float)(rc.height - py - 1) + jv) / (float)rc.height;
    V3 target = rc.cam.llc + u * rc.cam.horizontal + v * rc.cam.vertical;
    ps.o = rc.cam.origin;
    ps.d = target - rc.cam.origin;
    ps.beta = v3(1.0f);
    ps.w = v3(1.0f);
    ps.lp = v3(0.0f);
    ps.la = v3(0.0f);
    ps.pre = v3(1.0f);
    ps.att0 = v3(0.0f);
    ps.cur_abs = v3(0.0f);
    ps.mask = v3(1.0f);
    ps.prev_pdf = 0.0f;
    ps.prev_delta = 1;
    ps.first = 1;
    ps.clamp_mode = 0;
    ps.depth = rc.max_depth;
    ps.iors.n = 0;
}

// Entry test of TraceRay (Renderer.cs:1589-1603): depth and dead path.
RT_D bool path_alive(const PathState& ps) { return ps.depth > 0 && max3(ps.beta) >= 1e-4f; }

// The clamped sample radiance (ClampRadianceIndirect at the primary surface,
// then ClampRadiance; Renderer.cs:670, 1380-1381).
RT_D V3 path_resolve(const PathState& ps, const RenderConst& rc) {
    V3 L = ps.lp;
    if (ps.clamp_mode) L = L + ps.pre * clamp_lum(ps.att0 * sanitize(ps.la), rc.ind_max);
    return clamp_lum(L, rc.max_rad);
}

// NEE at a surface vertex: ComputeDirectLighting (Renderer.cs:1894-2036),
// every light (strategy All) or one picked light (Power, Uniform). The BSDF integrand and the MIS weight are evaluated
// before the shadow ray and the ray is dropped when they are zero (the
// reference casts it first; only the cost differs: every draw happens in the
// light sampler). Each unoccluded sample adds w * colour * brdf * Tr_medium,
// times the vertex weight, through the sink.
// MEDIUM = false compiles the participating-medium terms out (a batch none of
// whose scenes has a medium).
template <bool MEDIUM = true, class Sink>
RT_D void nee_surface(const SceneView& s, const RenderConst& rc, PathState& ps, const Surface& rec,
                      const Material& m, V3 view, Sink& sink) {
    float view_term = shadow_terminator(rec.n, rec.n, view);
    int to_la = ps.clamp_mode;
    int l0 = 0, l1 = s.num_lights;
    float p_pick = 1.0f, inv_pick = 1.0f;
    if (rc.light_pick) {   // single-light picking (Renderer.cs:1907-1974): lightAccum / pPick
        if (s.num_lights == 0) return;
        l0 = pick_light(s, rc.light_pick, ps.rng.next(), p_pick);
        l1 = l0 + 1;
        inv_pick = p_pick > 0.0f ? 1.0f / p_pick : 0.0f;
    }
    for (int li = l0; li < l1; li++) {
        const Light& l = s.lights[RT_IX(li, s.num_lights)];
        for (int si = 0; si < l.shadow_samples; si++) {
            LightSample ls = light_sample(s, l, rec.p, rec.n, si, ps.rng);
            if (ls.occluded || !ls.has_ray) continue;
            V3 brdf = bsdf_eval_direct(s, m, rec, ls.dir, view, rec.n);
            float term = view_term * shadow_terminator(rec.n, rec.n, ls.dir);
            brdf = brdf * term;
            if (is_zero(brdf)) {
                sink.skipped(ls.ray_o, ls.dir, ls.ray_tmax);
                continue;
            }
            V3 tr_m = v3(1.0f);
            if (MEDIUM && s.has_medium) tr_m = medium_tr(s, ls.dist >= kInf ? 1e30f : ls.dist);
            float wgt = 1.0f;
            if (!l.is_delta) {
                float pb = bsdf_pdf(m, rec, view, ls.dir);
                if (pb > 0.0f) {
                    float pl = p_pick * light_pdf(s, l, rec.p, ls.dir);   // pNee = pPick * pLightSample
                    wgt = (pl + pb > 0.0f) ? mis_weight(pl, pb, rc.mis_power) : 1.0f;
                }
            }
            wgt *= inv_pick;
            V3 c = ps.w * (wgt * ls.color * brdf * tr_m);
            sink.shadow(ps, ls.ray_o, ls.dir, ls.ray_tmax, c, to_la);
            sink.nee_surface(ps, li, m, rec, ls.dir, view, term, ps.w * (wgt * ls.color), ls.dist, tr_m, to_la);
        }
    }
}

// NEE at a medium scattering point: ComputeDirectLightingMedium
// (Renderer.cs:2099-2206), every light or one picked light.
template <class Sink>
RT_D void nee_medium(const SceneView& s, const RenderConst& rc, PathState& ps, V3 p, V3 wo, Sink& sink) {
    int to_la = ps.clamp_mode;
    int l0 = 0, l1 = s.num_lights;
    float p_pick = 1.0f, inv_pick = 1.0f;
    if (rc.light_pick) {   // single-light picking in the volumetric path (Renderer.cs:2110-2160)
        if (s.num_lights == 0) return;
        l0 = pick_light(s, rc.light_pick, ps.rng.next(), p_pick);
        l1 = l0 + 1;
        inv_pick = p_pick > 0.0f ? 1.0f / p_pick : 0.0f;
    }
    for (int li = l0; li < l1; li++) {
        const Light& l = s.lights[RT_IX(li, s.num_lights)];
        for (int si = 0; si < l.shadow_samples; si++) {
            LightSample ls = light_sample(s, l, p, v3(0.0f), si, ps.rng);
            if (ls.occluded || !ls.has_ray) continue;
            float ph = hg_eval(s.hg_g, wo, ls.dir);
            V3 tr_m = medium_tr(s, ls.dist >= kInf ? 1e30f : ls.dist);
            float wgt = 1.0f;
            if (!l.is_delta && ph > 0.0f) {
                float pl = p_pick * light_pdf(s, l, p, ls.dir);
                if (pl + ph > 0.0f) wgt = mis_weight(pl, ph, rc.mis_power);
            }
            wgt *= inv_pick;
            V3 c = ps.w * (wgt * ls.color * ph * tr_m);
            sink.shadow(ps, ls.ray_o, ls.dir, ls.ray_tmax, c, to_la);
            sink.nee_medium(ps, li, ls.dist, to_la);
        }
    }
}

// Russian roulette on the projected throughput (Renderer.cs:1283-1294).
// q_used: the survival probability a surviving path was drawn against, 0 when
// the roulette did not run.
RT_D bool russian_roulette(const RenderConst& rc, int depth, V3& att, V3& next_beta, Sampler& rng, float& q_used) {
    int used = rc.max_depth - depth;
    q_used = 0.0f;
    if (used >= rc.rr_min_bounces) {
        float q = fmaxf(next_beta.x, fmaxf(next_beta.y, next_beta.z));
        q = fmaxf(q, rc.rr_min_survival);
        q = fminf(q, 0.95f);
        if (rng.next() > q) return false;
        q_used = q;
        float inv = 1.0f / q;
        att = att * inv;
        next_beta = next_beta * inv;
    }
    return true;
}

RT_D V3 bl_factor(V3 sigma, float t) { return beer_lambert(v3(1.0f), sigma, t); }

// Adjoint hooks. shade_vertex reports every factor that multiplies the path
// weight and every term it adds, so that the path-replay adjoint can run the
// same code; the forward sinks inherit these empty versions, which compile
// away.
enum : int { SEG_ABSORPTION = 0, SEG_MEDIUM_PASS = 1, SEG_MEDIUM_SCATTER = 2 };
enum : int { SCATTER_SAMPLED = 0, SCATTER_DELTA = 1, SCATTER_LEGACY = 2 };
struct NoAdjoint {
    // ps.w is about to be multiplied by the factors of a segment of length t:
    // interior Beer-Lambert (all modes but SEG_MEDIUM_PASS) and the medium.
    RT_D void segment(const PathState&, float, int) {}
    // The interior absorption now belongs to material `mat` (-1: none).
    RT_D void interior(int) {}
    // An emitted-radiance term ps.w * we was just added.
    RT_D void emission(const PathState&, int, V3, int) {}
    // A surface NEE sample: the term coef * brdf * term * tr_m * tr went through shadow().
    RT_D void nee_surface(const PathState&, int, const Material&, const Surface&, V3, V3, float, V3, float, V3,
                          int) {}
    RT_D void nee_medium(const PathState&, int, float, int) {}
    // A path survived Russian roulette drawn against q = clamp(max(thr)); its
    // throughput now carries 1/q. first: the roulette of the first surface
    // vertex (whose attenuation becomes att0).
    RT_D void roulette(const PathState&, V3, float, int) {}
    // The vertex attenuation: att_pre before Russian roulette, att after. For
    // the legacy path, the lobe and direction of the null sample before it.
    RT_D void scatter(const PathState&, const Material&, const Surface&, V3, V3, int, int, float, V3, V3, int, V3) {}

    // Capture hooks (the AOV probe, Renderer.cs:1051-1054, 1139-1145,
    // 1271-1277, 1657-1662, 1716-1724, 1849-1850). None of them draws from
    // the sampler, so a capturing render traces the same paths.
    // The closest hit of the current ray (d its direction).
    RT_D void aov_ray(const Hit&, V3) {}
    // A medium scattering event at distance t along direction d.
    RT_D void aov_medium(float, V3) {}
    // The ray left the scene (the flat sky's radiance).
    RT_D void aov_miss(V3) {}
    // The surface ShadeSurface is about to shade.
    RT_D void aov_surface(V3, const Material&) {}
    // The bounce decision: a delta lobe with attenuation f, or a non-delta one.
    RT_D void aov_bounce(bool, V3) {}
};

// One vertex of TraceRay given the closest hit of the current ray: the
// volumetric branch (Renderer.cs:1704-1782), ShadeSurface (:1008-1228) and
// ShadeSampleBounce (:1235-1383). Returns true when the path continues with
// ps.o/ps.d as the next ray (ps.depth already decremented). MEDIUM = false
// compiles the volumetric branch out; TRANSMIT = false the specular
// transmission lobe and the IOR stack (no material has specTrans > 0).
template <bool MEDIUM = true, bool TRANSMIT = true, class Sink>
__device__ __forceinline__ bool shade_vertex(const SceneView& s, const RenderConst& rc, PathState& ps, const Hit& h,
                                             Sink& sink) {
    bool hit = h.kind != HIT_NONE;
    V3 beta_s = ps.beta;
    sink.aov_ray(h, ps.d);
    if (MEDIUM && s.has_medium) {
        float tmax = hit ? h.t : 1e30f;
        float tmed;
        V3 mb;
        bool sc = medium_sample(s, tmax, ps.rng, tmed, mb);
        if (sc) {
            V3 p = ps.o + ps.d * tmed;
            sink.aov_medium(tmed, ps.d);
            sink.segment(ps, tmed, SEG_MEDIUM_SCATTER);
            ps.w = ps.w * bl_factor(ps.cur_abs, tmed) * mb;
            nee_medium(s, rc, ps, p, ps.d, sink);
            V3 mthr = ps.beta * mb;
            int used = rc.max_depth - ps.depth;
            float scale = 1.0f;
            if (used >= rc.rr_min_bounces) {
                float q = fmaxf(mthr.x, fmaxf(mthr.y, mthr.z));
                q = fmaxf(q, rc.rr_min_survival);
                q = fminf(q, 0.95f);
                if (ps.rng.next() > q) return false;
                scale = 1.0f / q;
                sink.roulette(ps, mthr, q, 0);
            }
            float ppdf;
            V3 wi = hg_sample(s.hg_g, ps.d, ps.rng, ppdf);
            float pv = hg_eval(s.hg_g, ps.d, wi);
            float pw = ppdf > 1e-20f ? pv / ppdf : 0.0f;
            ps.beta = mthr * (pw * scale);
            ps.w = ps.w * (pw * scale);
            ps.o = p;
            ps.d = wi;
            ps.prev_pdf = ppdf;
            ps.prev_delta = 0;
            ps.first = 0;   // a medium first vertex: no primary clamp
            ps.depth -= 1;
            return path_alive(ps);
        }
        sink.segment(ps, tmax, SEG_MEDIUM_PASS);
        ps.w = ps.w * mb;
        beta_s = ps.beta * mb;
    }
    if (!hit) {   // SampleSky, then TraceRay's Beer-Lambert over an infinite segment
        if (s.sky_on) ps.add(ps.w * weight_sky(s, rc, ps.prev_pdf, ps.prev_delta) * bl_factor(ps.cur_abs, INFINITY),
                             ps.clamp_mode);
        sink.aov_miss(s.sky);
        return false;
    }
    sink.segment(ps, h.t, SEG_ABSORPTION);
    ps.w = ps.w * bl_factor(ps.cur_abs, h.t);
    Surface rec = make_surface(s, h, ps.o, ps.d);
    const Material& m = s.materials[rec.material];
    sink.aov_surface(rec.n, m);
    int to_la = ps.clamp_mode;
    if (m.type != 0) {   // Emissive: Emit (front face only), no NEE, no scatter
        if (rec.front && (m.emission.x > 0.0f || m.emission.y > 0.0f || m.emission.z > 0.0f)) {
            V3 we = weight_emission(s, rc, m.emission, rec.material, ps.o, ps.d, ps.prev_pdf, ps.prev_delta);
            ps.add(ps.w * we, to_la);
            sink.emission(ps, rec.material, we, to_la);
        }
        return false;
    }
    V3 view = normalize(-ps.d);
    float rel_eta = 0.0f;
    bool dielectric = TRANSMIT && !m.thin_walled && m.spec_trans_raw > 0.0f;
    if (dielectric) rel_eta = rec.front ? (ps.iors.top() / m.ior_raw) : (m.ior_raw / ps.iors.enclosing());
    nee_surface<MEDIUM>(s, rc, ps, rec, m, view, sink);
    BsdfSample bs;
    V3 att, next_o, next_d, next_beta;
    float next_pdf;
    int next_delta;
    V3 latt, ldir;
    int llobe = -1;
    int drawn = bsdf_sample_or_scatter<TRANSMIT>(s, m, rec, view, ps.d, rel_eta, ps.rng, bs, latt, ldir, llobe);
    if (drawn == 1) {   // ShadeSampleBounce
        if (bs.is_delta) {
            att = bs.f;
        } else {
            float a = fabsf(dot(rec.n, bs.wo));
            if (a <= 0.0f || bs.pdf <= 0.0f) return false;
            att = bs.f * a / bs.pdf;
        }
        sink.aov_bounce(bs.is_delta, bs.f);
        next_beta = beta_s * att;
        V3 att_pre = att, thr = next_beta;
        float q_rr;
        if (!russian_roulette(rc, ps.depth, att, next_beta, ps.rng, q_rr)) return false;
        if (q_rr > 0.0f) sink.roulette(ps, thr, q_rr, ps.first);
        sink.scatter(ps, m, rec, view, bs.wo, bs.lobe, bs.is_delta ? SCATTER_DELTA : SCATTER_SAMPLED, bs.pdf,
                     att_pre, att, -1, bs.wo);
        V3 off = dot(bs.wo, rec.n) >= 0.0f ? rec.n : -rec.n;
        next_o = offset_origin(rec.p, off);
        next_d = bs.wo;
        next_pdf = bs.is_delta ? 0.0f : bs.pdf;
        next_delta = bs.is_delta;
        if (bs.has_next_absorption) {
            ps.cur_abs = bs.next_absorption;
            sink.interior(near_zero(bs.next_absorption) ? -1 : rec.material);
        }
        if (TRANSMIT && rc.dielectrics && bs.transition == 1) ps.iors.push(dielectric ? m.ior_raw : ps.iors.top());
        if (TRANSMIT && rc.dielectrics && bs.transition == 2) ps.iors.pop();
    } else {   // Sample returned null: the legacy Scatter path (:1127-1225)
        if (drawn == 0) return false;
        V3 sdir = ldir;
        int lobe = llobe;
        att = latt;
        sink.aov_bounce(false, att);   // Disney's IsDeltaScatter is false
        next_beta = beta_s * att;
        V3 att_pre = att, thr = next_beta;
        float q_rr;
        if (!russian_roulette(rc, ps.depth, att, next_beta, ps.rng, q_rr)) return false;
        if (q_rr > 0.0f) sink.roulette(ps, thr, q_rr, ps.first);
        sink.scatter(ps, m, rec, view, sdir, lobe, SCATTER_LEGACY, 1.0f, att_pre, att, bs.lobe, bs.tried);
        next_o = rec.p;
        next_d = sdir;
        next_pdf = 0.0f;
        next_delta = 0;
        if (rc.dielectrics && dielectric && dot(sdir, rec.n) < 0.0f) {
            if (rec.front) ps.iors.push(m.ior_raw);
            else ps.iors.pop();
        }
    }
    if (ps.first) {   // primary surface: deeper terms are clamped as one (:1380-1381)
        ps.first = 0;
        ps.clamp_mode = 1;
        ps.pre = ps.w;
        ps.att0 = att;
        ps.w = v3(1.0f);
    } else {
        ps.w = ps.w * att;
    }
    ps.beta = next_beta;
    ps.o = next_o;
    ps.d = next_d;
    ps.prev_pdf = next_pdf;
    ps.prev_delta = next_delta;
    ps.depth -= 1;
    return path_alive(ps);
}

// Shadow sink of the megakernel: traces the shadow ray at once.
template <int STACK>
struct InlineShadows : NoAdjoint {
    const SceneView* s;
    int opaque;
    Counters* cnt;
    int* err;
    RT_D void shadow(PathState& ps, V3 o, V3 d, float tmax, V3 c, int to_la) {
        V3 tr = shadow_transmittance<STACK>(*s, opaque, o, d, kEps, tmax, cnt, err);
        if (near_zero(tr)) return;
        ps.add(c * tr, to_la);
    }
    // A shadow ray the reference casts but whose contribution is zero: traced
    // only by the counting build, so the work counts are the reference's.
    RT_D void skipped(V3 o, V3 d, float tmax) {
        if (cnt) shadow_transmittance<STACK>(*s, opaque, o, d, kEps, tmax, cnt, err);
    }
};

// Traces one camera sample of pixel (px, py) to the end and returns the
// clamped sample radiance. cnt (counting builds only) accumulates the work.
template <int STACK, bool COUNT>
__device__ V3 trace_sample(const SceneView& s, const RenderConst& rc, int px, int py, uint32_t sample_index,
                           Counters* cnt, int* err) {
    if (!COUNT) cnt = nullptr;
    PathState ps;
    path_init(ps, rc, px, py, sample_index);
    InlineShadows<STACK> sink{{}, &s, rc.opaque, cnt, err};
    while (path_alive(ps)) {
        Hit h;
        if (COUNT) cnt->closest_rays++;
        traverse<false, STACK>(s, ps.o, ps.d, kEps, kInf, h, COUNT ? &cnt->closest : nullptr, err);
        if (!shade_vertex(s, rc, ps, h, sink)) break;
    }
    return path_resolve(ps, rc);
}

// The AOV probe of one camera path (Renderer.cs:776-815): depth at the camera
// ray's first surface hit; albedo and normal at the first non-delta surface,
// with a specular chain's tint folded into weight; a medium scatter commits
// white with no normal, a miss the (black) sky.
struct AovProbe {
    bool pending, have_depth, camera;
    float depth;
    V3 weight, tent_albedo, tent_normal, albedo, normal;
    RT_D void reset() {
        pending = true;
        have_depth = false;
        camera = true;
        depth = -1.0f;
        weight = v3(1.0f);
        tent_albedo = v3(1.0f);
        tent_normal = v3(0.0f);
        albedo = v3(0.0f);
        normal = v3(0.0f);
    }
    RT_D void commit() {
        albedo = weight * tent_albedo;
        normal = tent_normal;
        pending = false;
    }
    RT_D void commit_as(V3 a, V3 n) {
        albedo = weight * a;
        normal = n;
        pending = false;
    }
};

RT_D V3 clamp01(V3 v) {   // Vector3.Clamp(v, Zero, One)
    return v3(fminf(fmaxf(v.x, 0.0f), 1.0f), fminf(fmaxf(v.y, 0.0f), 1.0f), fminf(fmaxf(v.z, 0.0f), 1.0f));
}

// The megakernel's shadow sink plus the capture hooks on a probe.
template <int STACK>
struct CaptureShadows : InlineShadows<STACK> {
    AovProbe* probe;
    RT_D void aov_ray(const Hit& h, V3 d) {
        AovProbe& p = *probe;
        if (p.camera && h.kind != HIT_NONE && p.pending && !p.have_depth) {   // :1657-1662
            p.depth = h.t * length(d);
            p.have_depth = true;
        }
        p.camera = false;
    }
    RT_D void aov_medium(float t, V3 d) {   // :1716-1724
        AovProbe& p = *probe;
        if (!p.pending) return;
        if (!p.have_depth) {
            p.depth = t * length(d);
            p.have_depth = true;
        }
        p.commit_as(v3(1.0f), v3(0.0f));
    }
    RT_D void aov_miss(V3 sky) {   // :1849-1850
        if (probe->pending) probe->commit_as(clamp01(sky), v3(0.0f));
    }
    RT_D void aov_surface(V3 n, const Material& m) {   // :1051-1054
        if (!probe->pending) return;
        probe->tent_normal = n;
        probe->tent_albedo = clamp01(m.base);   // AovAlbedo: baseColor, or an Emissive's colour
    }
    RT_D void aov_bounce(bool delta, V3 f) {   // :1139-1145, 1271-1277
        if (!probe->pending) return;
        if (delta) probe->weight = probe->weight * clamp01(f);
        else probe->commit();
    }
};

// trace_sample with the probe: returns the clamped sample radiance and leaves
// the path's committed features in *probe.
template <int STACK>
__device__ V3 trace_capture(const SceneView& s, const RenderConst& rc, int px, int py, uint32_t sample_index,
                            AovProbe* probe, int* err) {
    PathState ps;
    path_init(ps, rc, px, py, sample_index);
    probe->reset();
    CaptureShadows<STACK> sink{{{}, &s, rc.opaque, nullptr, err}, probe};
    while (path_alive(ps)) {
        Hit h;
        traverse<false, STACK>(s, ps.o, ps.d, kEps, kInf, h, nullptr, err);
        if (!shade_vertex(s, rc, ps, h, sink)) break;
    }
    if (probe->pending) probe->commit();   // CaptureAccumulator.Add (:835-837)
    return path_resolve(ps, rc);
}

}  // namespace rt
