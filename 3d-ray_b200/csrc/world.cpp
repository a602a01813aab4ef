// Host-side world assembly and the binned-SAH BVH build (see world.h).
// Compiled with -ffp-contract=off: every float result here must equal what the
// C# host computes for the same scene.
#include "world.h"

#include "sah.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <thread>

namespace rt {

namespace {

// One binned-SAH tree over `boxes`, built exactly like BvhNode's constructor
// (fat leaves <= 4, 16 bins per axis, traversal cost 0.5, in-place partition,
// median fallbacks). Nodes are emitted in pre-order into `out` with indices
// local to `out`; `idx` ends in leaf order.
struct SahBuilder {
    static const int kMaxLeaf = kSahMaxLeaf;
    const std::vector<Box>& boxes;
    std::vector<int>& idx;
    std::vector<NodeF>& out;
    int leaf_kind;
    int max_depth = 0;                // interior nodes on the longest root-leaf path

    SahBuilder(const std::vector<Box>& b, std::vector<int>& i, std::vector<NodeF>& o, int kind)
        : boxes(b), idx(i), out(o), leaf_kind(kind) {}

    static void set_node(NodeF& n, const Box& b, int a, int bb) {
        n.lo[0] = b.mn.x; n.lo[1] = b.mn.y; n.lo[2] = b.mn.z;
        n.hi[0] = b.mx.x; n.hi[1] = b.mx.y; n.hi[2] = b.mx.z;
        std::memcpy(&n.lo[3], &a, 4);
        std::memcpy(&n.hi[3], &bb, 4);
    }

    bool split(int start, int end, int& best_axis, int& mid) {   // BvhNode.cs:218-363
        return sah_split(start, end, idx.data(), [this](int item) { return boxes[item]; }, best_axis, mid);
    }

    // Returns the node index (local to `out`) and its box.
    int build(int start, int end, int depth, Box& box_out) {   // BvhNode.cs:91-152
        int me = (int)out.size();
        out.push_back(NodeF{});
        int span = end - start;
        if (span <= kMaxLeaf) {
            Box b = boxes[idx[start]];
            for (int i = 1; i < span; i++) b = surround(b, boxes[idx[start + i]]);
            set_node(out[me], b, ~start, span | (leaf_kind << 16));
            box_out = b;
            max_depth = std::max(max_depth, depth);
            return me;
        }
        int axis, mid;
        if (!split(start, end, axis, mid)) {
            axis = 0;
            mid = start + span / 2;
        }
        Box lb, rb;
        int l = build(start, mid, depth + 1, lb);
        int r = build(mid, end, depth + 1, rb);
        Box b = surround(lb, rb);
        set_node(out[me], b, l, r | (axis << 30));
        box_out = b;
        return me;
    }
};

void build_mesh(const float* tv, int64_t count, MeshBvh& mb) {
    std::vector<Box> boxes((size_t)count);
    for (int64_t t = 0; t < count; t++) {
        const float* p = tv + t * 9;
        boxes[t] = tri_box(v3(p[0], p[1], p[2]), v3(p[3], p[4], p[5]), v3(p[6], p[7], p[8]));
    }
    mb.nodes.clear();
    mb.order.resize((size_t)count);
    for (int64_t t = 0; t < count; t++) mb.order[t] = (int)t;
    Box box;
    if (count > 4) {   // Mesh.cs:93-96: BvhNode above 4 triangles
        SahBuilder sb(boxes, mb.order, mb.nodes, LEAF_TRIS);
        sb.build(0, (int)count, 0, box);
        mb.max_depth = sb.max_depth;
    } else {           // HittableList: flat scan, no box test
        box = boxes[0];
        for (int64_t t = 1; t < count; t++) box = surround(box, boxes[t]);
        NodeF n{};
        SahBuilder::set_node(n, box, ~0, (int)count | (LEAF_LIST << 16));
        mb.nodes.push_back(n);
        mb.max_depth = 0;
    }
    mb.box_mn = box.mn;
    mb.box_mx = box.mx;
}

float light_power(const Light& l, const Box& bounds) {
    if (l.type == LIGHT_GEOM_QUAD || l.type == LIGHT_GEOM_MESH || l.type == LIGHT_GEOM_SPHERE)   // GeometryLight.cs:116-120
        return kPi * l.rep_area * luminance(l.emission);
    if (l.type == LIGHT_AREA) return kPi * l.area * luminance(l.color) * l.intensity;   // AreaLight.cs:111
    if (l.type == LIGHT_SPHERE) return 4.0f * kPi * luminance(l.color) * l.intensity;   // SphereLight.cs:79-80
    if (l.type == LIGHT_ENV) {   // EnvironmentLight.ApproximatePower (:37-52): pi L times the mean cross-section
        V3 e = bounds.mx - bounds.mn;
        float cs = 0.5f * (e.x * e.y + e.y * e.z + e.x * e.z);
        return kPi * luminance(l.color) * cs;
    }
    V3 ext = bounds.mx - bounds.mn;                                                     // DirectionalLight.cs:82-88
    float radius = 0.5f * length(ext);
    float cs = kPi * radius * radius;
    return luminance(l.color) * l.intensity * cs;
}

// VNDF sampling (Materials/Microfacet.cs:100-124), host copy for the LUT build.
V3 vndf_host(V3 vl, float ax, float ay, float u1, float u2) {
    V3 vh = normalize(v3(ax * vl.x, ay * vl.y, vl.z));
    float lsq = vh.x * vh.x + vh.y * vh.y;
    V3 t1 = lsq > 0.0f ? v3(-vh.y, vh.x, 0.0f) / std::sqrt(lsq) : v3(1.0f, 0.0f, 0.0f);
    V3 t2 = cross(vh, t1);
    float r = std::sqrt(u1);
    float phi = 2.0f * kPi * u2;
    float a1 = r * std::cos(phi);
    float a2 = r * std::sin(phi);
    float s = 0.5f * (1.0f + vh.z);
    a2 = (1.0f - s) * std::sqrt(std::fmax(0.0f, 1.0f - a1 * a1)) + s * a2;
    V3 nh = a1 * t1 + a2 * t2 + std::sqrt(std::fmax(0.0f, 1.0f - a1 * a1 - a2 * a2)) * vh;
    return normalize(v3(ax * nh.x, ay * nh.y, std::fmax(0.0f, nh.z)));
}

float g1_aniso_host(V3 w, float ax, float ay) {   // Microfacet.cs:55-69
    float c2 = w.z * w.z;
    float lam;
    if (c2 < 1e-14f) {
        lam = 1e10f;
    } else {
        float num = (ax * w.x) * (ax * w.x) + (ay * w.y) * (ay * w.y);
        lam = 0.5f * (-1.0f + std::sqrt(1.0f + num / c2));
    }
    return 1.0f / (1.0f + lam);
}

float sample_eavg_host(const float* eavg, float alpha) {   // EnergyCompensationLut.cs:167-175
    alpha = clampf(alpha, 0.001f, 1.0f);
    float fal = alpha * 32.0f - 0.5f;
    int a0 = std::min(std::max((int)std::floor(fal), 0), 31);
    int a1 = std::min(a0 + 1, 31);
    float ta = clampf(fal - (float)a0, 0.0f, 1.0f);
    return eavg[a0] + (eavg[a1] - eavg[a0]) * ta;
}

}  // namespace

void build_energy_lut(float* e, float* eavg) {   // EnergyCompensationLut.cs:48-134
    const int kMu = 32, kAl = 32, kSpb = 2048;
    for (int ai = 0; ai < kAl; ai++) {
        float alpha = std::fmax(((float)ai + 0.5f) / (float)kAl, 0.001f);
        for (int mi = 0; mi < kMu; mi++) {
            float mu = ((float)mi + 0.5f) / (float)kMu;
            uint32_t seed = ((uint32_t)mi * 0x9E3779B9u) ^ ((uint32_t)ai * 0xB5297A4Du) ^ 0xC2B2AE3Du;
            float st = std::sqrt(std::fmax(0.0f, 1.0f - mu * mu));
            V3 V = v3(st, 0.0f, mu);
            double sum = 0.0;
            uint32_t s = seed == 0 ? 1u : seed;
            int hits = 0;
            for (int k = 0; k < kSpb; k++) {
                s ^= s << 13; s ^= s >> 17; s ^= s << 5;
                float u1 = (float)(s & 0x00FFFFFFu) / (float)0x01000000u;
                s ^= s << 13; s ^= s >> 17; s ^= s << 5;
                float u2 = (float)(s & 0x00FFFFFFu) / (float)0x01000000u;
                V3 H = vndf_host(V, alpha, alpha, u1, u2);
                float vdh = dot(V, H);
                V3 L = 2.0f * vdh * H - V;
                if (L.z <= 0.0f) continue;
                sum += (double)g1_aniso_host(L, alpha, alpha);
                hits++;
            }
            double m = sum / (double)kSpb;
            m = m < 0.0 ? 0.0 : (m > 1.0 ? 1.0 : m);
            e[mi * kAl + ai] = hits == 0 ? 0.0f : (float)m;
        }
        float avg = 0.0f;
        for (int mi = 0; mi < kMu; mi++) avg += 2.0f * e[mi * kAl + ai] * (((float)mi + 0.5f) / (float)kMu);
        eavg[ai] = clampf(avg / (float)kMu, 0.0f, 1.0f);
    }
}

Camera make_camera(const RtCameraDesc& c, float aspect) {   // Camera.cs:26-51
    V3 from = v3(c.look_from[0], c.look_from[1], c.look_from[2]);
    V3 at = v3(c.look_at[0], c.look_at[1], c.look_at[2]);
    V3 vup = v3(c.vup[0], c.vup[1], c.vup[2]);
    float theta = c.vfov_deg * kPi / 180.0f;
    float h = std::tan(theta / 2.0f);
    float vh = 2.0f * h;
    float vw = aspect * vh;
    V3 w = normalize(from - at);
    if (length_sq(cross(w, vup)) < 1e-8f) vup = std::fabs(w.x) < 0.9f ? v3(1, 0, 0) : v3(0, 0, 1);
    V3 u = normalize(cross(vup, w));
    V3 v = cross(w, u);
    float fd = c.focus_dist;
    Camera cam;
    cam.origin = from;
    cam.horizontal = fd * vw * u;
    cam.vertical = fd * vh * v;
    cam.llc = from - cam.horizontal / 2.0f - cam.vertical / 2.0f - fd * w;
    return cam;
}

Material make_material(const RtMaterialDesc& d, const float* eavg) {
    Material m{};
    m.type = d.type;
    m.thin_walled = d.thin_walled;
    m.has_tc = d.has_transmission_color;
    m.base = v3(d.base_color[0], d.base_color[1], d.base_color[2]);
    m.emission = m.base * std::fmax(d.intensity, 0.0f);   // Emissive: Albedo * Intensity
    // ShadingParams (DisneyBsdf.cs:237-291)
    m.metallic = clampf(d.metallic, 0.0f, 1.0f);
    m.roughness = clampf(d.roughness, 0.0f, 1.0f);
    m.specular = clampf(d.specular, 0.0f, 2.0f);
    m.specular_tint = clampf(d.specular_tint, 0.0f, 1.0f);
    m.sheen = clampf(d.sheen, 0.0f, 1.0f);
    m.sheen_tint = clampf(d.sheen_tint, 0.0f, 1.0f);
    m.sheen_roughness = clampf(d.sheen_roughness, 0.04f, 1.0f);
    m.clearcoat = clampf(d.clearcoat, 0.0f, 1.0f);
    m.clearcoat_gloss = clampf(d.clearcoat_gloss, 0.0f, 1.0f);
    m.spec_trans = clampf(d.spec_trans, 0.0f, 1.0f);
    m.ior = std::fmax(d.ior, 1.0001f);
    m.anisotropic = clampf(d.anisotropic, 0.0f, 1.0f);
    m.aniso_rotation = d.anisotropic_rotation - std::floor(d.anisotropic_rotation);
    m.diff_trans = clampf(d.diff_trans, 0.0f, 1.0f);
    m.alpha = std::fmax(m.roughness * m.roughness, 0.001f);
    float aspect = std::sqrt(1.0f - 0.9f * m.anisotropic);
    m.alpha_x = std::fmax(m.alpha / aspect, 0.001f);
    m.alpha_y = std::fmax(m.alpha * aspect, 0.001f);
    m.cc_alpha = d.coat_roughness >= 0.0f ? std::fmax(d.coat_roughness * d.coat_roughness, 0.001f)
                                          : lerpf(0.1f, 0.001f, m.clearcoat_gloss);
    float eta_c = std::fmax(d.coat_ior, 1.0001f);
    float r0 = (eta_c - 1.0f) / (eta_c + 1.0f);
    m.cc_f0 = r0 * r0;
    m.has_rotation = m.aniso_rotation != 0.0f;
    float ang = 2.0f * kPi * m.aniso_rotation;
    m.rot_cos = std::cos(ang);
    m.rot_sin = std::sin(ang);
    m.spec_trans_raw = d.spec_trans;
    m.ior_raw = std::fmax(d.ior, 1.0001f);
    // ComputeF0 (:1943-1959)
    V3 bc = m.base;
    {
        float r = (m.ior - 1.0f) / (m.ior + 1.0f);
        float f0d = r * r;
        float scaled = f0d * 2.0f * m.specular;
        float lum = luminance(bc);
        V3 tint = lum > 0.0f ? bc / lum : v3(1.0f);
        V3 diel = lerp(v3(scaled), scaled * tint, m.specular_tint);
        m.f0 = lerp(diel, bc, m.metallic);
        m.sheen_col = lerp(v3(1.0f), tint, m.sheen_tint);
    }
    // ResolveTransmission (:1016-1049)
    if (!d.has_transmission_color) {
        m.trans_tint = v3(std::sqrt(std::fmax(bc.x, 0.0f)), std::sqrt(std::fmax(bc.y, 0.0f)),
                          std::sqrt(std::fmax(bc.z, 0.0f)));
        m.trans_sigma = v3(0.0f);
    } else {
        V3 tc = v3(d.transmission_color[0], d.transmission_color[1], d.transmission_color[2]);
        float depth = std::fmax(d.transmission_depth, 0.0f);
        if (depth <= 0.0f) {
            m.trans_tint = tc;
            m.trans_sigma = v3(0.0f);
        } else {
            V3 c = v3(std::fmax(tc.x, 1e-6f), std::fmax(tc.y, 1e-6f), std::fmax(tc.z, 1e-6f));
            float inv = 1.0f / depth;
            m.trans_sigma = v3(-std::log(c.x) * inv, -std::log(c.y) * inv, -std::log(c.z) * inv);
            m.trans_tint = v3(1.0f);
        }
    }
    // ComputeLobeWeights (:1104-1139) and the probabilities (LobeWeights :1094-1101)
    float diffuse_all = (1.0f - m.metallic) * (1.0f - m.spec_trans);
    float diffuse_w = diffuse_all * (1.0f - m.diff_trans);
    float dt_w = diffuse_all * m.diff_trans;
    float spec_f0;
    if (m.metallic > 0.5f) {
        spec_f0 = luminance(bc);
    } else {
        float r = (m.ior - 1.0f) / (m.ior + 1.0f);
        spec_f0 = r * r * 2.0f * m.specular;
    }
    float spec_floor = 0.1f * (1.0f - m.spec_trans * 0.9f);
    float spec_w = std::fmax(spec_floor, lerpf(spec_f0, 1.0f, m.metallic));
    float trans_w = (1.0f - m.metallic) * m.spec_trans;
    float clear_w = m.clearcoat * 0.04f;
    float sheen_w = m.sheen * 0.25f * diffuse_all;
    m.alpha_iso = std::sqrt(m.alpha_x * m.alpha_y);
    m.e_avg = sample_eavg_host(eavg, m.alpha_iso);
    float ms_w = spec_w * (1.0f - m.e_avg);
    float sum = diffuse_w + spec_w + trans_w + clear_w + sheen_w + ms_w + dt_w;
    float total = sum < 1e-6f ? 1.0f : sum;
    m.p_d = diffuse_w / total;
    m.p_s = spec_w / total;
    m.p_t = trans_w / total;
    m.p_c = clear_w / total;
    m.p_sh = sheen_w / total;
    m.p_ms = ms_w / total;
    m.p_dt = dt_w / total;
    m.diffuse_w = (1.0f - m.metallic) * (1.0f - m.spec_trans) * (1.0f - m.diff_trans);
    m.diff_all = (1.0f - m.metallic) * (1.0f - m.spec_trans);
    return m;
}

namespace {

// Vertex normals of world triangle i, or nullptr when it is a flat Triangle
// (no normal array, or all nine floats zero).
const float* smooth_normals(const RtWorldDesc* w, int64_t i) {
    if (!w->tri_normals) return nullptr;
    const float* nn = w->tri_normals + i * 9;
    for (int k = 0; k < 9; k++)
        if (nn[k] != 0.0f) return nn;
    return nullptr;
}

// The SmoothTriangle constructor (Geometry/SmoothTriangle.cs:67-126) for world
// triangle i: normalised vertex normals and the tangent frame from the UV
// gradients, with the edge fallback for a degenerate mapping. Returns false
// for a flat triangle.
bool make_smooth(const RtWorldDesc* w, int64_t i, SmoothTri& st) {
    const float* nn = smooth_normals(w, i);
    if (!nn) return false;
    const float* p = w->tri_verts + i * 9;
    V3 v0 = v3(p[0], p[1], p[2]), v1 = v3(p[3], p[4], p[5]), v2 = v3(p[6], p[7], p[8]);
    st.n0 = normalize(v3(nn[0], nn[1], nn[2]));
    st.n1 = normalize(v3(nn[3], nn[4], nn[5]));
    st.n2 = normalize(v3(nn[6], nn[7], nn[8]));
    const float def_uv[6] = {0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 1.0f};   // the no-UV constructor (:133-139)
    const float* uv = w->tri_uvs ? w->tri_uvs + i * 6 : def_uv;
    for (int k = 0; k < 6; k++) st.uv[k] = uv[k];
    V3 e1 = v1 - v0, e2 = v2 - v0;
    float d1x = uv[2] - uv[0], d1y = uv[3] - uv[1];
    float d2x = uv[4] - uv[0], d2y = uv[5] - uv[1];
    float det = d1x * d2y - d2x * d1y;
    bool uv_frame = false;
    if (std::fabs(det) > 1e-8f) {
        float inv = 1.0f / det;
        V3 t = inv * (d2y * e1 - d1y * e2);
        V3 b = inv * ((-d2x) * e1 + d1x * e2);
        float tl = length(t), bl = length(b);
        if (tl > 1e-8f && bl > 1e-8f) {
            st.tangent = t / tl;
            st.bitangent = b / bl;
            uv_frame = true;
        }
    }
    if (!uv_frame) {
        st.tangent = normalize(e1);
        st.bitangent = normalize(e2);
    }
    st.v1 = v1;
    st.v2 = v2;
    return true;
}

}  // namespace

int build_world(const RtWorldDesc* w, HostScene& sc, std::string& err, const BuildOptions& opt) {
    if (!w || w->num_materials <= 0 || w->num_entities <= 0 || !w->materials || !w->entities) {
        err = "world needs at least one material and one entity";
        return RT_ERR_INVALID_ARG;
    }
    sc.lut_e.resize(1024);
    sc.lut_eavg.resize(32);
    build_energy_lut(sc.lut_e.data(), sc.lut_eavg.data());
    for (int i = 0; i < w->num_materials; i++) {
        const RtMaterialDesc& d = w->materials[i];
        if (d.type != RT_MAT_DISNEY && d.type != RT_MAT_EMISSIVE) {
            err = "material " + std::to_string(i) + ": only Disney and Emissive are on the GPU path";
            return RT_ERR_UNSUPPORTED;
        }
        if (d.type == RT_MAT_DISNEY && d.thin_film_thickness > 0.0f) {
            err = "material " + std::to_string(i) + ": thin-film iridescence is outside the GPU path";
            return RT_ERR_UNSUPPORTED;
        }
        sc.materials.push_back(make_material(d, sc.lut_eavg.data()));
    }
    const int ne = w->num_entities;
    // --- mesh BVHs (independent; built in parallel like BvhNode's Parallel.Invoke)
    std::vector<MeshBvh> mb((size_t)ne);
    std::vector<int> mesh_ids;
    for (int e = 0; e < ne; e++) {
        const RtEntityDesc& d = w->entities[e];
        if (d.material < 0 || d.material >= w->num_materials) {
            err = "entity " + std::to_string(e) + ": material index out of range";
            return RT_ERR_INVALID_ARG;
        }
        if (d.kind == RT_ENT_MESH) {
            if (d.count <= 0 || d.first < 0 || d.first + d.count > w->num_tris || !w->tri_verts) {
                err = "entity " + std::to_string(e) + ": triangle range out of bounds";
                return RT_ERR_INVALID_ARG;
            }
            for (int64_t t = d.first; t < d.first + d.count; t++) {
                const float* nn = smooth_normals(w, t);
                if (!nn) continue;
                for (int k = 0; k < 3; k++) {
                    V3 n = v3(nn[3 * k], nn[3 * k + 1], nn[3 * k + 2]);
                    if (!std::isfinite(n.x) || !std::isfinite(n.y) || !std::isfinite(n.z) || length_sq(n) == 0.0f) {
                        err = "triangle " + std::to_string(t) + ": a vertex normal is zero or not finite";
                        return RT_ERR_INVALID_ARG;
                    }
                }
            }
            mesh_ids.push_back(e);
        } else if (d.kind != RT_ENT_QUAD && d.kind != RT_ENT_SPHERE) {
            err = "entity " + std::to_string(e) + ": unsupported kind";
            return RT_ERR_UNSUPPORTED;
        }
    }
    {
        auto t0 = std::chrono::steady_clock::now();
        // Meshes of more than 4 triangles get a BvhNode tree; the device build
        // takes those when asked, the host the rest (and all on a device error).
        std::vector<int> host_ids;
        std::vector<int> dev_ids;
        std::vector<int64_t> dev_first, dev_count;
        int64_t dev_tris = 0;
        for (int e : mesh_ids) {
            const RtEntityDesc& d = w->entities[e];
            if (opt.device_builder && d.count > 4) {
                dev_ids.push_back(e);
                dev_first.push_back(d.first);
                dev_count.push_back(d.count);
                dev_tris += d.count;
            } else {
                host_ids.push_back(e);
            }
        }
        sc.bvh_on_device = 0;
        if (!dev_ids.empty() && dev_tris >= opt.device_min_tris) {
            std::vector<MeshBvh> got(dev_ids.size());
            std::string derr;
            if (opt.device_builder(w->tri_verts, dev_first.data(), dev_count.data(), (int)dev_ids.size(), got.data(),
                                   derr) == RT_OK) {
                for (size_t i = 0; i < dev_ids.size(); i++) mb[dev_ids[i]] = std::move(got[i]);
                sc.bvh_on_device = 1;
            }
        }
        if (!sc.bvh_on_device) host_ids = mesh_ids;
        std::atomic<size_t> next{0};
        unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), (unsigned)host_ids.size()));
        auto work = [&]() {
            for (;;) {
                size_t k = next.fetch_add(1);
                if (k >= host_ids.size()) break;
                int e = host_ids[k];
                const RtEntityDesc& d = w->entities[e];
                build_mesh(w->tri_verts + d.first * 9, d.count, mb[e]);
            }
        };
        std::vector<std::thread> pool;
        for (unsigned t = 1; t < nt; t++) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
        sc.bvh_build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    // --- entities, quads, spheres and their boxes (world objects in YAML order)
    std::vector<Box> ent_box((size_t)ne);
    int max_blas_depth = 0;
    for (int e = 0; e < ne; e++) {
        const RtEntityDesc& d = w->entities[e];
        Entity en{d.kind, d.material, (d.flags & RT_ENT_FLAG_BACKFACE_CULLED) ? ENT_BACKFACE_CULLED : 0, -1};
        if (d.kind == RT_ENT_QUAD) {   // Quad.cs:26-40, BoundingBox :113-120
            QuadData q{};
            q.q = v3(d.p[0], d.p[1], d.p[2]);
            q.u = v3(d.p[3], d.p[4], d.p[5]);
            q.v = v3(d.p[6], d.p[7], d.p[8]);
            V3 n = cross(q.u, q.v);
            q.normal = normalize(n);
            q.d = dot(q.normal, q.q);
            q.w = n / dot(n, n);
            q.tangent = normalize(q.u);
            q.bitangent = normalize(q.v);
            q.area = length(n);
            Box b{q.q, q.q + q.u + q.v};
            ent_box[e] = {vmin(b.mn, vmin(q.q + q.u, q.q + q.v)) - v3(0.0001f),
                          vmax(b.mx, vmax(q.q + q.u, q.q + q.v)) + v3(0.0001f)};
            en.index = (int)sc.quads.size();
            sc.quads.push_back(q);
        } else if (d.kind == RT_ENT_SPHERE) {   // Sphere.cs:271-275
            SphereData s{v3(d.p[0], d.p[1], d.p[2]), d.p[3]};
            V3 r = v3(s.r);
            ent_box[e] = {s.c - r, s.c + r};
            en.index = (int)sc.spheres.size();
            sc.spheres.push_back(s);
        } else {
            ent_box[e] = {mb[e].box_mn, mb[e].box_mx};
            max_blas_depth = std::max(max_blas_depth, mb[e].max_depth);
        }
        sc.entities.push_back(en);
    }
    for (int e = 0; e < ne; e++) {
        sc.ent_box.push_back(float4{ent_box[e].mn.x, ent_box[e].mn.y, ent_box[e].mn.z, 0.0f});
        sc.ent_box.push_back(float4{ent_box[e].mx.x, ent_box[e].mx.y, ent_box[e].mx.z, 0.0f});
    }
    // --- top level (SceneLoader.cs:460-485): BVH above 4 objects, else a flat list
    sc.top_is_bvh = ne > 4;
    int top_depth = 0;
    if (sc.top_is_bvh) {
        std::vector<int> order((size_t)ne);
        for (int e = 0; e < ne; e++) order[e] = e;
        SahBuilder sb(ent_box, order, sc.nodes, LEAF_ENTS);
        Box root_box;
        sc.top_root = sb.build(0, ne, 0, root_box);
        top_depth = sb.max_depth;
        sc.top_items = order;
    } else {
        sc.top_root = -1;
        sc.top_items.resize((size_t)ne);
        for (int e = 0; e < ne; e++) sc.top_items[e] = e;
    }
    // --- append mesh BVHs, relocating node and triangle indices
    for (int e : mesh_ids) {
        MeshBvh& m = mb[e];
        int node_base = (int)sc.nodes.size();
        int tri_base = (int)sc.tri_entity.size();
        for (NodeF n : m.nodes) {
            int a, b;
            std::memcpy(&a, &n.lo[3], 4);
            std::memcpy(&b, &n.hi[3], 4);
            if (a >= 0) {
                a += node_base;
                int r = b & 0x3FFFFFFF;
                b = (b & ~0x3FFFFFFF) | (r + node_base);
            } else {
                a = ~(~a + tri_base);
            }
            std::memcpy(&n.lo[3], &a, 4);
            std::memcpy(&n.hi[3], &b, 4);
            sc.nodes.push_back(n);
        }
        sc.entities[e].index = node_base;
        const RtEntityDesc& d = w->entities[e];
        for (int local : m.order) {
            const float* p = w->tri_verts + (d.first + local) * 9;
            V3 v0 = v3(p[0], p[1], p[2]), v1 = v3(p[3], p[4], p[5]), v2 = v3(p[6], p[7], p[8]);
            V3 e1 = v1 - v0, e2 = v2 - v0;   // Triangle.cs:35-47
            V3 cr = cross(e1, e2);
            float cl = length(cr);
            V3 n = cl > 0.0f ? cr / cl : v3(0.0f, 1.0f, 0.0f);
            sc.tris.push_back(float4{v0.x, v0.y, v0.z, n.x});
            sc.tris.push_back(float4{e1.x, e1.y, e1.z, n.y});
            sc.tris.push_back(float4{e2.x, e2.y, e2.z, n.z});
            sc.tri_entity.push_back(e);
            sc.tri_local.push_back(local);
            SmoothTri st;
            if (make_smooth(w, d.first + local, st)) {
                sc.tri_smooth.push_back((int)sc.smooth.size());
                sc.smooth.push_back(st);
            } else {
                sc.tri_smooth.push_back(-1);
            }
        }
    }
    if (sc.smooth.empty()) sc.tri_smooth.clear();
    // Worst-case traversal stack: one far child per interior level of each
    // tree, plus up to 4 pending entities of a top-level fat leaf.
    sc.max_stack = top_depth + 4 + max_blas_depth + 1;
    // --- child-box traversal layout
    {
        std::vector<int> cidx(sc.nodes.size(), -1);
        int n_int = 0;
        for (size_t i = 0; i < sc.nodes.size(); i++) {
            int a;
            std::memcpy(&a, &sc.nodes[i].lo[3], 4);
            if (a >= 0) cidx[i] = n_int++;
        }
        auto code_of = [&](int node) {
            int a, b;
            std::memcpy(&a, &sc.nodes[node].lo[3], 4);
            std::memcpy(&b, &sc.nodes[node].hi[3], 4);
            if (a >= 0) return cidx[node];
            return leaf_code(~a, b >> 16, b & 0xFFFF);
        };
        sc.cnodes.resize((size_t)n_int * 4);
        for (size_t i = 0; i < sc.nodes.size(); i++) {
            if (cidx[i] < 0) continue;
            int a, b;
            std::memcpy(&a, &sc.nodes[i].lo[3], 4);
            std::memcpy(&b, &sc.nodes[i].hi[3], 4);
            int l = a, r = b & 0x3FFFFFFF, axis = (int)((unsigned)b >> 30);
            const NodeF& L = sc.nodes[l];
            const NodeF& R = sc.nodes[r];
            int lc = code_of(l), rc = code_of(r);
            float lcf, rcf, axf, zero = 0.0f;
            std::memcpy(&lcf, &lc, 4);
            std::memcpy(&rcf, &rc, 4);
            std::memcpy(&axf, &axis, 4);
            float4* c = &sc.cnodes[(size_t)cidx[i] * 4];
            c[0] = float4{L.lo[0], L.lo[1], L.lo[2], lcf};
            c[1] = float4{L.hi[0], L.hi[1], L.hi[2], rcf};
            c[2] = float4{R.lo[0], R.lo[1], R.lo[2], axf};
            c[3] = float4{R.hi[0], R.hi[1], R.hi[2], zero};
        }
        if (sc.top_is_bvh) sc.top_root_code = code_of(sc.top_root);
        // --- four-wide layout: one record per interior node at even depth of
        // each tree, holding its grandchildren (see SceneView).
        {
            auto kids = [&](int node, int& l, int& r, int& axis) {
                int a, b;
                std::memcpy(&a, &sc.nodes[node].lo[3], 4);
                std::memcpy(&b, &sc.nodes[node].hi[3], 4);
                if (a < 0) return false;
                l = a;
                r = b & 0x3FFFFFFF;
                axis = (int)((unsigned)b >> 30);
                return true;
            };
            std::vector<int> ridx(sc.nodes.size(), -1), rnode;
            std::vector<int> work;
            if (sc.top_is_bvh) work.push_back(sc.top_root);
            for (int e : mesh_ids) work.push_back(sc.entities[e].index);
            while (!work.empty()) {
                int n = work.back();
                work.pop_back();
                int l = 0, r = 0, ax = 0;
                if (ridx[n] >= 0 || !kids(n, l, r, ax)) continue;
                ridx[n] = (int)rnode.size();
                rnode.push_back(n);
                for (int c : {l, r}) {
                    int cl = 0, cr = 0, cax = 0;
                    if (kids(c, cl, cr, cax)) {
                        work.push_back(cl);
                        work.push_back(cr);
                    }
                }
            }
            auto code4 = [&](int node) {
                int l = 0, r = 0, ax = 0;
                return kids(node, l, r, ax) ? ridx[node] : code_of(node);
            };
            sc.cnodes4.assign(rnode.size() * 8, float4{0.0f, 0.0f, 0.0f, 0.0f});
            const float inf = std::numeric_limits<float>::infinity();
            for (size_t k = 0; k < rnode.size(); k++) {
                int l = 0, r = 0, ax = 0;
                kids(rnode[k], l, r, ax);
                int slot_node[4] = {-1, -1, -1, -1};
                int axes[3] = {ax, 0, 0};
                for (int side = 0; side < 2; side++) {
                    int c = side == 0 ? l : r;
                    int cl = 0, cr = 0, cax = 0;
                    if (kids(c, cl, cr, cax)) {
                        slot_node[2 * side] = cl;
                        slot_node[2 * side + 1] = cr;
                        axes[1 + side] = cax;
                    } else {
                        slot_node[2 * side] = c;
                    }
                }
                float lo[3][4], hi[3][4];
                int codes[4];
                for (int j = 0; j < 4; j++) {
                    int g = slot_node[j];
                    for (int a = 0; a < 3; a++) {
                        lo[a][j] = g >= 0 ? sc.nodes[g].lo[a] : inf;
                        hi[a][j] = g >= 0 ? sc.nodes[g].hi[a] : inf;
                    }
                    codes[j] = g >= 0 ? code4(g) : INT_MIN;
                }
                float4* q = &sc.cnodes4[k * 8];
                for (int a = 0; a < 3; a++) {
                    q[a] = float4{lo[a][0], lo[a][1], lo[a][2], lo[a][3]};
                    q[3 + a] = float4{hi[a][0], hi[a][1], hi[a][2], hi[a][3]};
                }
                float cf[4], af[3];
                std::memcpy(cf, codes, sizeof(cf));
                std::memcpy(af, axes, sizeof(af));
                q[6] = float4{cf[0], cf[1], cf[2], cf[3]};
                q[7] = float4{af[0], af[1], af[2], 0.0f};
            }
            sc.mesh_root4.assign((size_t)ne, 0);
            for (int e : mesh_ids) sc.mesh_root4[(size_t)e] = code4(sc.entities[e].index);
            if (sc.top_is_bvh) sc.top_root4 = code4(sc.top_root);
            // a record pushes at most three slots; it spans two binary levels
            sc.max_stack4 = 3 * ((top_depth + 1) / 2) + 4 + 3 * ((max_blas_depth + 1) / 2) + 1;
        }
        for (int e : mesh_ids) sc.entities[e].index = code_of(sc.entities[e].index);
    }
    // --- explicit lights (SceneLoader.cs:446-458)
    for (int i = 0; i < w->num_lights; i++) {
        const RtLightDesc& d = w->lights[i];
        Light l{};
        l.quad = -1;
        l.mesh_root = -1;
        l.mesh_entity = -1;
        l.emissive_material = -1;
        l.color = v3(d.color[0], d.color[1], d.color[2]);
        l.intensity = d.intensity;
        if (d.type == RT_LIGHT_AREA) {   // AreaLight.cs:67-87
            l.type = LIGHT_AREA;
            l.corner = v3(d.corner[0], d.corner[1], d.corner[2]);
            l.u = v3(d.u[0], d.u[1], d.u[2]);
            l.v = v3(d.v[0], d.v[1], d.v[2]);
            l.shadow_samples = std::max(1, d.shadow_samples);
            l.soft_radius = std::fmax(0.0f, d.soft_radius);
            V3 cr = cross(l.u, l.v);
            l.area = length(cr);
            l.normal = cr / l.area;
            l.sqrt_samples = (int)std::ceil(std::sqrt((float)l.shadow_samples));
            l.inv_sqrt = 1.0f / (float)l.sqrt_samples;
            l.is_delta = 0;
            l.emissive_material = d.proxy_material;
            if (d.proxy_material >= w->num_materials) {
                err = "area light proxy material out of range";
                return RT_ERR_INVALID_ARG;
            }
        } else if (d.type == RT_LIGHT_DIRECTIONAL) {   // DirectionalLight.cs:55-72
            l.type = LIGHT_DIRECTIONAL;
            l.direction = normalize(v3(d.direction[0], d.direction[1], d.direction[2]));
            l.angular_radius = std::fmax(0.0f, d.angular_radius_deg);
            bool disc = l.angular_radius > 0.0f;
            float rad = l.angular_radius * kPi / 180.0f;
            l.cos_angular = disc ? std::cos(rad) : 1.0f;
            l.solid_angle = disc ? 2.0f * kPi * (1.0f - l.cos_angular) : 0.0f;
            l.shadow_samples = d.shadow_samples > 0 ? d.shadow_samples : (disc ? 4 : 1);
            l.sqrt_samples = (int)std::ceil(std::sqrt((float)l.shadow_samples));
            l.inv_sqrt = 1.0f / (float)l.sqrt_samples;
            l.is_delta = disc ? 0 : 1;
        } else if (d.type == RT_LIGHT_SPHERE) {   // SphereLight.cs:54-68
            l.type = LIGHT_SPHERE;
            l.center = v3(d.center[0], d.center[1], d.center[2]);
            l.radius = std::fmax(d.radius, kEps);
            l.shadow_samples = d.shadow_samples > 0 ? d.shadow_samples : 4;
            l.sqrt_samples = (int)std::ceil(std::sqrt((float)l.shadow_samples));
            l.inv_sqrt = 1.0f / (float)l.sqrt_samples;
            l.is_delta = 0;
            l.emissive_material = d.proxy_material;
            if (d.proxy_material >= w->num_materials) {
                err = "sphere light proxy material out of range";
                return RT_ERR_INVALID_ARG;
            }
        } else {
            err = "light " + std::to_string(i) + ": unsupported type";
            return RT_ERR_UNSUPPORTED;
        }
        sc.lights.push_back(l);
    }
    // --- geometry lights from emissive, non-proxy entities (SceneLoader.cs:805-887)
    int gls = std::max(1, w->geometry_light_samples);
    for (int e = 0; e < ne; e++) {
        const RtEntityDesc& d = w->entities[e];
        const Material& m = sc.materials[d.material];
        if (m.type != RT_MAT_EMISSIVE || w->materials[d.material].is_light_proxy) continue;
        Light l{};
        l.quad = -1;
        l.mesh_root = -1;
        l.mesh_entity = -1;
        l.shadow_samples = gls;
        l.sqrt_samples = (int)std::ceil(std::sqrt((float)gls));
        l.inv_sqrt = 1.0f / (float)l.sqrt_samples;
        l.is_delta = 0;
        l.emissive_material = d.material;
        l.emission = m.emission;
        if (d.kind == RT_ENT_QUAD) {
            l.type = LIGHT_GEOM_QUAD;
            l.quad = sc.entities[e].index;
            l.rep_area = sc.quads[l.quad].area;
        } else if (d.kind == RT_ENT_MESH) {
            l.type = LIGHT_GEOM_MESH;
            l.mesh_root = sc.entities[e].index;   // child code (after the layout pass)
            l.mesh_entity = e;
            l.mesh_first = (int)sc.light_tris.size();
            l.mesh_count = (int)d.count;
            float sum = 0.0f;
            for (int64_t t = 0; t < d.count; t++) {   // Mesh.cs:98-107, ComputeTriangleArea :195-203
                const float* p = w->tri_verts + (d.first + t) * 9;
                V3 v0 = v3(p[0], p[1], p[2]), v1 = v3(p[3], p[4], p[5]), v2 = v3(p[6], p[7], p[8]);
                LightTri lt{};
                lt.v0 = v0;
                lt.e1 = v1 - v0;
                lt.e2 = v2 - v0;
                V3 cr = cross(lt.e1, lt.e2);
                float cl = length(cr);
                lt.normal = cl > 0.0f ? cr / cl : v3(0.0f, 1.0f, 0.0f);
                float a = 0.5f * length(cross(v1 - v0, v2 - v0));
                sum += a;
                lt.cum_area = sum;
                lt.smooth = -1;
                SmoothTri st;
                if (make_smooth(w, d.first + t, st)) {   // SmoothTriangle.SampleAt (:219-230)
                    lt.smooth = (int)sc.smooth.size();
                    sc.smooth.push_back(st);
                }
                sc.light_tris.push_back(lt);
            }
            l.rep_area = sum;
        } else {   // a sphere: GeometryLight's cone sampling (ISolidAngleSamplable, GeometryLight.cs:94)
            l.type = LIGHT_GEOM_SPHERE;
            const SphereData& sp = sc.spheres[sc.entities[e].index];
            l.center = sp.c;
            l.radius = sp.r;
            l.rep_area = 4.0f * kPi * sp.r * sp.r;   // Sphere.SurfaceArea (Sphere.cs:78)
        }
        sc.lights.push_back(l);
    }
    // --- the flat sky and its EnvironmentLight (SceneLoader.cs:524-528; FlatSky.cs)
    sc.sky = v3(w->sky_color[0], w->sky_color[1], w->sky_color[2]);
    sc.sky_on = sc.sky.x != 0.0f || sc.sky.y != 0.0f || sc.sky.z != 0.0f;
    sc.env_light = -1;
    if (luminance(sc.sky) > 1e-6f) {   // FlatSky.HasImportanceSampling
        Light l{};
        l.type = LIGHT_ENV;
        l.quad = -1;
        l.mesh_root = -1;
        l.mesh_entity = -1;
        l.emissive_material = -1;
        l.color = sc.sky;
        l.shadow_samples = std::max(1, w->sky_light_samples);
        l.sqrt_samples = 1;
        l.inv_sqrt = 1.0f;
        l.is_delta = 0;
        sc.env_light = (int)sc.lights.size();
        sc.lights.push_back(l);
    }
    // --- emitter -> light map (Renderer.cs:409-425)
    sc.emitter_light.assign((size_t)w->num_materials, -1);
    for (size_t i = 0; i < sc.lights.size(); i++) {
        int t = sc.lights[i].type;
        if (t == LIGHT_GEOM_QUAD || t == LIGHT_GEOM_MESH || t == LIGHT_GEOM_SPHERE)
            sc.emitter_light[sc.lights[i].emissive_material] = (int)i;
    }
    for (size_t i = 0; i < sc.lights.size(); i++) {   // then every light's proxy, in list order
        int t = sc.lights[i].type;
        if ((t == LIGHT_AREA || t == LIGHT_SPHERE) && sc.lights[i].emissive_material >= 0)
            sc.emitter_light[sc.lights[i].emissive_material] = (int)i;
    }
    // --- RR classifier (Renderer.cs:361-378; ComputeFiniteSceneBounds :475-500)
    Box bounds;
    {
        bool any = false;
        Box acc = empty_box();
        if (sc.top_is_bvh) {
            Box b{v3(sc.nodes[sc.top_root].lo[0], sc.nodes[sc.top_root].lo[1], sc.nodes[sc.top_root].lo[2]),
                  v3(sc.nodes[sc.top_root].hi[0], sc.nodes[sc.top_root].hi[1], sc.nodes[sc.top_root].hi[2])};
            V3 dd = b.mx - b.mn;
            if (dd.x < 1.0e5f && dd.y < 1.0e5f && dd.z < 1.0e5f) {
                acc = b;
                any = true;
            }
        } else {
            for (int e = 0; e < ne; e++) {
                V3 dd = ent_box[e].mx - ent_box[e].mn;
                if (dd.x < 1.0e5f && dd.y < 1.0e5f && dd.z < 1.0e5f) {
                    acc = any ? surround(acc, ent_box[e]) : ent_box[e];
                    any = true;
                }
            }
        }
        if (any) {
            bounds = acc;
        } else {
            Box raw = ent_box[0];
            for (int e = 1; e < ne; e++) raw = surround(raw, ent_box[e]);
            bounds = {vmax(raw.mn, v3(-1.0e3f)), vmin(raw.mx, v3(1.0e3f))};
        }
    }
    // LightDistribution (Lights/LightDistribution.cs:30-102) over these bounds:
    // the power CDF (uniform when every power is zero), then the uniform one
    {
        size_t n = sc.lights.size();
        sc.pick_cdf.assign(2 * n, 0.0f);
        sc.pick_pdf.assign(2 * n, 0.0f);
        for (int mode = 0; mode < 2 && n > 0; mode++) {
            std::vector<float> power(n, 0.0f);
            float sum = 0.0f;
            if (mode == 0)
                for (size_t i = 0; i < n; i++) {
                    power[i] = std::fmax(0.0f, light_power(sc.lights[i], bounds));
                    sum += power[i];
                }
            float* cdf = sc.pick_cdf.data() + mode * n;
            float* pdf = sc.pick_pdf.data() + mode * n;
            float cum = 0.0f;
            if (sum > 0.0f) {
                float inv = 1.0f / sum;
                for (size_t i = 0; i < n; i++) {
                    pdf[i] = power[i] * inv;
                    cum += pdf[i];
                    cdf[i] = cum;
                }
            } else {
                float u = 1.0f / (float)n;
                for (size_t i = 0; i < n; i++) {
                    pdf[i] = u;
                    cum += u;
                    cdf[i] = cum;
                }
            }
            cdf[n - 1] = 1.0f;
        }
    }
    float flux = 0.0f;
    for (const Light& l : sc.lights) flux += light_power(l, bounds);
    V3 ext = bounds.mx - bounds.mn;
    float radius = std::fmax(0.5f * length(ext), 1e-3f);
    float area = 4.0f * kPi * radius * radius;
    sc.mean_irradiance = flux / area;
    bool indirect = sc.mean_irradiance < 0.5f;
    sc.rr_min_bounces = indirect ? 6 : 3;
    sc.rr_min_survival = indirect ? 0.40f : 0.10f;
    // --- medium
    if (w->medium.enabled) {
        sc.has_medium = 1;
        sc.sigma_a = vmax(v3(w->medium.sigma_a[0], w->medium.sigma_a[1], w->medium.sigma_a[2]), v3(0.0f));
        sc.sigma_s = vmax(v3(w->medium.sigma_s[0], w->medium.sigma_s[1], w->medium.sigma_s[2]), v3(0.0f));
        sc.sigma_t = sc.sigma_a + sc.sigma_s;
        sc.hg_g = std::fmax(-0.999f, std::fmin(0.999f, w->medium.g));
    }
    sc.camera = w->camera;
    return RT_OK;
}

}  // namespace rt
