// ORACLE — test infrastructure only.
//
// A scalar C++17 restatement of fiorenzobrioni/3d-ray's per-pixel bounce loop
// (C# / .NET 10, which cannot be compiled here: no dotnet/mono/csc). It is the
// CHECKER for the CUDA path: only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py may load it. The product path never links it.
//
// Parity status: the reference's own tests hold properties, not golden
// numbers; this restatement is pinned against those properties (BVH vs linear
// list, Sobol stratification/range, Disney reciprocity / pdf normalisation /
// Sample-vs-Evaluate consistency / furnace) in tests/. Bit-level agreement
// with the real C# at the System.Numerics.Vector3 / MathF boundary is
// UNPINNED: no dotnet is available to run it. Vector3 reductions are restated
// as (x*x + y*y) + z*z, Normalize as v / Length(v), MathF transcendentals call
// glibc (what .NET's MathF forwards to on Linux). Built with
// -ffp-contract=off and no fast-math, since C# never contracts to FMA.
//
// Each function cites the reference file:line it restates (paths relative to
// src/RayTracer/ in the reference repository).

#include <algorithm>
#include <cstdio>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "../include/rt3d.h"

namespace oracle {

// ---------------------------------------------------------------------------
// System.Numerics.Vector3 restated
// ---------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};
static inline V3 v3(float a) { return {a, a, a}; }
static inline V3 v3(float a, float b, float c) { return {a, b, c}; }
static inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
static inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
static inline V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
static inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
static inline V3& operator*=(V3& a, V3 b) { a = a * b; return a; }
static inline V3& operator*=(V3& a, float s) { a = a * s; return a; }
static inline V3& operator/=(V3& a, float s) { a = a / s; return a; }
static inline bool operator==(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline float length_sq(V3 a) { return dot(a, a); }
static inline float length(V3 a) { return std::sqrt(length_sq(a)); }
static inline V3 normalize(V3 a) { return a / length(a); }
static inline V3 vmin(V3 a, V3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
static inline V3 vmax(V3 a, V3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
static inline V3 lerp(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
static inline float get_axis(V3 v, int axis) { return axis == 0 ? v.x : axis == 1 ? v.y : v.z; }
static inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float lerpf(float a, float b, float t) { return a + (b - a) * t; }   // DisneyBsdf.cs:2005

static const float kPi = 3.14159265358979323846f;   // MathF.PI
static const float kEps = 1e-4f;                     // MathUtils.Epsilon (Core/MathUtils.cs:22)
static const float kInf = 3.40282347e+38f;           // MathUtils.Infinity = float.MaxValue
static const float kInv4Pi = 0.0795774715f;          // MathUtils.Inv4Pi

static inline float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }  // MathUtils.cs:213
static inline bool near_zero(V3 v) {   // MathUtils.cs:203-207
    const float s = 1e-8f;
    return std::fabs(v.x) < s && std::fabs(v.y) < s && std::fabs(v.z) < s;
}
static inline V3 offset_origin(V3 p, V3 n) { return p + n * kEps; }   // MathUtils.cs:221
static inline V3 reflect(V3 v, V3 n) { return v - 2.0f * dot(v, n) * n; }   // MathUtils.cs:157
static inline V3 refract(V3 uv, V3 n, float eta) {   // MathUtils.cs:160-166
    float cos_t = std::fmin(dot(-uv, n), 1.0f);
    V3 perp = eta * (uv + cos_t * n);
    V3 par = -std::sqrt(std::fabs(1.0f - length_sq(perp))) * n;
    return perp + par;
}
static inline float fresnel_dielectric(float cos_i, float eta) {   // MathUtils.cs:191-201
    cos_i = clampf(cos_i, 0.0f, 1.0f);
    float sin2_i = std::fmax(0.0f, 1.0f - cos_i * cos_i);
    float sin2_t = eta * eta * sin2_i;
    if (sin2_t >= 1.0f) return 1.0f;
    float cos_t = std::sqrt(1.0f - sin2_t);
    float r_parl = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    float r_perp = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    return 0.5f * (r_parl * r_parl + r_perp * r_perp);
}
static inline float shadow_terminator(V3 ng, V3 ns, V3 w) {   // MathUtils.cs:44-61
    float ng_w = dot(ng, w);
    if (ng_w <= 0.0f) return 0.0f;
    float ns_w = dot(ns, w);
    if (ns_w <= 0.0f) return 0.0f;
    float ng_ns = dot(ng, ns);
    if (ng_ns >= 0.9999f) return 1.0f;
    float g = ng_w / (ns_w * std::fmax(ng_ns, 1e-4f));
    if (g >= 1.0f) return 1.0f;
    if (g <= 0.0f) return 0.0f;
    float g2 = g * g;
    return (-g2 * g) + g2 + g;
}

// ---------------------------------------------------------------------------
// Owen-scrambled Sobol (Core/Sampling/OwenSobol.cs) and the per-thread
// dimension counter (Core/Sampling/Sampler.cs)
// ---------------------------------------------------------------------------
static const uint32_t kDim1Dirs[32] = {   // OwenSobol.cs:132-142 (x^2+x+1, m1=1)
    0x80000000u, 0xc0000000u, 0xa0000000u, 0xf0000000u, 0x88000000u, 0xcc000000u, 0xaa000000u, 0xff000000u,
    0x80800000u, 0xc0c00000u, 0xa0a00000u, 0xf0f00000u, 0x88880000u, 0xcccc0000u, 0xaaaa0000u, 0xffff0000u,
    0x80008000u, 0xc000c000u, 0xa000a000u, 0xf000f000u, 0x88008800u, 0xcc00cc00u, 0xaa00aa00u, 0xff00ff00u,
    0x80808080u, 0xc0c0c0c0u, 0xa0a0a0a0u, 0xf0f0f0f0u, 0x88888888u, 0xccccccccu, 0xaaaaaaaau, 0xffffffffu,
};
static inline uint32_t reverse_bits(uint32_t v) {   // OwenSobol.cs:194-202
    v = ((v & 0xaaaaaaaau) >> 1) | ((v & 0x55555555u) << 1);
    v = ((v & 0xccccccccu) >> 2) | ((v & 0x33333333u) << 2);
    v = ((v & 0xf0f0f0f0u) >> 4) | ((v & 0x0f0f0f0fu) << 4);
    v = ((v & 0xff00ff00u) >> 8) | ((v & 0x00ff00ffu) << 8);
    return (v >> 16) | (v << 16);
}
static inline uint32_t lk_permute(uint32_t v, uint32_t seed) {   // OwenSobol.cs:167-175
    v += seed;
    v ^= v * 0x6c50b47cu;
    v ^= v * 0xb82f1e52u;
    v ^= v * 0xc7afe638u;
    v ^= v * 0x8d22f6e6u;
    return v;
}
static inline uint32_t hash_u32(uint32_t x) {   // OwenSobol.cs:184-192
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
static inline uint32_t owen_scramble(uint32_t v, uint32_t seed) {   // OwenSobol.cs:151-157
    return reverse_bits(lk_permute(reverse_bits(v), seed));
}
static inline uint32_t sobol_value(uint32_t index, uint32_t dim) {   // OwenSobol.cs:98-117
    if (dim == 0u) return reverse_bits(index);
    uint32_t v = 0u;
    int k = 0;
    while (index != 0u) {
        if (index & 1u) v ^= kDim1Dirs[k];
        index >>= 1;
        k++;
    }
    return v;
}
float sobol_sample(uint32_t sample_index, uint32_t dim, uint32_t pixel_seed) {   // OwenSobol.cs:48-89
    uint32_t v;
    if (dim < 2u) {
        v = sobol_value(sample_index, dim);
    } else {
        uint32_t shuffle_seed = hash_u32(dim * 0x68bc21ebu + 0xc7afe638u);
        v = reverse_bits(owen_scramble(sample_index, shuffle_seed));
    }
    uint32_t scramble_seed = hash_u32(pixel_seed ^ hash_u32(dim * 0xa511e9b3u + 0x736f6c34u));
    v = owen_scramble(v, scramble_seed);
    return (float)(v >> 8) * (1.0f / 16777216.0f);   // ToFloat01, OwenSobol.cs:210
}

struct SamplerCtx {   // Sampler.cs:44-50
    uint32_t pixel_seed = 0, sample_index = 0, dim = 0;
    bool active = false;
    uint64_t prng = 0x9E3779B97F4A7C15ull;   // fallback when no pixel context is open
};
static thread_local SamplerCtx t_sampler;

static inline void begin_pixel_sample(uint32_t seed, uint32_t s) {   // Sampler.cs:75-83
    t_sampler.pixel_seed = seed;
    t_sampler.sample_index = s;
    t_sampler.dim = 0u;
    t_sampler.active = true;
}
static inline void end_pixel_sample() { t_sampler.active = false; }
static inline float random_float() {   // Sampler.cs:106-118 / MathUtils.cs:74
    SamplerCtx& c = t_sampler;
    if (!c.active) {
        // System.Random stand-in (only reached outside a pixel context).
        c.prng = c.prng * 6364136223846793005ull + 1442695040888963407ull;
        return (float)((c.prng >> 40) & 0xFFFFFFull) * (1.0f / 16777216.0f);
    }
    uint32_t d = c.dim++;
    return sobol_sample(c.sample_index, d, c.pixel_seed);
}
static inline V3 random_unit_vector() {   // MathUtils.cs:104-112
    float u = random_float();
    float v = random_float();
    float z = 1.0f - 2.0f * u;
    float r = std::sqrt(std::fmax(0.0f, 1.0f - z * z));
    float phi = 2.0f * kPi * v;
    return {r * std::cos(phi), r * std::sin(phi), z};
}

// ---------------------------------------------------------------------------
// Counters for the algorithmic-bytes model (B_s)
// ---------------------------------------------------------------------------
struct Counters {
    uint64_t node_visits = 0, tri_tests = 0, other_tests = 0;
    uint64_t closest_rays = 0, shadow_rays = 0, segments = 0, samples = 0;
};
static thread_local Counters t_cnt;
static thread_local bool t_counting = false;

// ---------------------------------------------------------------------------
// Core types: Ray (Core/Ray.cs), AABB (Core/AABB.cs), HitRecord
// ---------------------------------------------------------------------------
struct Ray {
    V3 o, d, inv;
    Ray() = default;
    Ray(V3 o_, V3 d_) : o(o_), d(d_), inv(v3(1.0f) / d_) {}   // Ray.cs:39-47
    V3 at(float t) const { return o + t * d; }                // Ray.cs:76
};

struct AABB {
    V3 mn, mx;
    bool hit(const Ray& r, float tmin, float tmax) const {   // AABB.cs:28-52
        if ((mn.x > mx.x) | (mn.y > mx.y) | (mn.z > mx.z)) return false;
        V3 t0 = (mn - r.o) * r.inv;
        V3 t1 = (mx - r.o) * r.inv;
        V3 ts = vmin(t0, t1);
        V3 tl = vmax(t0, t1);
        float te = std::fmax(tmin, std::fmax(ts.x, std::fmax(ts.y, ts.z)));
        float tx = std::fmin(tmax, std::fmin(tl.x, std::fmin(tl.y, tl.z)));
        return tx >= te;
    }
    float surface_area() const {   // AABB.cs:70-75
        V3 d = mx - mn;
        if (d.x < 0.0f || d.y < 0.0f || d.z < 0.0f) return 0.0f;
        return 2.0f * (d.x * d.y + d.x * d.z + d.y * d.z);
    }
};
static inline AABB surrounding(const AABB& a, const AABB& b) { return {vmin(a.mn, b.mn), vmax(a.mx, b.mx)}; }
static inline AABB aabb_empty() { return {v3(kInf), v3(-kInf)}; }   // AABB.cs:77

struct HitRecord {   // Core/HitRecord.cs (fields used on the path)
    float t = 0.0f;
    V3 p{}, n{};
    bool front = false;
    float u = 0.0f, v = 0.0f;
    V3 tangent{}, bitangent{};
    int material = -1;
    int entity = -1;
    int prim = -1;
    float relative_eta = 0.0f;
    void set_face_normal(const Ray& r, V3 outward) {   // HitRecord.cs:158-162
        front = dot(r.d, outward) < 0.0f;
        n = front ? outward : -outward;
    }
};

// ---------------------------------------------------------------------------
// Geometry (Geometry/*.cs) and the BVH (Acceleration/BvhNode.cs)
// ---------------------------------------------------------------------------
struct Hittable {
    virtual ~Hittable() = default;
    virtual bool hit(const Ray& r, float tmin, float tmax, HitRecord& rec) const = 0;
    virtual AABB bbox() const = 0;
};

struct Triangle : Hittable {   // Geometry/Triangle.cs, or SmoothTriangle.cs when smooth
    V3 v0, v1, v2, e1, e2, normal, tangent, bitangent;
    float area;
    int material, entity, prim;
    bool smooth = false;
    V3 n0{}, n1{}, n2{};
    float uv[6] = {0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 1.0f};
    // SmoothTriangle constructor (SmoothTriangle.cs:67-126): normalised vertex
    // normals, vertex UVs (the no-UV constructor's (0,0), (1,0), (0,1) when
    // uvs is null) and the tangent frame from the UV gradients, with the edge
    // fallback for a degenerate mapping. The face normal, area and edges are
    // the flat triangle's.
    void make_smooth(const float* nn, const float* uvs) {
        smooth = true;
        n0 = normalize(v3(nn[0], nn[1], nn[2]));
        n1 = normalize(v3(nn[3], nn[4], nn[5]));
        n2 = normalize(v3(nn[6], nn[7], nn[8]));
        if (uvs)
            for (int k = 0; k < 6; k++) uv[k] = uvs[k];
        float d1x = uv[2] - uv[0], d1y = uv[3] - uv[1];
        float d2x = uv[4] - uv[0], d2y = uv[5] - uv[1];
        float det = d1x * d2y - d2x * d1y;
        if (std::fabs(det) > 1e-8f) {
            float inv = 1.0f / det;
            V3 t = inv * (d2y * e1 - d1y * e2);
            V3 b = inv * ((-d2x) * e1 + d1x * e2);
            float tl = length(t), bl = length(b);
            if (tl > 1e-8f && bl > 1e-8f) {
                tangent = t / tl;
                bitangent = b / bl;
                return;
            }
        }
        tangent = normalize(e1);
        bitangent = normalize(e2);
    }
    Triangle(V3 a, V3 b, V3 c, int mat, int ent, int pr) : v0(a), v1(b), v2(c), material(mat), entity(ent), prim(pr) {
        e1 = v1 - v0;   // Triangle.cs:35-47
        e2 = v2 - v0;
        V3 cr = cross(e1, e2);
        float cl = length(cr);
        normal = cl > 0.0f ? cr / cl : v3(0, 1, 0);
        area = 0.5f * cl;
        tangent = length_sq(e1) > 0.0f ? normalize(e1) : v3(1, 0, 0);
        bitangent = length_sq(e2) > 0.0f ? normalize(e2) : v3(0, 0, 1);
    }
    bool hit(const Ray& r, float tmin, float tmax, HitRecord& rec) const override {   // Triangle.cs:49-89
        if (t_counting) t_cnt.tri_tests++;
        V3 h = cross(r.d, e2);
        float a = dot(e1, h);
        if (std::fabs(a) < 1e-7f) return false;
        float f = 1.0f / a;
        V3 s = r.o - v0;
        float u = f * dot(s, h);
        if (u < 0.0f || u > 1.0f) return false;
        V3 q = cross(s, e1);
        float v = f * dot(r.d, q);
        if (v < 0.0f || u + v > 1.0f) return false;
        float t = f * dot(e2, q);
        if (t < tmin || t > tmax) return false;
        rec.t = t;
        rec.p = r.at(t);
        if (smooth) {   // SmoothTriangle.cs:166-197: interpolated normal, face normal decides the side
            float w0 = 1.0f - u - v;
            V3 sn = normalize(w0 * n0 + u * n1 + v * n2);
            rec.front = dot(r.d, normal) < 0.0f;
            rec.n = rec.front ? sn : -sn;
        } else {
            rec.set_face_normal(r, normal);
        }
        // The barycentrics, for both kinds: a smooth triangle's record holds
        // the interpolated UV instead, which only texture lookups read, and
        // textures are constant on this path.
        rec.u = u;
        rec.v = v;
        rec.tangent = tangent;
        rec.bitangent = bitangent;
        rec.material = material;
        rec.entity = entity;
        rec.prim = prim;
        return true;
    }
    AABB bbox() const override {   // Triangle.cs:144-149
        V3 mn = vmin(vmin(v0, v1), v2) - v3(kEps);
        V3 mx = vmax(vmax(v0, v1), v2) + v3(kEps);
        return {mn, mx};
    }
    // Triangle.cs:130-140 (SampleAt)
    void sample_at(float xi1, float xi2, V3& p, V3& n, float& u, float& v) const {
        float r1 = std::sqrt(xi1);
        u = 1.0f - r1;
        v = xi2 * r1;
        if (smooth) {   // SmoothTriangle.SampleAt (:219-230): weights on the vertices themselves
            float w0 = 1.0f - u - v;
            p = w0 * v0 + u * v1 + v * v2;
            n = normalize(w0 * n0 + u * n1 + v * n2);
            return;
        }
        p = v0 + u * e1 + v * e2;
        n = normal;
    }
};

struct Quad : Hittable {   // Geometry/Quad.cs
    V3 q, u, v, normal, w, tangent, bitangent;
    float d, area;
    int material, entity;
    Quad(V3 q_, V3 u_, V3 v_, int mat, int ent) : q(q_), u(u_), v(v_), material(mat), entity(ent) {
        V3 nn = cross(u, v);   // Quad.cs:26-40
        normal = normalize(nn);
        d = dot(normal, q);
        w = nn / dot(nn, nn);
        tangent = normalize(u);
        bitangent = normalize(v);
        area = length(nn);
    }
    bool hit(const Ray& r, float tmin, float tmax, HitRecord& rec) const override {   // Quad.cs:42-86
        if (t_counting) t_cnt.other_tests++;
        float denom = dot(normal, r.d);
        if (std::fabs(denom) < 1e-8f) return false;
        float t = (d - dot(normal, r.o)) / denom;
        if (t < tmin || t > tmax) return false;
        V3 ip = r.at(t);
        V3 ph = ip - q;
        float alpha = dot(w, cross(ph, v));
        float beta = dot(w, cross(u, ph));
        if (alpha < 0 || alpha > 1 || beta < 0 || beta > 1) return false;
        rec.u = alpha;
        rec.v = beta;
        rec.t = t;
        rec.p = ip;
        rec.set_face_normal(r, normal);
        rec.tangent = tangent;
        rec.bitangent = bitangent;
        rec.material = material;
        rec.entity = entity;
        rec.prim = 0;
        return true;
    }
    AABB bbox() const override {   // Quad.cs:113-120
        AABB b{q, q + u + v};
        return {vmin(b.mn, vmin(q + u, q + v)) - v3(0.0001f), vmax(b.mx, vmax(q + u, q + v)) + v3(0.0001f)};
    }
};

struct Sphere : Hittable {   // Geometry/Sphere.cs
    V3 c;
    float r;
    int material, entity;
    Sphere(V3 c_, float r_, int mat, int ent) : c(c_), r(r_), material(mat), entity(ent) {}
    bool hit(const Ray& ray, float tmin, float tmax, HitRecord& rec) const override {   // Sphere.cs:20-70
        if (t_counting) t_cnt.other_tests++;
        V3 oc = ray.o - c;
        float a = length_sq(ray.d);
        float half_b = dot(oc, ray.d);
        float cc = length_sq(oc) - r * r;
        float disc = half_b * half_b - a * cc;
        if (disc < 0) return false;
        float sq = std::sqrt(disc);
        float root = (-half_b - sq) / a;
        if (root < tmin || root > tmax) {
            root = (-half_b + sq) / a;
            if (root < tmin || root > tmax) return false;
        }
        rec.t = root;
        rec.p = ray.at(rec.t);
        V3 outward = (rec.p - c) / r;
        rec.set_face_normal(ray, outward);
        // GetSphereUV only feeds textures; constant textures ignore it.
        rec.u = 0.0f;
        rec.v = 0.0f;
        V3 tdir = cross(v3(0, 1, 0), outward);
        if (length_sq(tdir) < 1e-4f) tdir = v3(1, 0, 0);
        rec.tangent = normalize(tdir);
        rec.bitangent = normalize(cross(outward, rec.tangent));
        rec.material = material;
        rec.entity = entity;
        rec.prim = 0;
        return true;
    }
    AABB bbox() const override { return {c - v3(r), c + v3(r)}; }   // Sphere.BoundingBox
};

struct BackFaceCulled : Hittable {   // Geometry/BackFaceCulledHittable.cs
    const Hittable* inner;
    explicit BackFaceCulled(const Hittable* h) : inner(h) {}
    bool hit(const Ray& r, float tmin, float tmax, HitRecord& rec) const override {
        HitRecord tmp;
        if (!inner->hit(r, tmin, tmax, tmp)) return false;
        if (!tmp.front) return false;
        rec = tmp;
        return true;
    }
    AABB bbox() const override { return inner->bbox(); }
};

struct HittableList : Hittable {   // Geometry/HittableList.cs
    std::vector<const Hittable*> objs;
    bool hit(const Ray& r, float tmin, float tmax, HitRecord& rec) const override {   // :19-37
        HitRecord tmp;
        bool any = false;
        float closest = tmax;
        for (size_t i = 0; i < objs.size(); i++) {
            if (objs[i]->hit(r, tmin, closest, tmp)) {
                any = true;
                closest = tmp.t;
                rec = tmp;
            }
        }
        return any;
    }
    AABB bbox() const override {   // :40-48
        if (objs.empty()) return aabb_empty();
        AABB b = objs[0]->bbox();
        for (size_t i = 1; i < objs.size(); i++) b = surrounding(b, objs[i]->bbox());
        return b;
    }
};

// Export record of one BVH node in build (pre-order) order, for structure comparison.
struct FlatNode {
    AABB box;
    int leaf;          // 1 = fat leaf
    int axis;
    int first, count;  // leaf range in the partitioned list
};

struct BvhNode : Hittable {   // Acceleration/BvhNode.cs
    static const int kMaxLeaf = 4;       // :53
    static const int kBins = 16;         // :60
    static constexpr float kTrav = 0.5f; // :68
    const BvhNode* left = nullptr;
    const BvhNode* right = nullptr;
    std::vector<const Hittable*> prims;
    AABB box;
    int axis = 0;
    int first = 0;
    std::vector<std::unique_ptr<BvhNode>>* arena = nullptr;

    // Builds over objs[start, end) and partitions objs in place (BvhNode.cs:91-152).
    BvhNode(std::vector<const Hittable*>& objs, int start, int end, std::vector<std::unique_ptr<BvhNode>>* ar)
        : arena(ar) {
        int span = end - start;
        first = start;
        if (span <= kMaxLeaf) {
            box = objs[start]->bbox();
            prims.push_back(objs[start]);
            for (int i = 1; i < span; i++) {
                prims.push_back(objs[start + i]);
                box = surrounding(box, objs[start + i]->bbox());
            }
            axis = 0;
            return;
        }
        int best_axis, mid;
        if (!sah_split(objs, start, end, best_axis, mid)) {
            best_axis = 0;
            mid = start + span / 2;
        }
        axis = best_axis;
        ar->emplace_back(new BvhNode(objs, start, mid, ar));
        BvhNode* l = ar->back().get();
        ar->emplace_back(new BvhNode(objs, mid, end, ar));
        BvhNode* r = ar->back().get();
        left = l;
        right = r;
        box = surrounding(l->box, r->box);
    }

    static bool sah_split(std::vector<const Hittable*>& objs, int start, int end, int& best_axis, int& mid) {
        // BvhNode.cs:218-363
        int span = end - start;
        V3 cmin = v3(kInf), cmax = v3(-kInf);
        for (int i = start; i < end; i++) {
            AABB b = objs[i]->bbox();
            V3 c = (b.mn + b.mx) * 0.5f;
            cmin = vmin(cmin, c);
            cmax = vmax(cmax, c);
        }
        V3 ext = cmax - cmin;
        float max_ext = std::fmax(ext.x, std::fmax(ext.y, ext.z));
        if (max_ext <= 0.0f) {
            best_axis = -1;
            mid = start;
            return false;
        }
        best_axis = -1;
        int best_bin = -1;
        float best_cost = kInf;
        int bin_count[kBins], pre_count[kBins], suf_count[kBins];
        AABB bin_box[kBins], pre_box[kBins], suf_box[kBins];
        for (int ax = 0; ax < 3; ax++) {
            float e = get_axis(ext, ax);
            if (e <= 0.0f) continue;
            float c0 = get_axis(cmin, ax);
            float scale = (float)kBins / e;
            for (int i = 0; i < kBins; i++) {
                bin_count[i] = 0;
                bin_box[i] = aabb_empty();
            }
            for (int i = start; i < end; i++) {
                AABB b = objs[i]->bbox();
                float c = get_axis((b.mn + b.mx) * 0.5f, ax);
                int idx = (int)((c - c0) * scale);
                if (idx < 0) idx = 0;
                else if (idx >= kBins) idx = kBins - 1;
                bin_count[idx]++;
                bin_box[idx] = surrounding(bin_box[idx], b);
            }
            int cum = 0;
            AABB cb = aabb_empty();
            for (int i = 0; i < kBins; i++) {
                cum += bin_count[i];
                cb = surrounding(cb, bin_box[i]);
                pre_count[i] = cum;
                pre_box[i] = cb;
            }
            cum = 0;
            cb = aabb_empty();
            for (int i = kBins - 1; i >= 0; i--) {
                cum += bin_count[i];
                cb = surrounding(cb, bin_box[i]);
                suf_count[i] = cum;
                suf_box[i] = cb;
            }
            float parent_area = pre_box[kBins - 1].surface_area();
            if (parent_area <= 0.0f) continue;
            for (int i = 0; i < kBins - 1; i++) {
                int nl = pre_count[i], nr = suf_count[i + 1];
                if (nl == 0 || nr == 0) continue;
                float cost = kTrav + (nl * pre_box[i].surface_area() + nr * suf_box[i + 1].surface_area()) / parent_area;
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = ax;
                    best_bin = i;
                }
            }
        }
        if (best_axis < 0) {
            mid = start;
            return false;
        }
        float axis_min = get_axis(cmin, best_axis);
        float axis_scale = (float)kBins / get_axis(ext, best_axis);
        int wp = start;
        for (int i = start; i < end; i++) {
            AABB b = objs[i]->bbox();
            float c = get_axis((b.mn + b.mx) * 0.5f, best_axis);
            int idx = (int)((c - axis_min) * axis_scale);
            if (idx < 0) idx = 0;
            else if (idx >= kBins) idx = kBins - 1;
            if (idx <= best_bin) {
                std::swap(objs[i], objs[wp]);
                wp++;
            }
        }
        mid = wp;
        if (mid == start || mid == end) mid = start + span / 2;
        return true;
    }

    bool hit(const Ray& r, float tmin, float tmax, HitRecord& rec) const override {   // BvhNode.cs:157-206
        if (t_counting) t_cnt.node_visits++;
        if (!box.hit(r, tmin, tmax)) return false;
        if (!prims.empty()) {
            bool any = false;
            float closest = tmax;
            for (size_t i = 0; i < prims.size(); i++) {
                if (prims[i]->hit(r, tmin, closest, rec)) {
                    any = true;
                    closest = rec.t;
                }
            }
            return any;
        }
        float dir_axis = get_axis(r.d, axis);
        const BvhNode *near_n, *far_n;
        if (dir_axis >= 0.0f) {
            near_n = left;
            far_n = right;
        } else {
            near_n = right;
            far_n = left;
        }
        bool hn = near_n->hit(r, tmin, tmax, rec);
        bool hf = far_n->hit(r, tmin, hn ? rec.t : tmax, rec);
        return hn || hf;
    }
    AABB bbox() const override { return box; }

    void flatten(std::vector<FlatNode>& out) const {   // pre-order: node, left subtree, right subtree
        FlatNode f;
        f.box = box;
        f.leaf = prims.empty() ? 0 : 1;
        f.axis = axis;
        f.first = first;
        f.count = (int)prims.size();
        out.push_back(f);
        if (!prims.empty()) return;
        left->flatten(out);
        right->flatten(out);
    }
};

struct Mesh : Hittable {   // Geometry/Mesh.cs
    std::vector<std::unique_ptr<Triangle>> tris;   // original order
    std::vector<const Hittable*> bvh_input;        // partitioned copy (BVH build order)
    std::vector<std::unique_ptr<BvhNode>> arena;
    std::unique_ptr<BvhNode> root;
    HittableList flat;
    bool use_bvh = false;
    std::vector<float> cum_area;
    float total_area = 0.0f;
    int material = -1;

    void finish() {   // Mesh.cs:75-108
        bvh_input.clear();
        for (auto& t : tris) bvh_input.push_back(t.get());
        if (tris.size() > 4) {   // BvhThreshold = 4 (Mesh.cs:93-96)
            use_bvh = true;
            root.reset(new BvhNode(bvh_input, 0, (int)bvh_input.size(), &arena));
        } else {
            flat.objs = bvh_input;
        }
        cum_area.resize(tris.size());
        float sum = 0;
        for (size_t i = 0; i < tris.size(); i++) {
            float a = 0.5f * length(cross(tris[i]->v1 - tris[i]->v0, tris[i]->v2 - tris[i]->v0));   // :195-203
            sum += a;
            cum_area[i] = sum;
        }
        total_area = sum;
    }
    bool hit(const Ray& r, float tmin, float tmax, HitRecord& rec) const override {   // :110-116
        return use_bvh ? root->hit(r, tmin, tmax, rec) : flat.hit(r, tmin, tmax, rec);
    }
    AABB bbox() const override { return use_bvh ? root->bbox() : flat.bbox(); }
    int pick_by_cdf(float target) const {   // Mesh.cs:173-178 (Array.BinarySearch)
        int idx = (int)(std::lower_bound(cum_area.begin(), cum_area.end(), target) - cum_area.begin());
        return std::min(std::max(idx, 0), (int)tris.size() - 1);
    }
};

// ---------------------------------------------------------------------------
// Materials
// ---------------------------------------------------------------------------
struct ShadingParams {   // DisneyBsdf.cs:213-293
    float metallic, roughness, specular, specular_tint, sheen, sheen_tint, sheen_roughness;
    float clearcoat, clearcoat_gloss, spec_trans, ior, anisotropic, anisotropic_rotation, diff_trans;
    float alpha, alpha_x, alpha_y, clearcoat_alpha, clearcoat_f0, thin_film_nm, thin_film_ior;
};

struct Material {
    RtMaterialDesc d;
    ShadingParams sp;
    bool is_emissive() const { return d.type == RT_MAT_EMISSIVE; }
};

static ShadingParams make_shading_params(const RtMaterialDesc& m) {   // DisneyBsdf.cs:237-291
    ShadingParams s;
    s.metallic = clampf(m.metallic, 0.0f, 1.0f);
    s.roughness = clampf(m.roughness, 0.0f, 1.0f);
    s.specular = clampf(m.specular, 0.0f, 2.0f);
    s.specular_tint = clampf(m.specular_tint, 0.0f, 1.0f);
    s.sheen = clampf(m.sheen, 0.0f, 1.0f);
    s.sheen_tint = clampf(m.sheen_tint, 0.0f, 1.0f);
    s.sheen_roughness = clampf(m.sheen_roughness, 0.04f, 1.0f);
    s.clearcoat = clampf(m.clearcoat, 0.0f, 1.0f);
    s.clearcoat_gloss = clampf(m.clearcoat_gloss, 0.0f, 1.0f);
    s.spec_trans = clampf(m.spec_trans, 0.0f, 1.0f);
    s.ior = std::fmax(m.ior, 1.0001f);
    s.anisotropic = clampf(m.anisotropic, 0.0f, 1.0f);
    s.anisotropic_rotation = m.anisotropic_rotation - std::floor(m.anisotropic_rotation);
    s.diff_trans = clampf(m.diff_trans, 0.0f, 1.0f);
    s.alpha = std::fmax(s.roughness * s.roughness, 0.001f);
    float aspect = std::sqrt(1.0f - 0.9f * s.anisotropic);
    s.alpha_x = std::fmax(s.alpha / aspect, 0.001f);
    s.alpha_y = std::fmax(s.alpha * aspect, 0.001f);
    s.clearcoat_alpha = m.coat_roughness >= 0.0f ? std::fmax(m.coat_roughness * m.coat_roughness, 0.001f)
                                                 : lerpf(0.1f, 0.001f, s.clearcoat_gloss);
    float eta_coat = std::fmax(m.coat_ior, 1.0001f);
    float r0 = (eta_coat - 1.0f) / (eta_coat + 1.0f);
    s.clearcoat_f0 = r0 * r0;
    s.thin_film_nm = std::fmax(m.thin_film_thickness, 0.0f);
    s.thin_film_ior = std::fmax(m.thin_film_ior, 1.0001f);
    return s;
}

// Kulla-Conty LUT (Materials/EnergyCompensationLut.cs)
struct EnergyLut {
    static const int kMu = 32, kAl = 32, kSpb = 2048;
    float e[kMu * kAl];
    float eavg[kAl];
    EnergyLut();
    float sample_e(float mu, float alpha) const;
    float sample_eavg(float alpha) const;
};

// Microfacet (Materials/Microfacet.cs)
static inline void build_tangent_frame(V3 n, V3& t, V3& b) {   // :22-37
    if (n.z < -0.999f) {
        t = v3(0, -1, 0);
        b = v3(-1, 0, 0);
    } else {
        float a = 1.0f / (1.0f + n.z);
        float bb = -n.x * n.y * a;
        t = v3(1.0f - n.x * n.x * a, bb, -n.x);
        b = v3(bb, 1.0f - n.y * n.y * a, -n.y);
    }
}
static inline float d_ggx_aniso(V3 h, float ax, float ay) {   // :43-49
    float hx = h.x / ax;
    float hy = h.y / ay;
    float d = hx * hx + hy * hy + h.z * h.z;
    return 1.0f / std::fmax(kPi * ax * ay * d * d, 1e-20f);
}
static inline float lambda_ggx_aniso(V3 w, float ax, float ay) {   // :55-61
    float c2 = w.z * w.z;
    if (c2 < 1e-14f) return 1e10f;
    float num = (ax * w.x) * (ax * w.x) + (ay * w.y) * (ay * w.y);
    return 0.5f * (-1.0f + std::sqrt(1.0f + num / c2));
}
static inline float g1_ggx_aniso(V3 w, float ax, float ay) { return 1.0f / (1.0f + lambda_ggx_aniso(w, ax, ay)); }
static inline float smith_g1(float ndx, float alpha) {   // :75-81
    float a2 = alpha * alpha;
    float n2 = ndx * ndx;
    float denom = ndx + std::sqrt(a2 + (1.0f - a2) * n2);
    return 2.0f * ndx / std::fmax(denom, 1e-7f);
}
static inline V3 sample_ggx_vndf_aniso(V3 vl, float ax, float ay, float u1, float u2) {   // :100-124
    V3 vh = normalize(v3(ax * vl.x, ay * vl.y, vl.z));
    float len_sq = vh.x * vh.x + vh.y * vh.y;
    V3 t1 = len_sq > 0.0f ? v3(-vh.y, vh.x, 0.0f) / std::sqrt(len_sq) : v3(1, 0, 0);
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

EnergyLut::EnergyLut() {   // EnergyCompensationLut.cs:48-74
    auto mu_value = [](int i) { return ((float)i + 0.5f) / (float)kMu; };
    auto alpha_value = [](int i) { return std::fmax(((float)i + 0.5f) / (float)kAl, 0.001f); };
    for (int ai = 0; ai < kAl; ai++) {
        float alpha = alpha_value(ai);
        for (int mi = 0; mi < kMu; mi++) {
            float mu = mu_value(mi);
            uint32_t seed = ((uint32_t)mi * 0x9E3779B9u) ^ ((uint32_t)ai * 0xB5297A4Du) ^ 0xC2B2AE3Du;
            // IntegrateE (:95-120)
            float sin_t = std::sqrt(std::fmax(0.0f, 1.0f - mu * mu));
            V3 V = v3(sin_t, 0.0f, mu);
            double sum = 0.0;
            uint32_t st = seed == 0 ? 1u : seed;
            int hits = 0;
            auto next = [&st]() {   // :127-134 xorshift32
                st ^= st << 13;
                st ^= st >> 17;
                st ^= st << 5;
                return (float)(st & 0x00FFFFFFu) / (float)0x01000000u;
            };
            for (int s = 0; s < kSpb; s++) {
                float u1 = next();
                float u2 = next();
                V3 H = sample_ggx_vndf_aniso(V, alpha, alpha, u1, u2);
                float vdh = dot(V, H);
                V3 L = 2.0f * vdh * H - V;
                if (L.z <= 0.0f) continue;
                sum += (double)g1_ggx_aniso(L, alpha, alpha);
                hits++;
            }
            double m = sum / (double)kSpb;
            m = m < 0.0 ? 0.0 : (m > 1.0 ? 1.0 : m);
            e[mi * kAl + ai] = hits == 0 ? 0.0f : (float)m;
        }
        float avg = 0.0f;
        for (int mi = 0; mi < kMu; mi++) avg += 2.0f * e[mi * kAl + ai] * mu_value(mi);
        eavg[ai] = clampf(avg / (float)kMu, 0.0f, 1.0f);
    }
}
float EnergyLut::sample_e(float mu, float alpha) const {   // :140-161
    mu = clampf(mu, 0.0f, 1.0f);
    alpha = clampf(alpha, 0.001f, 1.0f);
    float fmu = mu * kMu - 0.5f;
    float fal = alpha * kAl - 0.5f;
    int mi0 = std::min(std::max((int)std::floor(fmu), 0), kMu - 1);
    int ai0 = std::min(std::max((int)std::floor(fal), 0), kAl - 1);
    int mi1 = std::min(mi0 + 1, kMu - 1);
    int ai1 = std::min(ai0 + 1, kAl - 1);
    float tu = clampf(fmu - (float)mi0, 0.0f, 1.0f);
    float ta = clampf(fal - (float)ai0, 0.0f, 1.0f);
    float e00 = e[mi0 * kAl + ai0], e01 = e[mi0 * kAl + ai1];
    float e10 = e[mi1 * kAl + ai0], e11 = e[mi1 * kAl + ai1];
    float e0 = e00 + (e01 - e00) * ta;
    float e1 = e10 + (e11 - e10) * ta;
    return e0 + (e1 - e0) * tu;
}
float EnergyLut::sample_eavg(float alpha) const {   // :167-175
    alpha = clampf(alpha, 0.001f, 1.0f);
    float fal = alpha * kAl - 0.5f;
    int ai0 = std::min(std::max((int)std::floor(fal), 0), kAl - 1);
    int ai1 = std::min(ai0 + 1, kAl - 1);
    float ta = clampf(fal - (float)ai0, 0.0f, 1.0f);
    return eavg[ai0] + (eavg[ai1] - eavg[ai0]) * ta;
}

static const EnergyLut& energy_lut() {
    static EnergyLut lut;   // EnergyCompensationLut.Prewarm (Renderer.cs:441)
    return lut;
}

// Sheen (Materials/SheenCharlie.cs)
static inline float sheen_d(float ndh, float alpha) {   // :24-34
    alpha = std::fmax(alpha, 0.04f);
    float inv = 1.0f / alpha;
    float c2 = ndh * ndh;
    float s2 = std::fmax(1.0f - c2, 0.0f);
    float sp = std::pow(s2, 0.5f * inv);
    return (2.0f + inv) * sp / (2.0f * kPi);
}
static inline float sheen_lambda_log(float c, float alpha) {   // :40-65
    float a, b, cc, d, e;
    if (alpha < 0.25f) {
        a = 25.3245f; b = 3.32435f; cc = 0.16801f; d = -1.27393f; e = -4.85967f;
    } else {
        a = 21.5473f; b = 3.82987f; cc = 0.19823f; d = -1.97760f; e = -4.32054f;
    }
    return a / (1.0f + b * std::pow(c, cc)) + d * c + e;
}
static inline float sheen_lambda(float c, float alpha) {   // :71-85
    c = clampf(c, 1e-4f, 1.0f);
    const float split = 0.25f, window = 0.05f;
    if (alpha <= split - window) return std::exp(sheen_lambda_log(c, 0.0f));
    if (alpha >= split + window) return std::exp(sheen_lambda_log(c, 1.0f));
    float t = (alpha - (split - window)) / (2.0f * window);
    float lo = std::exp(sheen_lambda_log(c, 0.0f));
    float hi = std::exp(sheen_lambda_log(c, 1.0f));
    return lo + (hi - lo) * t;
}
static inline float sheen_brdf(float ndv, float ndl, float ndh, float alpha) {   // :92-121
    float denom = 4.0f * std::fmax(ndv, 1e-6f) * std::fmax(ndl, 1e-6f);
    float g = 1.0f / ((1.0f + sheen_lambda(ndv, alpha)) * (1.0f + sheen_lambda(ndl, alpha)));
    return sheen_d(ndh, alpha) * g / denom;
}

enum Lobe { kDiffuse = 0, kSpecular, kTransmission, kSheen, kMultiscatter, kDiffTrans, kClearcoat };
static const float kDeltaAlpha = 2.5e-3f;   // DisneyBsdf.cs:1167

struct BsdfSample {   // Materials/BsdfSample.cs:62-85
    V3 wo, f;
    float pdf;
    bool is_delta;
    bool has_next_absorption;
    V3 next_absorption;
    int transition;   // 0 none, 1 enter, 2 exit
};

struct Frame {   // DisneyBsdf.cs:1725-1738
    V3 t, b, n;
    V3 to_local(V3 w) const { return v3(dot(w, t), dot(w, b), dot(w, n)); }
    V3 to_world(V3 w) const { return w.x * t + w.y * b + w.z * n; }
};

struct LobeWeights {   // DisneyBsdf.cs:1069-1102
    float d, s, t, c, sh, ms, dt, total;
    float p_d() const { return d / total; }
    float p_s() const { return s / total; }
    float p_t() const { return t / total; }
    float p_c() const { return c / total; }
    float p_sh() const { return sh / total; }
    float p_ms() const { return ms / total; }
    float p_dt() const { return dt / total; }
};

struct Disney {
    const Material& m;
    explicit Disney(const Material& mat) : m(mat) {}
    V3 base() const { return v3(m.d.base_color[0], m.d.base_color[1], m.d.base_color[2]); }

    static float schlick_weight(float c) {   // :1994-1999
        float x = clampf(1.0f - c, 0.0f, 1.0f);
        float x2 = x * x;
        return x2 * x2 * x;
    }
    static V3 fresnel_schlick(float c, V3 f0) {   // :1963-1967
        float w = schlick_weight(c);
        return f0 + (v3(1.0f) - f0) * w;
    }
    V3 eval_fresnel(float c, V3 f0) const {   // :1984-1989 (thin film off: thickness 0)
        return fresnel_schlick(c, f0);
    }
    static V3 compute_f0(V3 bc, const ShadingParams& sp) {   // :1943-1959
        float r = (sp.ior - 1.0f) / (sp.ior + 1.0f);
        float f0d = r * r;
        float scaled = f0d * 2.0f * sp.specular;
        float lum = luminance(bc);
        V3 tint = lum > 0.0f ? bc / lum : v3(1.0f);
        V3 diel = lerp(v3(scaled), scaled * tint, sp.specular_tint);
        return lerp(diel, bc, sp.metallic);
    }
    static V3 multiscatter_weight(V3 f0, const ShadingParams& sp, float ndv, float ndl) {   // :1906-1926
        const EnergyLut& lut = energy_lut();
        float a_iso = std::sqrt(sp.alpha_x * sp.alpha_y);
        float e_out = lut.sample_e(ndv, a_iso);
        float e_in = lut.sample_e(ndl, a_iso);
        float e_avg = lut.sample_eavg(a_iso);
        float one_m = std::fmax(1.0f - e_avg, 1e-6f);
        V3 f_avg = f0 + (v3(1.0f) - f0) * (1.0f / 21.0f);
        V3 denom = v3(1.0f) - f_avg * (1.0f - e_avg);
        denom = v3(std::fmax(denom.x, 1e-6f), std::fmax(denom.y, 1e-6f), std::fmax(denom.z, 1e-6f));
        V3 f_ms = f_avg * f_avg * e_avg / denom;
        return f_ms * ((1.0f - e_out) * (1.0f - e_in) / one_m);
    }
    static V3 eval_multiscatter(V3 f0, const ShadingParams& sp, float ndv, float ndl) {   // :1934-1936
        return multiscatter_weight(f0, sp, ndv, ndl) * (1.0f / kPi);
    }
    static Frame shading_frame(const HitRecord& rec, float rotation) {   // :1840-1877
        V3 n = rec.n, t, b;
        if (length_sq(rec.tangent) > 1e-10f && length_sq(rec.bitangent) > 1e-10f) {
            t = rec.tangent - dot(rec.tangent, n) * n;
            float tl = length_sq(t);
            if (tl > 1e-10f) {
                t /= std::sqrt(tl);
                b = cross(n, t);
            } else {
                build_tangent_frame(n, t, b);
            }
        } else {
            build_tangent_frame(n, t, b);
        }
        if (rotation != 0.0f) {
            float angle = 2.0f * kPi * rotation;
            float c = std::cos(angle), s = std::sin(angle);
            V3 tr = c * t + s * b;
            V3 br = -s * t + c * b;
            t = tr;
            b = br;
        }
        return {t, b, n};
    }
    static V3 coat_normal(const HitRecord& rec) { return rec.n; }   // :1754 (no coat normal map)
    static Frame clearcoat_frame(const HitRecord& rec) {   // :1781-1786
        V3 cn = coat_normal(rec), t, b;
        build_tangent_frame(cn, t, b);
        return {t, b, cn};
    }
    static LobeWeights lobe_weights(V3 bc, const ShadingParams& sp) {   // :1104-1139
        float diffuse_all = (1.0f - sp.metallic) * (1.0f - sp.spec_trans);
        float diffuse_w = diffuse_all * (1.0f - sp.diff_trans);
        float diff_trans_w = diffuse_all * sp.diff_trans;
        float spec_f0;
        if (sp.metallic > 0.5f) {
            spec_f0 = luminance(bc);
        } else {
            float r = (sp.ior - 1.0f) / (sp.ior + 1.0f);
            spec_f0 = r * r * 2.0f * sp.specular;
        }
        float spec_floor = 0.1f * (1.0f - sp.spec_trans * 0.9f);
        float spec_w = std::fmax(spec_floor, lerpf(spec_f0, 1.0f, sp.metallic));
        float trans_w = (1.0f - sp.metallic) * sp.spec_trans;
        float clear_w = sp.clearcoat * 0.04f;
        float sheen_w = sp.sheen * 0.25f * diffuse_all;
        float a_iso = std::sqrt(sp.alpha_x * sp.alpha_y);
        float e_avg = energy_lut().sample_eavg(a_iso);
        float ms_w = spec_w * (1.0f - e_avg);
        LobeWeights w;
        w.d = diffuse_w; w.s = spec_w; w.t = trans_w; w.c = clear_w; w.sh = sheen_w; w.ms = ms_w; w.dt = diff_trans_w;
        float sum = diffuse_w + spec_w + trans_w + clear_w + sheen_w + ms_w + diff_trans_w;
        w.total = sum < 1e-6f ? 1.0f : sum;
        return w;
    }
    // ResolveTransmission (:1016-1049)
    void resolve_transmission(V3 bc, V3& tint, V3& sigma) const {
        if (!m.d.has_transmission_color) {
            tint = v3(std::sqrt(std::fmax(bc.x, 0.0f)), std::sqrt(std::fmax(bc.y, 0.0f)), std::sqrt(std::fmax(bc.z, 0.0f)));
            sigma = v3(0.0f);
            return;
        }
        V3 tc = v3(m.d.transmission_color[0], m.d.transmission_color[1], m.d.transmission_color[2]);
        float depth = std::fmax(m.d.transmission_depth, 0.0f);
        if (depth <= 0.0f) {
            tint = tc;
            sigma = v3(0.0f);
            return;
        }
        V3 c = v3(std::fmax(tc.x, 1e-6f), std::fmax(tc.y, 1e-6f), std::fmax(tc.z, 1e-6f));
        float inv_d = 1.0f / depth;
        sigma = v3(-std::log(c.x) * inv_d, -std::log(c.y) * inv_d, -std::log(c.z) * inv_d);
        tint = v3(1.0f);
    }

    // EvaluateDirect (:418-535)
    V3 evaluate_direct(V3 to_light, V3 to_eye, V3 normal, const HitRecord& rec) const {
        float ndl = std::fmax(dot(normal, to_light), 0.0f);
        if (ndl <= 0.0f) return v3(0.0f);
        float ndv = std::fmax(dot(normal, to_eye), 0.001f);
        V3 H = normalize(to_light + to_eye);
        float ndh = std::fmax(dot(normal, H), 0.0f);
        float vdh = std::fmax(dot(to_eye, H), 0.0f);
        float ldh = std::fmax(dot(to_light, H), 0.0f);
        V3 bc = base();
        const ShadingParams& sp = m.sp;
        float diffuse_w = (1.0f - sp.metallic) * (1.0f - sp.spec_trans) * (1.0f - sp.diff_trans);
        V3 diffuse = v3(0.0f);
        if (diffuse_w > 0.0f) {
            float fd90 = 0.5f + 2.0f * sp.roughness * ldh * ldh;
            float fi = schlick_weight(ndv);
            float fo = schlick_weight(ndl);
            float fd = (1.0f + (fd90 - 1.0f) * fi) * (1.0f + (fd90 - 1.0f) * fo);
            diffuse = bc * fd * (diffuse_w * ndl / kPi);
        }
        V3 f0 = compute_f0(bc, sp);
        V3 specular = v3(0.0f);
        if (sp.alpha > kDeltaAlpha) {
            Frame fr = shading_frame(rec, sp.anisotropic_rotation);
            V3 vl = fr.to_local(to_eye), ll = fr.to_local(to_light), hl = fr.to_local(H);
            float D = d_ggx_aniso(hl, sp.alpha_x, sp.alpha_y);
            float G = g1_ggx_aniso(vl, sp.alpha_x, sp.alpha_y) * g1_ggx_aniso(ll, sp.alpha_x, sp.alpha_y);
            V3 F = eval_fresnel(vdh, f0);
            specular = D * G * F / std::fmax(4.0f * ndv, 1e-6f);
        }
        V3 clearcoat = v3(0.0f);
        if (sp.clearcoat > 0.0f && sp.clearcoat_alpha > kDeltaAlpha) {
            V3 cn = coat_normal(rec);
            float cc_ndv = std::fmax(dot(cn, to_eye), 0.001f);
            float cc_ndl = dot(cn, to_light);
            if (cc_ndl > 0.0f) {
                float cc_ndh = std::fmax(dot(cn, H), 0.0f);
                float cc_vdh = std::fmax(dot(to_eye, H), 0.0f);
                float ca2 = sp.clearcoat_alpha * sp.clearcoat_alpha;
                float cden = cc_ndh * cc_ndh * (ca2 - 1.0f) + 1.0f;
                float cD = ca2 / (kPi * cden * cden);
                float cG = smith_g1(cc_ndv, sp.clearcoat_alpha) * smith_g1(cc_ndl, sp.clearcoat_alpha);
                float cF = sp.clearcoat_f0 + (1.0f - sp.clearcoat_f0) * schlick_weight(cc_vdh);
                clearcoat = v3(sp.clearcoat * 0.25f * cD * cG * cF / std::fmax(4.0f * cc_ndv, 1e-6f));
            }
        }
        V3 sheen = v3(0.0f);
        if (sp.sheen > 0.0f && diffuse_w > 0.0f) {
            float lum = luminance(bc);
            V3 tint = lum > 0.0f ? bc / lum : v3(1.0f);
            V3 scol = lerp(v3(1.0f), tint, sp.sheen_tint);
            float sb = sheen_brdf(ndv, ndl, ndh, sp.sheen_roughness);
            sheen = sp.sheen * sb * scol * ndl;
        }
        V3 ms = eval_multiscatter(f0, sp, ndv, ndl) * ndl;
        return diffuse + sheen + specular + ms + clearcoat;
    }

    // Evaluate (:649-771)
    V3 evaluate(V3 V, V3 L, const HitRecord& rec) const {
        V3 N = rec.n;
        float ndl = dot(N, L);
        float ndv = dot(N, V);
        if (ndv <= 0.0f) return v3(0.0f);
        V3 bc = base();
        const ShadingParams& sp = m.sp;
        if (ndl <= 0.0f) {
            float diff_all = (1.0f - sp.metallic) * (1.0f - sp.spec_trans);
            if (diff_all <= 0.0f || sp.diff_trans <= 0.0f) return v3(0.0f);
            return bc * (diff_all * sp.diff_trans / kPi);
        }
        V3 hraw = V + L;
        float hl2 = length_sq(hraw);
        if (hl2 < 1e-14f) return v3(0.0f);
        V3 H = hraw / std::sqrt(hl2);
        float ndh = std::fmax(dot(N, H), 0.0f);
        float vdh = std::fmax(dot(V, H), 0.0f);
        float ldh = std::fmax(dot(L, H), 0.0f);
        float diffuse_s = (1.0f - sp.metallic) * (1.0f - sp.spec_trans) * (1.0f - sp.diff_trans);
        V3 diffuse = v3(0.0f);
        if (diffuse_s > 0.0f) {
            float fd90 = 0.5f + 2.0f * sp.roughness * ldh * ldh;
            float fi = schlick_weight(ndv);
            float fo = schlick_weight(ndl);
            float fd = (1.0f + (fd90 - 1.0f) * fi) * (1.0f + (fd90 - 1.0f) * fo);
            diffuse = bc * fd * (diffuse_s / kPi);
        }
        V3 sheen = v3(0.0f);
        if (sp.sheen > 0.0f && diffuse_s > 0.0f) {
            float lum = luminance(bc);
            V3 tint = lum > 0.0f ? bc / lum : v3(1.0f);
            V3 scol = lerp(v3(1.0f), tint, sp.sheen_tint);
            float sb = sheen_brdf(ndv, ndl, ndh, sp.sheen_roughness);
            sheen = sp.sheen * sb * scol;
        }
        Frame fr = shading_frame(rec, sp.anisotropic_rotation);
        V3 vl = fr.to_local(V), ll = fr.to_local(L), hl = fr.to_local(H);
        float D = d_ggx_aniso(hl, sp.alpha_x, sp.alpha_y);
        float G = g1_ggx_aniso(vl, sp.alpha_x, sp.alpha_y) * g1_ggx_aniso(ll, sp.alpha_x, sp.alpha_y);
        V3 f0 = compute_f0(bc, sp);
        V3 F = eval_fresnel(vdh, f0);
        V3 specular = D * G / std::fmax(4.0f * ndv * ndl, 1e-7f) * F;
        V3 clearcoat = v3(0.0f);
        if (sp.clearcoat > 0.0f) {
            V3 cn = coat_normal(rec);
            float cc_ndv = dot(cn, V);
            float cc_ndl = dot(cn, L);
            if (cc_ndv > 0.0f && cc_ndl > 0.0f) {
                float cc_ndh = std::fmax(dot(cn, H), 0.0f);
                float cc_vdh = std::fmax(dot(V, H), 0.0f);
                float ca2 = sp.clearcoat_alpha * sp.clearcoat_alpha;
                float cden = cc_ndh * cc_ndh * (ca2 - 1.0f) + 1.0f;
                float cD = ca2 / (kPi * cden * cden);
                float cG = smith_g1(cc_ndv, sp.clearcoat_alpha) * smith_g1(cc_ndl, sp.clearcoat_alpha);
                float cF = sp.clearcoat_f0 + (1.0f - sp.clearcoat_f0) * schlick_weight(cc_vdh);
                float cc = sp.clearcoat * 0.25f * cD * cG * cF / std::fmax(4.0f * cc_ndv * cc_ndl, 1e-7f);
                clearcoat = v3(cc);
            }
        }
        V3 ms = eval_multiscatter(f0, sp, ndv, ndl);
        return diffuse + sheen + specular + ms + clearcoat;
    }

    // Pdf (:783-870)
    float pdf(V3 V, V3 L, const HitRecord& rec) const {
        V3 N = rec.n;
        float ndl = dot(N, L);
        float ndv = dot(N, V);
        if (ndv <= 0.0f) return 0.0f;
        V3 bc = base();
        const ShadingParams& sp = m.sp;
        LobeWeights w = lobe_weights(bc, sp);
        float cos_pdf = ndl > 0.0f ? ndl / kPi : 0.0f;
        float dt_pdf = ndl < 0.0f ? -ndl / kPi : 0.0f;
        float spec_pdf = 0.0f, cc_pdf = 0.0f;
        V3 hraw = V + L;
        float hl2 = length_sq(hraw);
        if (hl2 >= 1e-14f) {
            V3 H = hraw / std::sqrt(hl2);
            float ndh = dot(N, H);
            if (ndh > 0.0f && sp.alpha > kDeltaAlpha) {
                float safe_ndv = std::fmax(ndv, 1e-7f);
                Frame fr = shading_frame(rec, sp.anisotropic_rotation);
                V3 vl = fr.to_local(V), hl = fr.to_local(H);
                float D = d_ggx_aniso(hl, sp.alpha_x, sp.alpha_y);
                float g1v = g1_ggx_aniso(vl, sp.alpha_x, sp.alpha_y);
                spec_pdf = g1v * D / (4.0f * safe_ndv);
            }
            if (sp.clearcoat_alpha > kDeltaAlpha) {
                V3 cn = coat_normal(rec);
                float cc_ndv = dot(cn, V);
                float cc_ndh = dot(cn, H);
                if (cc_ndv > 0.0f && cc_ndh > 0.0f) {
                    float safe = std::fmax(cc_ndv, 1e-7f);
                    float ca2 = sp.clearcoat_alpha * sp.clearcoat_alpha;
                    float cden = cc_ndh * cc_ndh * (ca2 - 1.0f) + 1.0f;
                    float cD = ca2 / (kPi * cden * cden);
                    float cg1v = smith_g1(cc_ndv, sp.clearcoat_alpha);
                    cc_pdf = cg1v * cD / (4.0f * safe);
                }
            }
        }
        return w.p_d() * cos_pdf + w.p_sh() * cos_pdf + w.p_ms() * cos_pdf + w.p_s() * spec_pdf + w.p_c() * cc_pdf +
               w.p_dt() * dt_pdf;
    }

    // ScatterInternal (:1176-1248) and the lobe samplers (:1263-1709)
    bool scatter_internal(V3 ray_in_dir, const HitRecord& rec, V3& att, V3& out_dir, int& lobe) const {
        V3 bc = base();
        const ShadingParams& sp = m.sp;
        V3 N = rec.n;
        V3 V = normalize(-ray_in_dir);
        LobeWeights w = lobe_weights(bc, sp);
        float pd = w.p_d(), ps = w.p_s(), pt = w.p_t(), psh = w.p_sh(), pms = w.p_ms(), pdt = w.p_dt();
        float rnd = random_float();
        bool result;
        if (rnd < pd) {
            lobe = kDiffuse;
            result = scatter_diffuse(rec, bc, N, V, sp, pd, att, out_dir);
        } else if ((rnd -= pd) < ps) {
            lobe = kSpecular;
            result = scatter_specular(rec, bc, N, V, sp, ps, att, out_dir);
        } else if ((rnd -= ps) < pt) {
            lobe = kTransmission;
            result = scatter_transmission(ray_in_dir, rec, bc, N, V, sp, pt, att, out_dir);
        } else if ((rnd -= pt) < psh) {
            lobe = kSheen;
            result = scatter_sheen(rec, bc, N, V, sp, psh, att, out_dir);
        } else if ((rnd -= psh) < pms) {
            lobe = kMultiscatter;
            result = scatter_multiscatter(rec, bc, N, V, sp, pms, att, out_dir);
        } else if ((rnd -= pms) < pdt) {
            lobe = kDiffTrans;
            result = scatter_diff_trans(rec, bc, N, V, sp, pdt, att, out_dir);
        } else {
            lobe = kClearcoat;
            result = scatter_clearcoat(rec, N, V, sp, w.p_c(), att, out_dir);
        }
        if (std::isnan(att.x) || std::isinf(att.x) || std::isnan(att.y) || std::isinf(att.y) || std::isnan(att.z) ||
            std::isinf(att.z))
            att = bc;
        return result;
    }
    bool scatter_diffuse(const HitRecord&, V3 bc, V3 N, V3 V, const ShadingParams& sp, float prob, V3& att,
                         V3& dir) const {   // :1263-1306
        V3 sd = N + random_unit_vector();
        if (near_zero(sd)) sd = N;
        sd = normalize(sd);
        dir = sd;
        V3 L = sd;
        float ndv = std::fmax(dot(N, V), 0.001f);
        float ndl = std::fmax(dot(N, L), 0.001f);
        V3 hraw = V + L;
        float hl2 = length_sq(hraw);
        V3 H = hl2 > 1e-7f ? hraw / std::sqrt(hl2) : N;
        float ldh = std::fmax(dot(L, H), 0.0f);
        float fd90 = 0.5f + 2.0f * sp.roughness * ldh * ldh;
        float fi = schlick_weight(ndv), fo = schlick_weight(ndl);
        float fd = (1.0f + (fd90 - 1.0f) * fi) * (1.0f + (fd90 - 1.0f) * fo);
        att = bc * fd;
        att *= (1.0f - sp.diff_trans);
        att /= std::fmax(prob, 0.1f);
        return true;
    }
    bool scatter_diff_trans(const HitRecord&, V3 bc, V3 N, V3, const ShadingParams& sp, float prob, V3& att,
                            V3& dir) const {   // :1321-1338
        V3 sd = -N + random_unit_vector();
        if (near_zero(sd)) sd = -N;
        sd = normalize(sd);
        dir = sd;
        att = bc * sp.diff_trans;
        att /= std::fmax(prob, 0.05f);
        return true;
    }
    bool scatter_sheen(const HitRecord&, V3 bc, V3 N, V3 V, const ShadingParams& sp, float prob, V3& att,
                       V3& dir) const {   // :1354-1388
        V3 sd = N + random_unit_vector();
        if (near_zero(sd)) sd = N;
        sd = normalize(sd);
        dir = sd;
        V3 L = sd;
        float ndv = std::fmax(dot(N, V), 1e-4f);
        float ndl = std::fmax(dot(N, L), 1e-4f);
        V3 hraw = V + L;
        float hl2 = length_sq(hraw);
        V3 H = hl2 > 1e-7f ? hraw / std::sqrt(hl2) : N;
        float ndh = std::fmax(dot(N, H), 0.0f);
        float sb = sheen_brdf(ndv, ndl, ndh, sp.sheen_roughness);
        float lum = luminance(bc);
        V3 tint = lum > 0.0f ? bc / lum : v3(1.0f);
        V3 scol = lerp(v3(1.0f), tint, sp.sheen_tint);
        att = sp.sheen * kPi * sb * scol;
        att /= std::fmax(prob, 0.1f);
        return true;
    }
    bool scatter_specular(const HitRecord& rec, V3 bc, V3 N, V3 V, const ShadingParams& sp, float prob, V3& att,
                          V3& dir) const {   // :1399-1444
        Frame fr = shading_frame(rec, sp.anisotropic_rotation);
        V3 vl = fr.to_local(V);
        float u1 = random_float();
        float u2 = random_float();
        V3 hl = sample_ggx_vndf_aniso(vl, sp.alpha_x, sp.alpha_y, u1, u2);
        V3 H = fr.to_world(hl);
        V3 L = reflect(-V, H);
        if (dot(L, N) <= 0.0f) {
            att = v3(0.0f);
            dir = N;
            return false;
        }
        dir = L;
        float vdh = std::fmax(dot(V, H), 1e-4f);
        V3 f0 = compute_f0(bc, sp);
        V3 fres = eval_fresnel(vdh, f0);
        V3 ll = fr.to_local(L);
        float g1l = g1_ggx_aniso(ll, sp.alpha_x, sp.alpha_y);
        att = fres * g1l;
        att /= std::fmax(prob, 0.1f);
        return true;
    }
    bool scatter_transmission(V3 ray_in_dir, const HitRecord& rec, V3 bc, V3 N, V3 V, const ShadingParams& sp,
                              float prob, V3& att, V3& dir) const {   // :1473-1608
        bool thin = m.d.thin_walled != 0;
        float eta = thin ? (1.0f / sp.ior)
                         : (rec.relative_eta > 0.0f ? rec.relative_eta : (rec.front ? (1.0f / sp.ior) : sp.ior));
        V3 unit = normalize(ray_in_dir);
        Frame fr = shading_frame(rec, sp.anisotropic_rotation);
        bool rough = sp.roughness > 0.01f;
        V3 Ht;
        if (rough) {
            V3 vl = fr.to_local(V);
            float u1 = random_float();
            float u2 = random_float();
            V3 hl = sample_ggx_vndf_aniso(vl, sp.alpha_x, sp.alpha_y, u1, u2);
            Ht = fr.to_world(hl);
        } else {
            Ht = N;
        }
        if (dot(Ht, unit) > 0.0f) Ht = -Ht;
        float cos_t = std::fmin(dot(-unit, Ht), 1.0f);
        float sin_t = std::sqrt(std::fmax(0.0f, 1.0f - cos_t * cos_t));
        bool cannot = !thin && eta * sin_t > 1.0f;
        V3 d;
        bool is_refl;
        float fr_ = cannot ? 1.0f : fresnel_dielectric(cos_t, eta);
        if (fr_ > random_float()) {
            d = reflect(unit, Ht);
            is_refl = true;
        } else if (thin) {
            d = unit;
            is_refl = false;
        } else {
            d = refract(unit, Ht, eta);
            is_refl = false;
        }
        if (near_zero(d)) {
            d = reflect(unit, N);
            is_refl = true;
        }
        dir = normalize(d);
        V3 col;
        if (is_refl) {
            col = v3(1.0f);
        } else {
            V3 tint, sigma;
            resolve_transmission(bc, tint, sigma);
            col = tint;
        }
        att = col;
        if (rough) {
            V3 ll = fr.to_local(dir);
            ll.z = std::fabs(ll.z);
            att *= g1_ggx_aniso(ll, sp.alpha_x, sp.alpha_y);
        }
        att /= std::fmax(prob, 0.1f);
        return true;
    }
    bool scatter_clearcoat(const HitRecord& rec, V3 N, V3 V, const ShadingParams& sp, float prob, V3& att,
                           V3& dir) const {   // :1623-1678
        Frame fr = clearcoat_frame(rec);
        V3 cn = fr.n;
        if (dot(cn, V) <= 0.0f) {
            att = v3(0.0f);
            dir = N;
            return false;
        }
        V3 vl = fr.to_local(V);
        float u1 = random_float();
        float u2 = random_float();
        V3 hl = sample_ggx_vndf_aniso(vl, sp.clearcoat_alpha, sp.clearcoat_alpha, u1, u2);
        V3 H = fr.to_world(hl);
        V3 L = reflect(-V, H);
        if (dot(L, N) <= 0.0f || dot(L, cn) <= 0.0f) {
            att = v3(0.0f);
            dir = N;
            return false;
        }
        dir = L;
        float cc_ndl = std::fmax(dot(cn, L), 1e-4f);
        float cc_vdh = std::fmax(dot(V, H), 1e-4f);
        float fres = sp.clearcoat_f0 + (1.0f - sp.clearcoat_f0) * schlick_weight(cc_vdh);
        float g1l = smith_g1(cc_ndl, sp.clearcoat_alpha);
        att = v3(fres * g1l);
        att /= std::fmax(prob, 0.1f);
        return true;
    }
    bool scatter_multiscatter(const HitRecord&, V3 bc, V3 N, V3 V, const ShadingParams& sp, float prob, V3& att,
                              V3& dir) const {   // :1688-1709
        V3 sd = N + random_unit_vector();
        if (near_zero(sd)) sd = N;
        sd = normalize(sd);
        dir = sd;
        V3 L = sd;
        float ndv = std::fmax(dot(N, V), 1e-3f);
        float ndl = std::fmax(dot(N, L), 1e-3f);
        V3 f0 = compute_f0(bc, sp);
        V3 weight = multiscatter_weight(f0, sp, ndv, ndl);
        att = weight / std::fmax(prob, 0.05f);
        return true;
    }

    // Sample (:893-997). Returns false for "null".
    bool sample(V3 V, const HitRecord& rec, BsdfSample& out, int& lobe_out) const {
        V3 att, wo;
        int lobe = -1;
        lobe_out = -1;
        if (!scatter_internal(-V, rec, att, wo, lobe)) {
            lobe_out = lobe;
            return false;
        }
        lobe_out = lobe;
        float ndwo = dot(rec.n, wo);
        out.has_next_absorption = false;
        out.transition = 0;
        if (lobe == kDiffTrans) {
            V3 fb = evaluate(V, wo, rec);
            float pb = pdf(V, wo, rec);
            if (pb <= 0.0f) {
                out.wo = wo; out.f = att; out.pdf = 1.0f; out.is_delta = true;
                return true;
            }
            out.wo = wo; out.f = fb; out.pdf = pb; out.is_delta = false;
            return true;
        }
        if (lobe == kTransmission) {
            if (ndwo < 0.0f && !m.d.thin_walled) {
                V3 tint, sigma;
                resolve_transmission(base(), tint, sigma);
                bool has_sigma = sigma.x > 0.0f || sigma.y > 0.0f || sigma.z > 0.0f;
                if (rec.front && has_sigma) {
                    out.has_next_absorption = true;
                    out.next_absorption = sigma;
                } else if (!rec.front) {
                    out.has_next_absorption = true;
                    out.next_absorption = v3(0.0f);
                }
                out.transition = rec.front ? 1 : 2;
            }
            out.wo = wo; out.f = att; out.pdf = 1.0f; out.is_delta = true;
            return true;
        }
        if (ndwo <= 0.0f) return false;
        const ShadingParams& sp = m.sp;
        bool nd_spec = lobe == kSpecular && sp.alpha <= kDeltaAlpha;
        bool nd_coat = lobe == kClearcoat && sp.clearcoat_alpha <= kDeltaAlpha;
        if (nd_spec || nd_coat) {
            out.wo = wo; out.f = att; out.pdf = 1.0f; out.is_delta = true;
            return true;
        }
        out.wo = wo;
        out.f = evaluate(V, wo, rec);
        out.pdf = pdf(V, wo, rec);
        out.is_delta = false;
        return true;
    }

    // ShadowTransmittance (:560-584)
    V3 shadow_transmittance(V3 wi, const HitRecord& rec) const {
        float st = m.d.spec_trans;   // SpecTrans.Value (unclamped read, as the reference)
        if (st <= 0.0f) return v3(0.0f);
        float ior = std::fmax(m.d.ior, 1.0001f);
        float eta = 1.0f / ior;
        float c = std::fmin(std::fabs(dot(wi, rec.n)), 1.0f);
        float fr = fresnel_dielectric(c, eta);
        V3 tint, sigma;
        resolve_transmission(base(), tint, sigma);
        return st * (1.0f - fr) * tint;
    }
    V3 shadow_absorption() const {   // :609-614
        V3 tint, sigma;
        resolve_transmission(base(), tint, sigma);
        return sigma;
    }
    bool dielectric_ior(float& ior) const {   // :620-632
        if (m.d.thin_walled || m.d.spec_trans <= 0.0f) {
            ior = 1.0f;
            return false;
        }
        ior = std::fmax(m.d.ior, 1.0001f);
        return true;
    }
};

// ---------------------------------------------------------------------------
// Lights (Lights/*.cs)
// ---------------------------------------------------------------------------
struct LightSample {
    bool in_shadow;
    V3 color, dir;
    float dist;
};

struct Scene;
static V3 shadow_transmittance(const Scene& sc, const Ray& ray, float tmin, float tmax, int max_bounces = 8);

struct Light {
    int type = 0;   // 0 geometry-quad, 1 geometry-mesh, 2 geometry-triangle, 3 area, 4 directional,
                    // 5 geometry-sphere (cone sampled), 6 sphere light
    int shadow_samples = 1;
    int sqrt_samples = 1;
    float inv_sqrt = 1.0f;
    bool is_delta = false;
    int emissive_material = -1;   // GeometryLight.Material / AreaLight.ProxyMaterial
    const Quad* quad = nullptr;
    const Mesh* mesh = nullptr;
    // area light
    V3 corner{}, u{}, v{}, color{}, normal{};
    float intensity = 0.0f, area = 0.0f, soft_radius = 0.0f;
    // directional
    V3 direction{};
    float angular_radius = 0.0f, cos_angular = 1.0f, solid_angle = 0.0f;
    V3 rep_point{};
    float rep_area = 0.0f;
    V3 center{};   // sphere lights
    float radius = 0.0f;
};   // type 7: EnvironmentLight over the flat sky (colour in `color`)

struct Scene {
    std::vector<Material> mats;
    std::vector<std::unique_ptr<Hittable>> owned;
    std::vector<std::unique_ptr<Mesh>> meshes;
    std::vector<const Hittable*> objects;      // world list in entity order (SceneLoader.cs:446)
    std::vector<const Hittable*> bvh_objects;  // finite objects, partitioned by the top-level build
    std::vector<std::unique_ptr<BvhNode>> arena;
    std::unique_ptr<BvhNode> top;
    HittableList world;
    bool top_is_bvh = false;
    std::vector<Light> lights;
    std::vector<int> emitter_to_light;         // material index -> light index, -1 if none
    int rr_min_bounces = 3;
    float rr_min_survival = 0.1f;
    float mean_irradiance = 0.0f;
    // camera
    V3 cam_origin{}, cam_llc{}, cam_h{}, cam_v{};
    RtCameraDesc cam_desc{};
    float lens_radius = 0.0f;
    // medium
    bool has_medium = false;
    V3 sigma_a{}, sigma_s{}, sigma_t{};
    float hg_g = 0.0f;
    V3 sky{};            // flat sky radiance
    int env_light = -1;  // its EnvironmentLight
    std::vector<float> pick_cdf[2], pick_pdf[2];   // LightDistribution: power, uniform
    std::vector<const Hittable*> entity_ptr;   // entity index -> leaf hittable

    bool world_hit(const Ray& r, float tmin, float tmax, HitRecord& rec) const { return world.hit(r, tmin, tmax, rec); }
};

static float light_approx_power(const Light& l, const AABB& bounds, const Scene& sc) {
    if (l.type == 6) return 4.0f * kPi * luminance(l.color) * l.intensity;   // SphereLight.ApproximatePower (:79-80)
    if (l.type == 7) {   // EnvironmentLight.ApproximatePower (:37-52)
        V3 e = bounds.mx - bounds.mn;
        float cs = 0.5f * (e.x * e.y + e.y * e.z + e.x * e.z);
        return kPi * luminance(l.color) * cs;
    }
    if (l.type <= 2 || l.type == 5) {   // GeometryLight.ApproximatePower (:116-120)
        const Material& m = sc.mats[l.emissive_material];
        V3 em = v3(m.d.base_color[0], m.d.base_color[1], m.d.base_color[2]) * std::fmax(m.d.intensity, 0.0f);
        return kPi * l.rep_area * luminance(em);
    }
    if (l.type == 3) return kPi * l.area * luminance(l.color) * l.intensity;   // AreaLight.cs:111-112
    V3 ext = bounds.mx - bounds.mn;                                            // DirectionalLight.cs:82-88
    float radius = 0.5f * length(ext);
    float cross_section = kPi * radius * radius;
    return luminance(l.color) * l.intensity * cross_section;
}

// Sphere.LocalToWorld (Sphere.cs:230-246, the same frame as SphereLight's and
// DirectionalLight's) of a cone direction: cosTheta = 1 - xi1 (1 - cosMax),
// phi = 2 pi xi2 (Sphere.cs:160-169, SphereLight.cs:87-96).
static V3 cone_dir(V3 w, float cos_max, float xi1, float xi2) {
    float ct = 1.0f - xi1 * (1.0f - cos_max);
    float st = std::sqrt(std::fmax(0.0f, 1.0f - ct * ct));
    float phi = 2.0f * kPi * xi2;
    V3 loc = v3(st * std::cos(phi), st * std::sin(phi), ct);
    V3 uu, vv;
    if (w.z < -0.999f) {
        uu = v3(0, -1, 0);
        vv = v3(-1, 0, 0);
    } else {
        float a = 1.0f / (1.0f + w.z);
        float b = -w.x * w.y * a;
        uu = v3(1.0f - w.x * w.x * a, b, -w.x);
        vv = v3(b, 1.0f - w.y * w.y * a, -w.y);
    }
    V3 res = loc.x * uu + loc.y * vv + loc.z * w;
    float l2 = length_sq(res);
    return l2 > 1e-8f ? res / std::sqrt(l2) : w;
}

// Sphere.SolidAnglePdf (:205-226) = SphereLight.PdfSolidAngle (:179-200).
static float sphere_cone_pdf(V3 center, float radius, V3 p, V3 wi) {
    V3 tc = center - p;
    float d2 = length_sq(tc);
    float r2 = radius * radius;
    if (d2 <= r2) return 1.0f / (4.0f * kPi);
    float cmax = std::sqrt(std::fmax(0.0f, 1.0f - r2 / d2));
    float wl = length(wi);
    if (wl < kEps) return 0.0f;
    float dist = std::sqrt(d2);
    V3 wd = tc / dist;
    float ct = dot(wi, wd) / wl;
    if (ct < cmax) return 0.0f;
    float sa = 2.0f * kPi * (1.0f - cmax);
    return sa > kEps ? 1.0f / sa : 0.0f;
}

// GeometryLight.ComputeAreaSample (:149-190) for quads / triangles / meshes,
// GeometryLight.ComputeSolidAngleSample (:202-238) for spheres,
// SphereLight.IlluminateAndTestStratified (:72-141),
// AreaLight.IlluminateAndTestStratified (:129-178), DirectionalLight (:102-160).
static LightSample illuminate(const Scene& sc, const Light& l, V3 hit_p, V3 surf_n, int s) {
    if (l.type == 7) {   // EnvironmentLight.IlluminateAndTest (:54-90), FlatSky.ImportanceSample
        V3 dir = random_unit_vector();
        float pdf = 1.0f / (4.0f * kPi);
        if (length_sq(surf_n) > 0.0f && dot(surf_n, dir) <= 0.0f) return {true, v3(0.0f), dir, kInf};
        V3 so = offset_origin(hit_p, surf_n);
        V3 tr = shadow_transmittance(sc, Ray(so, dir), kEps, kInf);
        if (near_zero(tr)) return {true, v3(0.0f), dir, kInf};
        return {false, l.color * tr / (pdf * (float)l.shadow_samples), dir, kInf};
    }
    if (l.type == 5) {
        int su = s % l.sqrt_samples, sv = s / l.sqrt_samples;   // Sphere.SampleSolidAngleStratified
        float inv = 1.0f / (float)l.sqrt_samples;
        float xi1 = ((float)su + random_float()) * inv;
        float xi2 = ((float)sv + random_float()) * inv;
        V3 tc = l.center - hit_p;   // Sphere.SampleSolidAngleCore (:137-200)
        float dist_sq = length_sq(tc);
        float r_sq = l.radius * l.radius;
        V3 sp, nrm;
        float pdf;
        if (dist_sq <= r_sq) {
            V3 pu = random_unit_vector();
            sp = l.center + pu * l.radius;
            nrm = pu;
            pdf = 1.0f / (4.0f * kPi);
        } else {
            float dist = std::sqrt(dist_sq);
            V3 wd = tc / dist;
            float cmax = std::sqrt(std::fmax(0.0f, 1.0f - r_sq / dist_sq));
            V3 dw = cone_dir(wd, cmax, xi1, xi2);
            V3 oc = hit_p - l.center;
            float b = dot(oc, dw);
            float c = length_sq(oc) - r_sq;
            float disc = b * b - c;
            float t;
            if (disc <= 0.0f) {
                t = -b;
            } else {
                float sq = std::sqrt(disc);
                t = -b - sq;
                if (t < kEps) t = -b + sq;
            }
            sp = hit_p + t * dw;
            nrm = normalize(sp - l.center);
            float sa = 2.0f * kPi * (1.0f - cmax);
            pdf = sa > kEps ? 1.0f / sa : 0.0f;
        }
        if (pdf <= 0.0f) return {true, v3(0.0f), v3(0, 1, 0), 0.0f};
        V3 to_l = sp - hit_p;
        float d2 = length_sq(to_l);
        if (d2 < kEps * kEps) return {true, v3(0.0f), v3(0, 1, 0), 0.0f};
        float dist = std::sqrt(d2);
        V3 dir = to_l / dist;
        float cos_l = std::fmax(0.0f, dot(-dir, nrm));
        if (cos_l <= 0.0f) return {false, v3(0.0f), dir, dist};
        V3 so = offset_origin(hit_p, surf_n);
        Ray sr(so, dir);
        float tmax = length(sp - so) - kEps;
        V3 tr = shadow_transmittance(sc, sr, kEps, tmax);
        if (near_zero(tr)) return {true, v3(0.0f), dir, dist};
        const Material& m = sc.mats[l.emissive_material];
        V3 em = v3(m.d.base_color[0], m.d.base_color[1], m.d.base_color[2]) * std::fmax(m.d.intensity, 0.0f);
        float atten = 1.0f / (pdf * (float)l.shadow_samples);
        return {false, em * atten * tr, dir, dist};
    }
    if (l.type == 6) {
        V3 tc = l.center - hit_p;
        float dist_sq = length_sq(tc);
        if (dist_sq < kEps * kEps) return {true, v3(0.0f), v3(0, 1, 0), 0.0f};
        float dist = std::sqrt(dist_sq);
        V3 wd = tc / dist;
        float s2 = l.radius * l.radius / dist_sq;
        float cmax = s2 >= 1.0f ? -1.0f : std::sqrt(1.0f - s2);
        int su = s % l.sqrt_samples, sv = s / l.sqrt_samples;
        float xi1 = ((float)su + random_float()) * l.inv_sqrt;
        float xi2 = ((float)sv + random_float()) * l.inv_sqrt;
        V3 dw = cone_dir(wd, cmax, xi1, xi2);
        V3 oc = hit_p - l.center;
        float b = dot(oc, dw);
        float c = length_sq(oc) - l.radius * l.radius;
        float disc = b * b - c;
        if (disc < 0.0f) {
            V3 cp = l.center + normalize(dw) * l.radius;
            return {true, v3(0.0f), dw, length(cp - hit_p)};
        }
        float sq = std::sqrt(disc);
        float t = -b - sq;
        if (t < kEps) t = -b + sq;
        if (t < kEps) return {true, v3(0.0f), dw, 0.0f};
        V3 sp = hit_p + t * dw;
        V3 ln = (sp - l.center) / l.radius;
        float cos_l = std::fmax(0.0f, dot(-dw, ln));
        if (cos_l <= 0.0f) return {false, v3(0.0f), dw, t};
        V3 so = offset_origin(hit_p, surf_n);
        Ray sr(so, dw);
        float tmax = length(sp - so) - kEps;
        V3 tr = shadow_transmittance(sc, sr, kEps, tmax);
        if (near_zero(tr)) return {true, v3(0.0f), dw, t};
        float sa = 2.0f * kPi * (1.0f - cmax);
        float atten = l.intensity * sa / (float)l.shadow_samples;
        return {false, l.color * atten * tr, dw, t};
    }
    if (l.type <= 2) {
        V3 sp, ln;
        float uvx = 0.5f, uvy = 0.5f, area;
        if (l.type == 0) {   // Quad.SampleStratified (:99-109)
            int su = s % l.sqrt_samples, sv = s / l.sqrt_samples;
            float inv = 1.0f / (float)l.sqrt_samples;
            float uu = ((float)su + random_float()) * inv;
            float vv = ((float)sv + random_float()) * inv;
            sp = l.quad->q + uu * l.quad->u + vv * l.quad->v;
            ln = l.quad->normal;
            uvx = uu;
            uvy = vv;
            area = l.quad->area;
        } else {             // Mesh.SampleStratified (:151-171)
            const Mesh* m = l.mesh;
            int total = std::max(1, l.sqrt_samples * l.sqrt_samples);
            float stratum = 1.0f / (float)total;
            float jit = ((float)s + random_float()) * stratum;
            float target = clampf(jit, 0.0f, 0.9999999f) * m->total_area;
            int idx = m->pick_by_cdf(target);
            float x1 = random_float();
            float x2 = random_float();
            m->tris[idx]->sample_at(x1, x2, sp, ln, uvx, uvy);
            area = m->total_area;
        }
        (void)uvx;
        (void)uvy;
        V3 to_l = sp - hit_p;
        float d2 = length_sq(to_l);
        if (d2 < kEps * kEps) return {true, v3(0.0f), v3(0, 1, 0), 0.0f};
        float dist = std::sqrt(d2);
        V3 dir = to_l / dist;
        float cos_l = std::fmax(0.0f, dot(-dir, ln));
        if (cos_l <= 0.0f) return {true, v3(0.0f), dir, dist};
        V3 so = offset_origin(hit_p, surf_n);
        Ray sr(so, dir);
        float tmax = length(sp - so) - kEps;
        V3 tr = shadow_transmittance(sc, sr, kEps, tmax);
        if (near_zero(tr)) return {true, v3(0.0f), dir, dist};
        const Material& m = sc.mats[l.emissive_material];
        V3 em = v3(m.d.base_color[0], m.d.base_color[1], m.d.base_color[2]) * std::fmax(m.d.intensity, 0.0f);
        float att_d2 = d2;
        float atten = area * cos_l / (att_d2 * (float)l.shadow_samples);
        return {false, em * atten * tr, dir, dist};
    }
    if (l.type == 3) {
        int su = s % l.sqrt_samples, sv = s / l.sqrt_samples;
        float ru = ((float)su + random_float()) * l.inv_sqrt;
        float rv = ((float)sv + random_float()) * l.inv_sqrt;
        V3 sp = l.corner + ru * l.u + rv * l.v;
        V3 to_l = sp - hit_p;
        float d2 = length_sq(to_l);
        if (d2 < kEps * kEps) return {true, v3(0.0f), v3(0, 1, 0), 0.0f};
        float dist = std::sqrt(d2);
        V3 dir = to_l / dist;
        float cos_l = std::fmax(0.0f, dot(-dir, l.normal));
        if (cos_l <= 0.0f) return {false, v3(0.0f), dir, dist};
        V3 so = offset_origin(hit_p, surf_n);
        Ray sr(so, dir);
        float tmax = length(sp - so) - kEps;
        V3 tr = shadow_transmittance(sc, sr, kEps, tmax);
        if (near_zero(tr)) return {true, v3(0.0f), dir, dist};
        float att_d2 = d2;
        if (l.soft_radius > 0.0f) att_d2 = std::fmax(att_d2, l.soft_radius * l.soft_radius);
        float atten = l.intensity * l.area * cos_l / (att_d2 * (float)l.shadow_samples);
        return {false, l.color * atten * tr, dir, dist};
    }
    // Directional light
    V3 to_l;
    if (l.angular_radius > 0.0f) {
        int su = s % l.sqrt_samples, sv = s / l.sqrt_samples;
        float xi1 = ((float)su + random_float()) * l.inv_sqrt;
        float xi2 = ((float)sv + random_float()) * l.inv_sqrt;
        float ct = 1.0f - xi1 * (1.0f - l.cos_angular);
        float st = std::sqrt(std::fmax(0.0f, 1.0f - ct * ct));
        float phi = 2.0f * kPi * xi2;
        V3 w = -l.direction;
        V3 loc = v3(st * std::cos(phi), st * std::sin(phi), ct);
        V3 uu, vv;   // DirectionalLight.LocalToWorld (:192-213)
        if (w.z < -0.999f) {
            uu = v3(0, -1, 0);
            vv = v3(-1, 0, 0);
        } else {
            float a = 1.0f / (1.0f + w.z);
            float b = -w.x * w.y * a;
            uu = v3(1.0f - w.x * w.x * a, b, -w.x);
            vv = v3(b, 1.0f - w.y * w.y * a, -w.y);
        }
        V3 res = loc.x * uu + loc.y * vv + loc.z * w;
        float l2 = length_sq(res);
        to_l = l2 > 1e-8f ? res / std::sqrt(l2) : w;
    } else {
        to_l = -l.direction;
    }
    V3 so = offset_origin(hit_p, surf_n);
    Ray sr(so, to_l);
    V3 tr = shadow_transmittance(sc, sr, kEps, kInf);
    if (near_zero(tr)) return {true, v3(0.0f), to_l, kInf};
    float e = l.intensity / (float)l.shadow_samples;
    return {false, l.color * e * tr, to_l, kInf};
}

// ILight.PdfSolidAngle implementations.
static float light_pdf(const Light& l, V3 p, V3 wi) {
    if (l.type == 5 || l.type == 6) return sphere_cone_pdf(l.center, l.radius, p, wi);
    if (l.type == 7) return 1.0f / (4.0f * kPi);   // FlatSky.Pdf
    if (l.type == 0 || l.type == 1) {   // GeometryLight.PdfSolidAngle area fallback (:254-279)
        Ray r(p, wi);
        HitRecord rec;
        bool saved = t_counting;
        t_counting = false;
        bool h = l.type == 0 ? l.quad->hit(r, kEps, kInf, rec) : l.mesh->hit(r, kEps, kInf, rec);
        t_counting = saved;
        if (!h) return 0.0f;
        float cos_l = std::fabs(dot(-wi, rec.n));
        if (cos_l < 1e-6f) return 0.0f;
        float d2 = rec.t * rec.t;
        float area = l.rep_area;
        if (area < 1e-12f) return 0.0f;
        return d2 / (area * cos_l);
    }
    if (l.type == 3) {   // AreaLight.PdfSolidAngle (:189-226)
        float denom = dot(l.normal, wi);
        if (std::fabs(denom) < 1e-7f) return 0.0f;
        float t = dot(l.corner - p, l.normal) / denom;
        if (t <= kEps) return 0.0f;
        V3 hp = p + t * wi;
        V3 loc = hp - l.corner;
        float uu = dot(l.u, l.u), vv = dot(l.v, l.v), uv = dot(l.u, l.v);
        float det = uu * vv - uv * uv;
        if (det < 1e-12f) return 0.0f;
        float lu = dot(loc, l.u), lv = dot(loc, l.v);
        float a = (lu * vv - lv * uv) / det;
        float b = (lv * uu - lu * uv) / det;
        if (a < 0.0f || a > 1.0f || b < 0.0f || b > 1.0f) return 0.0f;
        float cos_l = std::fabs(denom);
        if (cos_l < 1e-6f) return 0.0f;
        return (t * t) / (l.area * cos_l);
    }
    if (l.type == 4) {   // DirectionalLight.PdfSolidAngle (:169-181)
        if (l.angular_radius <= 0.0f) return 0.0f;
        if (l.solid_angle <= 0.0f) return 0.0f;
        float wl = length(wi);
        if (wl < kEps) return 0.0f;
        float ct = dot(wi / wl, -l.direction);
        if (ct < l.cos_angular) return 0.0f;
        return 1.0f / l.solid_angle;
    }
    return 0.0f;
}

// Geometry/ShadowRay.cs:59-157
static V3 shadow_transmittance(const Scene& sc, const Ray& ray, float tmin, float tmax, int max_bounces) {
    if (t_counting) t_cnt.shadow_rays++;
    V3 thr = v3(1.0f);
    V3 o = ray.o, d = ray.d;
    float remaining = tmax;
    V3 sigma = v3(0.0f), entry{};
    bool in_med = false;
    for (int i = 0; i < max_bounces; i++) {
        HitRecord rec;
        Ray step(o, d);
        if (!sc.world_hit(step, tmin, remaining, rec)) return thr;
        const Material& m = sc.mats[rec.material];
        if (in_med) {
            float dd = length(rec.p - entry);
            thr = v3(thr.x * std::exp(-sigma.x * dd), thr.y * std::exp(-sigma.y * dd), thr.z * std::exp(-sigma.z * dd));
            in_med = false;
            if (near_zero(thr)) return v3(0.0f);
        }
        V3 t = m.is_emissive() ? v3(0.0f) : Disney(m).shadow_transmittance(d, rec);
        if (near_zero(t)) return v3(0.0f);
        thr *= t;
        if (near_zero(thr)) return v3(0.0f);
        if (rec.front) {
            V3 sg = m.is_emissive() ? v3(0.0f) : Disney(m).shadow_absorption();
            if (!near_zero(sg)) {
                in_med = true;
                entry = rec.p;
                sigma = sg;
            }
        }
        V3 on = dot(d, rec.n) >= 0.0f ? rec.n : -rec.n;
        o = offset_origin(rec.p, on);
        remaining -= rec.t + 2.0f * kEps;
        if (remaining <= tmin) return thr;
    }
    return v3(0.0f);
}

// ---------------------------------------------------------------------------
// The renderer (Rendering/Renderer.cs)
// ---------------------------------------------------------------------------
struct IorStack {   // Volumetrics/IorStack.cs
    float slots[8];
    int count = 0;
    float top() const { return count == 0 ? 1.0f : slots[count - 1]; }
    float enclosing() const { return count >= 2 ? slots[count - 2] : 1.0f; }
    void push(float ior) {
        if (count >= 8) {
            for (int i = 0; i < 7; i++) slots[i] = slots[i + 1];
            slots[7] = ior;
            return;
        }
        slots[count++] = ior;
    }
    void pop() {
        if (count == 0) return;
        count--;
    }
};

// ---------------------------------------------------------------------------
// Homogeneous medium and Henyey-Greenstein phase (Volumetrics/), as free
// functions of their parameters and uniform draws.
// ---------------------------------------------------------------------------
static V3 medium_transmittance(V3 sigma_t, float t) {   // HomogeneousMedium.Transmittance (:36-44)
    float d = std::fmin(std::fmax(t, 0.0f), 1e30f);
    return v3(std::exp(-sigma_t.x * d), std::exp(-sigma_t.y * d), std::exp(-sigma_t.z * d));
}
static float hg_evaluate(float g, V3 wo, V3 wi) {   // HenyeyGreensteinPhase.cs:23-30
    float mu = dot(wo, wi);
    float denom = 1.0f + g * g - 2.0f * g * mu;
    return kInv4Pi * (1.0f - g * g) / (denom * std::sqrt(denom));
}
static V3 hg_draw(float g, V3 wo, float u1, float u2, float& pdf) {   // HenyeyGreensteinPhase.cs:32-54
    float ct;
    if (std::fabs(g) < 1e-3f) {
        ct = 1.0f - 2.0f * u1;
    } else {
        float sqr = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
        ct = (1.0f + g * g - sqr * sqr) / (2.0f * g);
    }
    float st = std::sqrt(std::fmax(0.0f, 1.0f - ct * ct));
    float phi = 2.0f * kPi * u2;
    V3 w = wo;
    V3 a = std::fabs(w.x) > 0.9f ? v3(0, 1, 0) : v3(1, 0, 0);
    V3 v = normalize(cross(w, a));
    V3 u = cross(w, v);
    V3 wi = st * std::cos(phi) * u + st * std::sin(phi) * v + ct * w;
    wi = normalize(wi);
    pdf = hg_evaluate(g, wo, wi);
    return wi;
}
// HomogeneousMedium.Sample (:46-76): hero channel floor(3 u_ch), then the
// distance draw (taken only when that channel's sigma_t is positive).
template <class Draw>
static bool medium_draw(V3 sigma_t, V3 sigma_s, float tmax, float u_ch, Draw draw, float& t, V3& beta) {
    int ch = (int)(u_ch * 3.0f);
    if (ch > 2) ch = 2;
    float st = ch == 0 ? sigma_t.x : ch == 1 ? sigma_t.y : sigma_t.z;
    if (st <= 0.0f) {
        t = tmax;
        beta = v3(1.0f);
        return false;
    }
    float dist = -std::log(1.0f - draw()) / st;
    bool scattered = dist < tmax;
    t = scattered ? dist : tmax;
    V3 tr = medium_transmittance(sigma_t, t);
    V3 dens = scattered ? sigma_t * tr : tr;
    float pdf = (dens.x + dens.y + dens.z) / 3.0f;
    if (pdf < 1e-20f) pdf = 1.0f;
    beta = scattered ? (tr * sigma_s / pdf) : (tr / pdf);
    return scattered;
}

struct RenderCfg {
    int max_depth;
    float max_radiance, indirect_max;
    int mis_power;
    int rr_min_bounces;
    float rr_min_survival;
    int light_pick = 0;   // LightSamplingStrategy: 0 All, 1 Power, 2 Uniform
};

static inline V3 sanitize(V3 c) {   // Renderer.cs:917-923
    if (std::isnan(c.x) || std::isinf(c.x)) c.x = 0.0f;
    if (std::isnan(c.y) || std::isinf(c.y)) c.y = 0.0f;
    if (std::isnan(c.z) || std::isinf(c.z)) c.z = 0.0f;
    return vmax(c, v3(0.0f));
}

// The AOV probe of the camera path being traced (Renderer.cs:755-815), one
// per thread like the reference's [ThreadStatic] t_aovProbe; null while not
// capturing, so every hook is one test.
struct AovProbe {
    bool pending = false, have_depth = false, camera = false;
    float depth = -1.0f;
    V3 weight{}, tent_albedo{}, tent_normal{}, albedo{}, normal{};
    void reset() {
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
    void commit() {
        albedo = weight * tent_albedo;
        normal = tent_normal;
        pending = false;
    }
    void commit_as(V3 a, V3 n) {
        albedo = weight * a;
        normal = n;
        pending = false;
    }
};
static thread_local AovProbe* t_probe = nullptr;

static inline V3 clamp01(V3 v) {   // Renderer.Clamp01: Vector3.Clamp(v, Zero, One)
    return v3(std::fmin(std::fmax(v.x, 0.0f), 1.0f), std::fmin(std::fmax(v.y, 0.0f), 1.0f),
              std::fmin(std::fmax(v.z, 0.0f), 1.0f));
}

struct Tracer {
    const Scene& sc;
    RenderCfg cfg;

    float mis(float p, float q) const {   // Renderer.cs:1534-1543
        if (cfg.mis_power) {
            float p2 = p * p, q2 = q * q;
            return p2 / (p2 + q2 + 1e-30f);
        }
        return p / (p + q + 1e-30f);
    }
    V3 clamp_radiance(V3 c) const {   // :931-944
        c = sanitize(c);
        float lum = luminance(c);
        if (lum > cfg.max_radiance) c *= cfg.max_radiance / lum;
        return c;
    }
    V3 clamp_indirect(V3 c) const {   // :963-972
        c = sanitize(c);
        float lum = luminance(c);
        if (lum > cfg.indirect_max && lum > 0.0f) c *= cfg.indirect_max / lum;
        return c;
    }
    V3 weight_emission(V3 raw, int mat, const Ray& ray, float prev_pdf, bool prev_delta) const {   // :1549-1565
        if (prev_delta) return raw;
        int li = sc.emitter_to_light[mat];
        if (li >= 0) {
            float pl = light_pdf(sc.lights[li], ray.o, ray.d);
            if (prev_pdf + pl <= 1e-20f) return v3(0.0f);
            return raw * mis(prev_pdf, pl);
        }
        return raw;
    }

    // ComputeDirectLighting, strategy All (:1894-2036)
    // LightDistribution.Sample (LightDistribution.cs:104-122)
    int pick_light(float xi, float& pdf) const {
        const std::vector<float>& cdf = sc.pick_cdf[cfg.light_pick - 1];
        const std::vector<float>& pp = sc.pick_pdf[cfg.light_pick - 1];
        int n = (int)cdf.size();
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

    V3 direct_lighting(const HitRecord& rec, V3 view, const Disney& bsdf) const {
        V3 result = v3(0.0f);
        float view_term = shadow_terminator(rec.n, rec.n, view);   // ShadingNg == Normal (no normal maps)
        if (cfg.light_pick) {   // single-light picking (:1907-1974)
            if (sc.lights.empty()) return result;
            float p_pick;
            const Light& l = sc.lights[pick_light(random_float(), p_pick)];
            V3 acc = v3(0.0f);
            for (int s = 0; s < l.shadow_samples; s++) {
                LightSample ls = illuminate(sc, l, rec.p, rec.n, s);
                if (ls.in_shadow) continue;
                V3 brdf = bsdf.evaluate_direct(ls.dir, view, rec.n, rec);
                brdf *= view_term * shadow_terminator(rec.n, rec.n, ls.dir);
                if (brdf == v3(0.0f)) continue;
                V3 tr = v3(1.0f);
                if (sc.has_medium) {
                    float sd = std::isinf(ls.dist) || ls.dist >= kInf ? 1e30f : ls.dist;
                    tr = medium_tr(sd);
                }
                float w_nee = 1.0f;
                if (!l.is_delta) {
                    float p_bsdf = bsdf.pdf(view, ls.dir, rec);
                    if (p_bsdf > 0.0f) {
                        float p_nee = p_pick * light_pdf(l, rec.p, ls.dir);
                        w_nee = (p_nee + p_bsdf > 0.0f) ? mis(p_nee, p_bsdf) : 1.0f;
                    }
                }
                acc += w_nee * ls.color * brdf * tr;
            }
            if (p_pick > 0.0f) result += acc / p_pick;
            return result;
        }
        for (size_t li = 0; li < sc.lights.size(); li++) {
            const Light& l = sc.lights[li];
            V3 acc = v3(0.0f);
            for (int s = 0; s < l.shadow_samples; s++) {
                LightSample ls = illuminate(sc, l, rec.p, rec.n, s);
                if (ls.in_shadow) continue;
                V3 brdf = bsdf.evaluate_direct(ls.dir, view, rec.n, rec);
                brdf *= view_term * shadow_terminator(rec.n, rec.n, ls.dir);
                if (brdf == v3(0.0f)) continue;
                V3 tr = v3(1.0f);
                if (sc.has_medium) {
                    float sd = std::isinf(ls.dist) || ls.dist >= kInf ? 1e30f : ls.dist;
                    tr = medium_tr(sd);
                }
                float w_nee = 1.0f;
                if (!l.is_delta) {
                    float p_bsdf = bsdf.pdf(view, ls.dir, rec);
                    if (p_bsdf > 0.0f) {
                        float p_l = light_pdf(l, rec.p, ls.dir);
                        w_nee = (p_l + p_bsdf > 0.0f) ? mis(p_l, p_bsdf) : 1.0f;
                    }
                }
                acc += w_nee * ls.color * brdf * tr;
            }
            result += acc;
        }
        return result;
    }

    V3 medium_tr(float t) const { return medium_transmittance(sc.sigma_t, t); }
    float hg_eval(V3 wo, V3 wi) const { return hg_evaluate(sc.hg_g, wo, wi); }
    V3 hg_sample(V3 wo, float& pdf) const {
        float u1 = random_float(), u2 = random_float();
        return hg_draw(sc.hg_g, wo, u1, u2, pdf);
    }
    // ComputeDirectLightingMedium, strategy All (:2162-2203)
    V3 direct_lighting_medium(V3 p, V3 wo) const {
        V3 result = v3(0.0f);
        if (cfg.light_pick) {   // single-light picking in the volumetric path (:2110-2160)
            if (sc.lights.empty()) return result;
            float p_pick;
            const Light& l = sc.lights[pick_light(random_float(), p_pick)];
            V3 acc = v3(0.0f);
            for (int s = 0; s < l.shadow_samples; s++) {
                LightSample ls = illuminate(sc, l, p, v3(0.0f), s);
                if (ls.in_shadow) continue;
                float ph = hg_eval(wo, ls.dir);
                float sd = ls.dist >= kInf ? 1e30f : ls.dist;
                V3 tr = medium_tr(sd);
                float w_nee = 1.0f;
                if (!l.is_delta) {
                    float pp = hg_eval(wo, ls.dir);
                    if (pp > 0.0f) {
                        float p_nee = p_pick * light_pdf(l, p, ls.dir);
                        if (p_nee + pp > 0.0f) w_nee = mis(p_nee, pp);
                    }
                }
                acc += w_nee * ls.color * ph * tr;
            }
            if (p_pick > 0.0f) result += acc / p_pick;
            return result;
        }
        for (size_t li = 0; li < sc.lights.size(); li++) {
            const Light& l = sc.lights[li];
            V3 acc = v3(0.0f);
            for (int s = 0; s < l.shadow_samples; s++) {
                LightSample ls = illuminate(sc, l, p, v3(0.0f), s);
                if (ls.in_shadow) continue;
                float ph = hg_eval(wo, ls.dir);
                float sd = ls.dist >= kInf ? 1e30f : ls.dist;
                V3 tr = medium_tr(sd);
                float w_nee = 1.0f;
                if (!l.is_delta) {
                    float pp = hg_eval(wo, ls.dir);   // Phase.Pdf == Evaluate for HG
                    if (pp > 0.0f) {
                        float pl = light_pdf(l, p, ls.dir);
                        if (pl + pp > 0.0f) w_nee = mis(pl, pp);
                    }
                }
                acc += w_nee * ls.color * ph * tr;
            }
            result += acc;
        }
        return result;
    }
    // HomogeneousMedium.Sample (:46-76)
    bool medium_sample(float tmax, float& t, V3& beta) const {
        float u_ch = random_float();
        return medium_draw(sc.sigma_t, sc.sigma_s, tmax, u_ch, [&] { return random_float(); }, t, beta);
    }
    static V3 beer_lambert(V3 rad, V3 sigma, float t) {   // :1791-1800
        if (sigma.x <= 0.0f && sigma.y <= 0.0f && sigma.z <= 0.0f) return rad;
        if (std::isinf(t) && t > 0) return v3(0.0f);
        if (t <= 0.0f) return rad;
        return rad * v3(sigma.x > 0.0f ? std::exp(-sigma.x * t) : 1.0f, sigma.y > 0.0f ? std::exp(-sigma.y * t) : 1.0f,
                        sigma.z > 0.0f ? std::exp(-sigma.z * t) : 1.0f);
    }

    V3 rr_and_recurse(V3 att, V3 beta, int depth, V3 emitted, V3 direct, bool& killed, V3& next_beta) const {
        next_beta = beta * att;
        int used = cfg.max_depth - depth;
        killed = false;
        if (used >= cfg.rr_min_bounces) {
            float q = std::fmax(next_beta.x, std::fmax(next_beta.y, next_beta.z));
            q = std::fmax(q, cfg.rr_min_survival);
            q = std::fmin(q, 0.95f);
            if (random_float() > q) {
                killed = true;
                return emitted + direct;
            }
            float inv = 1.0f / q;
            att *= inv;
            next_beta *= inv;
        }
        return att;
    }

    // ShadeSurface (:1008-1228) + ShadeSampleBounce (:1235-1383)
    V3 shade_surface(const Ray& ray, HitRecord& rec, int depth, float prev_pdf, bool prev_delta, V3 cur_abs,
                     V3 beta, IorStack& iors) const {
        const Material& m = sc.mats[rec.material];
        if (t_probe && t_probe->pending) {   // AOV tentative surface (:1051-1054): AovAlbedo is the colour
            t_probe->tent_normal = rec.n;
            t_probe->tent_albedo = clamp01(v3(m.d.base_color[0], m.d.base_color[1], m.d.base_color[2]));
        }
        V3 emitted = v3(0.0f);
        if (m.is_emissive()) {   // Emissive.Emit (:86-90)
            if (rec.front) {
                V3 raw = v3(m.d.base_color[0], m.d.base_color[1], m.d.base_color[2]) * std::fmax(m.d.intensity, 0.0f);
                if (raw.x > 0.0f || raw.y > 0.0f || raw.z > 0.0f)
                    emitted = weight_emission(raw, rec.material, ray, prev_pdf, prev_delta);
            }
        }
        V3 view = normalize(-ray.d);
        if (m.is_emissive()) return emitted;   // NeedsDirectLighting false, Sample null, Scatter false
        Disney bsdf(m);
        float mat_ior;
        if (bsdf.dielectric_ior(mat_ior) && mat_ior > 0.0f)
            rec.relative_eta = rec.front ? (iors.top() / mat_ior) : (mat_ior / iors.enclosing());
        V3 direct = direct_lighting(rec, view, bsdf);
        BsdfSample s;
        int lobe;
        if (bsdf.sample(view, rec, s, lobe)) {
            // ShadeSampleBounce
            V3 att;
            if (s.is_delta) {
                att = s.f;
            } else {
                float ndwo = dot(rec.n, s.wo);
                float a = std::fabs(ndwo);
                if (a <= 0.0f || s.pdf <= 0.0f) return emitted + direct;
                att = s.f * a / s.pdf;
            }
            if (t_probe && t_probe->pending) {   // AOV first-non-delta decision (:1271-1277)
                if (s.is_delta) t_probe->weight = t_probe->weight * clamp01(s.f);
                else t_probe->commit();
            }
            bool killed;
            V3 nb;
            V3 r = rr_and_recurse(att, beta, depth, emitted, direct, killed, nb);
            if (killed) return r;
            att = r;
            V3 off = dot(s.wo, rec.n) >= 0.0f ? rec.n : -rec.n;
            Ray sc_ray(offset_origin(rec.p, off), s.wo);
            float next_pdf = s.is_delta ? 0.0f : s.pdf;
            V3 next_abs = s.has_next_absorption ? s.next_absorption : cur_abs;
            V3 ind;
            if (s.transition != 0) {
                IorStack ni = iors;
                if (s.transition == 1) {
                    float pi;
                    ni.push(bsdf.dielectric_ior(pi) ? pi : iors.top());
                } else {
                    ni.pop();
                }
                ind = trace(sc_ray, depth - 1, next_pdf, s.is_delta, ni, next_abs, nb);
            } else {
                ind = trace(sc_ray, depth - 1, next_pdf, s.is_delta, iors, next_abs, nb);
            }
            ind = sanitize(ind);
            V3 contrib = att * ind;
            if (depth == cfg.max_depth) contrib = clamp_indirect(contrib);
            return emitted + direct + contrib;
        }
        // Sample returned null: legacy Scatter path (:1127-1225)
        V3 att, dir;
        int lobe2;
        if (bsdf.scatter_internal(ray.d, rec, att, dir, lobe2)) {
            if (t_probe && t_probe->pending) t_probe->commit();   // (:1139-1145); Disney is not delta-scatter
            bool killed;
            V3 nb;
            V3 r = rr_and_recurse(att, beta, depth, emitted, direct, killed, nb);
            if (killed) return r;
            att = r;
            Ray sc_ray(rec.p, dir);
            IorStack ni = iors;
            float si;
            if (bsdf.dielectric_ior(si) && dot(sc_ray.d, rec.n) < 0.0f) {
                if (rec.front) ni.push(si);
                else ni.pop();
            }
            V3 ind = trace(sc_ray, depth - 1, 0.0f, false, ni, cur_abs, nb);
            ind = sanitize(ind);
            V3 contrib = att * ind;
            if (depth == cfg.max_depth) contrib = clamp_indirect(contrib);
            return emitted + direct + contrib;
        }
        return emitted + direct;
    }

    // SampleSky (:1820-1861) for a flat sky: the AOV miss commit, then the
    // radiance, MIS-weighted against the EnvironmentLight unless the bounce
    // before was delta.
    V3 sample_sky(float prev_pdf, bool prev_delta) const {
        if (t_probe && t_probe->pending) t_probe->commit_as(clamp01(sc.sky), v3(0.0f));   // :1849-1850
        if (prev_delta || sc.env_light < 0) return sc.sky;
        float pl = 1.0f / (4.0f * kPi);
        if (prev_pdf + pl <= 1e-20f) return v3(0.0f);
        return sc.sky * mis(prev_pdf, pl);
    }

    // TraceRay (:1581-1783)
    V3 trace(const Ray& ray, int depth, float prev_pdf, bool prev_delta, IorStack& iors, V3 cur_abs, V3 beta) const {
        if (depth <= 0) return v3(0.0f);
        float bmax = std::fmax(beta.x, std::fmax(beta.y, beta.z));
        if (bmax < 1e-4f) return v3(0.0f);
        HitRecord rec;
        bool saved = t_counting;
        if (t_counting) {
            t_cnt.closest_rays++;
            t_cnt.segments++;
        }
        bool hit = sc.world_hit(ray, kEps, kInf, rec);
        t_counting = saved;
        if (t_probe) {   // AOV depth: the camera ray's first surface hit (:1657-1662)
            if (t_probe->camera && hit && t_probe->pending && !t_probe->have_depth) {
                t_probe->depth = rec.t * length(ray.d);
                t_probe->have_depth = true;
            }
            t_probe->camera = false;
        }
        if (!sc.has_medium) {
            V3 res = !hit ? sample_sky(prev_pdf, prev_delta)
                          : shade_surface(ray, rec, depth, prev_pdf, prev_delta, cur_abs, beta, iors);
            return beer_lambert(res, cur_abs, hit ? rec.t : INFINITY);
        }
        float tmax = hit ? rec.t : 1e30f;
        float tmed;
        V3 mb;
        bool scattered = medium_sample(tmax, tmed, mb);
        if (scattered) {
            V3 p = ray.o + ray.d * tmed;
            if (t_probe && t_probe->pending) {   // AOV at a medium scatter (:1716-1724)
                if (!t_probe->have_depth) {
                    t_probe->depth = tmed * length(ray.d);
                    t_probe->have_depth = true;
                }
                t_probe->commit_as(v3(1.0f), v3(0.0f));
            }
            V3 lnee = direct_lighting_medium(p, ray.d);
            V3 lind = v3(0.0f);
            V3 mthr = beta * mb;
            int used = cfg.max_depth - depth;
            float scale = 1.0f;
            bool kill = false;
            if (used >= cfg.rr_min_bounces) {
                float q = std::fmax(mthr.x, std::fmax(mthr.y, mthr.z));
                q = std::fmax(q, cfg.rr_min_survival);
                q = std::fmin(q, 0.95f);
                if (random_float() > q) kill = true;
                else scale = 1.0f / q;
            }
            if (!kill) {
                float ppdf;
                V3 wi = hg_sample(ray.d, ppdf);
                float pv = hg_eval(ray.d, wi);
                float pw = ppdf > 1e-20f ? pv / ppdf : 0.0f;
                V3 nthr = mthr * (pw * scale);
                lind = pw * scale * trace(Ray(p, wi), depth - 1, ppdf, false, iors, cur_abs, nthr);
            }
            return beer_lambert(mb * (lnee + lind), cur_abs, tmed);
        }
        V3 so = !hit ? mb * sample_sky(prev_pdf, prev_delta)
                     : mb * shade_surface(ray, rec, depth, prev_pdf, prev_delta, cur_abs, beta * mb, iors);
        return beer_lambert(so, cur_abs, hit ? rec.t : INFINITY);
    }
};

// Per-pixel loop body (Renderer.cs:600-720), Sobol branch.
static V3 render_pixel(const Scene& sc, const Tracer& tr, int i, int j, int width, int height, int spp, int spp_offset) {
    V3 cum = v3(0.0f);
    uint32_t seed = (uint32_t)(i * 73856093) ^ (uint32_t)(j * 19349663);   // :615
    for (int s = spp_offset; s < spp_offset + spp; s++) {
        begin_pixel_sample(seed, (uint32_t)s);
        float ju = random_float();
        float jv = random_float();
        float u = ((float)i + ju) / (float)width;
        float v = ((float)(height - j - 1) + jv) / (float)height;
        // Camera.GetRayWithDifferentials pinhole (Camera.cs:127-139)
        V3 target = sc.cam_llc + u * sc.cam_h + v * sc.cam_v;
        Ray ray(sc.cam_origin, target - sc.cam_origin);
        IorStack iors;
        if (t_counting) t_cnt.samples++;
        V3 smp = tr.trace(ray, tr.cfg.max_depth, 0.0f, true, iors, v3(0.0f), v3(1.0f));
        end_pixel_sample();
        smp = tr.clamp_radiance(smp);
        cum += smp;
    }
    return cum;
}

// render_pixel with CaptureAccumulator (Renderer.cs:817-882): the even/odd
// halves of the clamped samples and of the probe's features. Writes the
// pixel's means into the 23-value record `o` (beauty, beauty A, beauty B,
// albedo A, albedo B, normal A, normal B, depth A, depth B).
static void render_pixel_capture(const Scene& sc, const Tracer& tr, int i, int j, int width, int height, int spp,
                                 int spp_offset, float* o) {
    V3 cum = v3(0.0f), sa = v3(0.0f), sb = v3(0.0f), aa = v3(0.0f), ab = v3(0.0f), na = v3(0.0f), nb = v3(0.0f);
    float da = 0.0f, db = 0.0f;
    int ca = 0, cb = 0;
    AovProbe probe;
    t_probe = &probe;
    uint32_t seed = (uint32_t)(i * 73856093) ^ (uint32_t)(j * 19349663);
    for (int s = 0; s < spp; s++) {
        begin_pixel_sample(seed, (uint32_t)(spp_offset + s));
        float ju = random_float();
        float jv = random_float();
        float u = ((float)i + ju) / (float)width;
        float v = ((float)(height - j - 1) + jv) / (float)height;
        V3 target = sc.cam_llc + u * sc.cam_h + v * sc.cam_v;
        Ray ray(sc.cam_origin, target - sc.cam_origin);
        IorStack iors;
        probe.reset();
        V3 smp = tr.trace(ray, tr.cfg.max_depth, 0.0f, true, iors, v3(0.0f), v3(1.0f));
        end_pixel_sample();
        smp = tr.clamp_radiance(smp);
        cum += smp;
        if (probe.pending) probe.commit();
        if ((s & 1) == 0) {
            sa += smp;
            aa += probe.albedo;
            na += probe.normal;
            if (probe.have_depth) {
                da += probe.depth;
                ca++;
            }
        } else {
            sb += smp;
            ab += probe.albedo;
            nb += probe.normal;
            if (probe.have_depth) {
                db += probe.depth;
                cb++;
            }
        }
    }
    t_probe = nullptr;
    int n_a = (spp + 1) / 2, n_b = spp / 2;
    auto put3 = [&](int at, V3 c) {
        o[at] = c.x;
        o[at + 1] = c.y;
        o[at + 2] = c.z;
    };
    put3(0, cum / (float)spp);
    V3 ma = sa / (float)n_a;
    put3(3, ma);
    put3(6, n_b > 0 ? sb / (float)n_b : ma);
    V3 a2 = aa / (float)n_a;
    put3(9, a2);
    put3(12, n_b > 0 ? ab / (float)n_b : a2);
    V3 n2 = na / (float)n_a;
    put3(15, n2);
    put3(18, n_b > 0 ? nb / (float)n_b : n2);
    float dA = ca > 0 ? da / (float)ca : -1.0f;
    o[21] = dA;
    o[22] = n_b > 0 ? (cb > 0 ? db / (float)cb : -1.0f) : dA;
}

}  // namespace oracle

// ===========================================================================
// C API for the test harness (ctypes)
// ===========================================================================
using namespace oracle;

namespace {

void build_camera(Scene& sc, const RtCameraDesc& c, float aspect) {   // Camera.cs:26-51
    sc.cam_desc = c;
    V3 from = v3(c.look_from[0], c.look_from[1], c.look_from[2]);
    V3 at = v3(c.look_at[0], c.look_at[1], c.look_at[2]);
    V3 vup = v3(c.vup[0], c.vup[1], c.vup[2]);
    float theta = c.vfov_deg * kPi / 180.0f;   // MathUtils.DegreesToRadians
    float h = std::tan(theta / 2.0f);
    float vh = 2.0f * h;
    float vw = aspect * vh;
    V3 w = normalize(from - at);
    if (length_sq(cross(w, vup)) < 1e-8f) vup = std::fabs(w.x) < 0.9f ? v3(1, 0, 0) : v3(0, 0, 1);
    V3 u = normalize(cross(vup, w));
    V3 v = cross(w, u);
    float fd = c.focus_dist;
    sc.cam_origin = from;
    sc.cam_h = fd * vw * u;
    sc.cam_v = fd * vh * v;
    sc.cam_llc = from - sc.cam_h / 2.0f - sc.cam_v / 2.0f - fd * w;
    sc.lens_radius = c.aperture / 2.0f;
}

thread_local char g_err[256];

}  // namespace

extern "C" {

const char* or_last_error(void) { return g_err; }

float or_sobol(uint32_t idx, uint32_t dim, uint32_t seed) { return sobol_sample(idx, dim, seed); }

int or_sobol_batch(const uint32_t* idx, const uint32_t* dim, const uint32_t* seed, int64_t n, float* out) {
    for (int64_t i = 0; i < n; i++) out[i] = sobol_sample(idx[i], dim[i], seed[i]);
    return 0;
}

// Medium and phase test entry points (VolumetricsTests.cs).
float or_hg_eval(float g, const float* wo, const float* wi) {
    return hg_evaluate(g, v3(wo[0], wo[1], wo[2]), v3(wi[0], wi[1], wi[2]));
}
float or_hg_sample(float g, const float* wo, float u1, float u2, float* wi) {
    float pdf = 0.0f;
    V3 r = hg_draw(g, v3(wo[0], wo[1], wo[2]), u1, u2, pdf);
    wi[0] = r.x;
    wi[1] = r.y;
    wi[2] = r.z;
    return pdf;
}
int or_medium_transmittance(const float* sigma_t, float t, float* out) {
    V3 r = medium_transmittance(v3(sigma_t[0], sigma_t[1], sigma_t[2]), t);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    return 0;
}
int or_medium_sample(const float* sigma_a, const float* sigma_s, float tmax, float u_ch, float u_d, float* t,
                     float* beta) {
    V3 sa = v3(sigma_a[0], sigma_a[1], sigma_a[2]), ss = v3(sigma_s[0], sigma_s[1], sigma_s[2]);
    V3 b;
    bool sc = medium_draw(sa + ss, ss, tmax, u_ch, [&] { return u_d; }, *t, b);
    beta[0] = b.x;
    beta[1] = b.y;
    beta[2] = b.z;
    return sc ? 1 : 0;
}

int or_energy_lut(float* e, float* eavg) {
    const EnergyLut& l = energy_lut();
    if (e) std::memcpy(e, l.e, sizeof(l.e));
    if (eavg) std::memcpy(eavg, l.eavg, sizeof(l.eavg));
    return 0;
}

int or_scene_create(const RtWorldDesc* w, void** out) {
    if (!w || !out) return -1;
    auto sc = std::make_unique<Scene>();
    for (int i = 0; i < w->num_materials; i++) {
        Material m;
        m.d = w->materials[i];
        m.sp = make_shading_params(m.d);
        sc->mats.push_back(m);
    }
    sc->emitter_to_light.assign(sc->mats.size(), -1);
    // Entities in YAML order (SceneLoader.cs:346-443)
    std::vector<const Hittable*> geometry_light_src;
    std::vector<int> geometry_light_kind;
    for (int e = 0; e < w->num_entities; e++) {
        const RtEntityDesc& ed = w->entities[e];
        const Hittable* h = nullptr;
        if (ed.kind == RT_ENT_QUAD) {
            auto q = std::make_unique<Quad>(v3(ed.p[0], ed.p[1], ed.p[2]), v3(ed.p[3], ed.p[4], ed.p[5]),
                                            v3(ed.p[6], ed.p[7], ed.p[8]), ed.material, e);
            h = q.get();
            sc->owned.push_back(std::move(q));
            if (ed.flags & RT_ENT_FLAG_BACKFACE_CULLED) {
                auto bf = std::make_unique<BackFaceCulled>(h);
                h = bf.get();
                sc->owned.push_back(std::move(bf));
            }
        } else if (ed.kind == RT_ENT_SPHERE) {
            auto s = std::make_unique<Sphere>(v3(ed.p[0], ed.p[1], ed.p[2]), ed.p[3], ed.material, e);
            h = s.get();
            sc->owned.push_back(std::move(s));
        } else if (ed.kind == RT_ENT_MESH) {
            auto m = std::make_unique<Mesh>();
            m->material = ed.material;
            for (int64_t t = 0; t < ed.count; t++) {
                const float* p = w->tri_verts + (ed.first + t) * 9;
                m->tris.emplace_back(new Triangle(v3(p[0], p[1], p[2]), v3(p[3], p[4], p[5]), v3(p[6], p[7], p[8]),
                                                  ed.material, e, (int)t));
                if (w->tri_normals) {   // ObjLoader.BuildTrianglesDirect: a face with normals is smooth
                    const float* nn = w->tri_normals + (ed.first + t) * 9;
                    bool any = false;
                    for (int k = 0; k < 9; k++) any = any || nn[k] != 0.0f;
                    if (any) m->tris.back()->make_smooth(nn, w->tri_uvs ? w->tri_uvs + (ed.first + t) * 6 : nullptr);
                }
            }
            m->finish();
            h = m.get();
            sc->meshes.push_back(std::move(m));
        } else {
            std::snprintf(g_err, sizeof(g_err), "unsupported entity kind %d", ed.kind);
            return -6;
        }
        sc->objects.push_back(h);
        sc->entity_ptr.push_back(h);
    }
    // Explicit lights (SceneLoader.cs:446-458), area lights' proxies are entities already.
    for (int i = 0; i < w->num_lights; i++) {
        const RtLightDesc& ld = w->lights[i];
        Light l;
        if (ld.type == RT_LIGHT_AREA) {
            l.type = 3;
            l.corner = v3(ld.corner[0], ld.corner[1], ld.corner[2]);
            l.u = v3(ld.u[0], ld.u[1], ld.u[2]);
            l.v = v3(ld.v[0], ld.v[1], ld.v[2]);
            l.color = v3(ld.color[0], ld.color[1], ld.color[2]);
            l.intensity = ld.intensity;
            l.shadow_samples = std::max(1, ld.shadow_samples);
            l.soft_radius = std::fmax(0.0f, ld.soft_radius);
            V3 cr = cross(l.u, l.v);
            l.area = length(cr);
            l.normal = cr / l.area;
            l.sqrt_samples = (int)std::ceil(std::sqrt((float)l.shadow_samples));
            l.inv_sqrt = 1.0f / (float)l.sqrt_samples;
            l.is_delta = false;
            l.emissive_material = ld.proxy_material;
        } else if (ld.type == RT_LIGHT_DIRECTIONAL) {
            l.type = 4;
            l.direction = normalize(v3(ld.direction[0], ld.direction[1], ld.direction[2]));
            l.color = v3(ld.color[0], ld.color[1], ld.color[2]);
            l.intensity = ld.intensity;
            l.angular_radius = std::fmax(0.0f, ld.angular_radius_deg);
            bool disc = l.angular_radius > 0.0f;
            float rad = l.angular_radius * kPi / 180.0f;
            l.cos_angular = disc ? std::cos(rad) : 1.0f;
            l.solid_angle = disc ? 2.0f * kPi * (1.0f - l.cos_angular) : 0.0f;
            l.shadow_samples = ld.shadow_samples > 0 ? ld.shadow_samples : (disc ? 4 : 1);
            l.sqrt_samples = (int)std::ceil(std::sqrt((float)l.shadow_samples));
            l.inv_sqrt = 1.0f / (float)l.sqrt_samples;
            l.is_delta = !disc;
        } else if (ld.type == RT_LIGHT_SPHERE) {   // SphereLight.cs:54-68
            l.type = 6;
            l.center = v3(ld.center[0], ld.center[1], ld.center[2]);
            l.radius = std::fmax(ld.radius, kEps);
            l.color = v3(ld.color[0], ld.color[1], ld.color[2]);
            l.intensity = ld.intensity;
            l.shadow_samples = ld.shadow_samples > 0 ? ld.shadow_samples : 4;
            l.sqrt_samples = (int)std::ceil(std::sqrt((float)l.shadow_samples));
            l.inv_sqrt = 1.0f / (float)l.sqrt_samples;
            l.is_delta = false;
            l.emissive_material = ld.proxy_material;
        } else {
            std::snprintf(g_err, sizeof(g_err), "unsupported light type %d", ld.type);
            return -6;
        }
        sc->lights.push_back(l);
    }
    // World assembly (SceneLoader.cs:460-485)
    if (sc->objects.size() > 4) {
        sc->top_is_bvh = true;
        sc->bvh_objects = sc->objects;
        sc->top.reset(new BvhNode(sc->bvh_objects, 0, (int)sc->bvh_objects.size(), &sc->arena));
        sc->world.objs.push_back(sc->top.get());
    } else {
        sc->world.objs = sc->objects;
    }
    // Camera: aspect from the render size, set in or_render (Camera depends on W/H).
    // Geometry lights (SceneLoader.cs:805-887)
    int gls = std::max(1, w->geometry_light_samples);
    for (int e = 0; e < w->num_entities; e++) {
        const RtEntityDesc& ed = w->entities[e];
        const Material& m = sc->mats[ed.material];
        if (!m.is_emissive() || m.d.is_light_proxy) continue;
        Light l;
        l.shadow_samples = gls;
        l.sqrt_samples = (int)std::ceil(std::sqrt((float)gls));
        l.inv_sqrt = 1.0f / (float)l.sqrt_samples;
        l.is_delta = false;
        l.emissive_material = ed.material;
        AABB bb = sc->entity_ptr[e]->bbox();
        l.rep_point = 0.5f * (bb.mn + bb.mx);
        if (ed.kind == RT_ENT_QUAD) {
            l.type = 0;
            const BackFaceCulled* bf = dynamic_cast<const BackFaceCulled*>(sc->entity_ptr[e]);
            l.quad = bf ? static_cast<const Quad*>(bf->inner) : static_cast<const Quad*>(sc->entity_ptr[e]);
            l.rep_area = l.quad->area;
        } else if (ed.kind == RT_ENT_MESH) {
            l.type = 1;
            l.mesh = static_cast<const Mesh*>(sc->entity_ptr[e]);
            l.rep_area = l.mesh->total_area;
        } else {   // a sphere: cone sampling (ISolidAngleSamplable)
            l.type = 5;
            const Sphere* sp = static_cast<const Sphere*>(sc->entity_ptr[e]);
            l.center = sp->c;
            l.radius = sp->r;
            l.rep_area = 4.0f * kPi * sp->r * sp->r;   // Sphere.SurfaceArea
        }
        sc->lights.push_back(l);
    }
    // The flat sky and its EnvironmentLight (SceneLoader.cs:524-528)
    sc->sky = v3(w->sky_color[0], w->sky_color[1], w->sky_color[2]);
    if (luminance(sc->sky) > 1e-6f) {
        Light l;
        l.type = 7;
        l.color = sc->sky;
        l.shadow_samples = std::max(1, (int)w->sky_light_samples);
        l.is_delta = false;
        sc->env_light = (int)sc->lights.size();
        sc->lights.push_back(l);
    }
    // Emitter -> light map (Renderer.cs:409-425): geometry lights first, then proxies.
    for (size_t li = 0; li < sc->lights.size(); li++)
        if (sc->lights[li].type <= 2 || sc->lights[li].type == 5)
            sc->emitter_to_light[sc->lights[li].emissive_material] = (int)li;
    for (size_t li = 0; li < sc->lights.size(); li++)
        if ((sc->lights[li].type == 3 || sc->lights[li].type == 6) && sc->lights[li].emissive_material >= 0)
            sc->emitter_to_light[sc->lights[li].emissive_material] = (int)li;
    // RR classifier (Renderer.cs:361-378, ComputeFiniteSceneBounds :475-500)
    AABB bounds;
    {
        bool any = false;
        AABB acc = aabb_empty();
        for (const Hittable* o : sc->world.objs) {
            AABB b = o->bbox();
            V3 d = b.mx - b.mn;
            if (d.x < 1.0e5f && d.y < 1.0e5f && d.z < 1.0e5f) {
                acc = any ? surrounding(acc, b) : b;
                any = true;
            }
        }
        if (any) {
            bounds = acc;
        } else {
            AABB raw = sc->world.bbox();
            bounds = {vmax(raw.mn, v3(-1.0e3f)), vmin(raw.mx, v3(1.0e3f))};
        }
    }
    // LightDistribution (LightDistribution.cs:30-102): power, then forced uniform
    for (int mode = 0; mode < 2; mode++) {
        size_t n = sc->lights.size();
        std::vector<float>& cdf = sc->pick_cdf[mode];
        std::vector<float>& pdf = sc->pick_pdf[mode];
        cdf.assign(n, 0.0f);
        pdf.assign(n, 0.0f);
        if (n == 0) continue;
        std::vector<float> power(n, 0.0f);
        float sum = 0.0f;
        if (mode == 0)
            for (size_t i = 0; i < n; i++) {
                power[i] = std::fmax(0.0f, light_approx_power(sc->lights[i], bounds, *sc));
                sum += power[i];
            }
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
    float flux = 0.0f;
    for (const Light& l : sc->lights) flux += light_approx_power(l, bounds, *sc);
    V3 ext = bounds.mx - bounds.mn;
    float radius = std::fmax(0.5f * length(ext), 1e-3f);
    float sphere_area = 4.0f * kPi * radius * radius;
    sc->mean_irradiance = flux / sphere_area;
    bool indirect = sc->mean_irradiance < 0.5f;
    sc->rr_min_bounces = indirect ? 6 : 3;
    sc->rr_min_survival = indirect ? 0.40f : 0.10f;
    // Medium
    if (w->medium.enabled) {
        sc->has_medium = true;
        sc->sigma_a = vmax(v3(w->medium.sigma_a[0], w->medium.sigma_a[1], w->medium.sigma_a[2]), v3(0.0f));
        sc->sigma_s = vmax(v3(w->medium.sigma_s[0], w->medium.sigma_s[1], w->medium.sigma_s[2]), v3(0.0f));
        sc->sigma_t = sc->sigma_a + sc->sigma_s;
        sc->hg_g = std::fmax(-0.999f, std::fmin(0.999f, w->medium.g));
    }
    sc->cam_desc = w->camera;
    (void)energy_lut();
    *out = sc.release();
    return 0;
}

int or_scene_destroy(void* s) {
    delete static_cast<Scene*>(s);
    return 0;
}

int or_scene_info(void* s, int32_t* rr_min_bounces, float* rr_min_survival, float* mean_irr, int32_t* num_lights,
                  int32_t* top_is_bvh) {
    Scene* sc = static_cast<Scene*>(s);
    if (rr_min_bounces) *rr_min_bounces = sc->rr_min_bounces;
    if (rr_min_survival) *rr_min_survival = sc->rr_min_survival;
    if (mean_irr) *mean_irr = sc->mean_irradiance;
    if (num_lights) *num_lights = (int32_t)sc->lights.size();
    if (top_is_bvh) *top_is_bvh = sc->top_is_bvh ? 1 : 0;
    return 0;
}

// Pre-order node export of the top-level build: 10 words per node
// (bmin xyz, bmax xyz as float bits, leaf, axis, first, count) and the
// partitioned entity order. Returns the node count.
int64_t or_export_top(void* s, int32_t* nodes, int64_t max_nodes, int32_t* order, int64_t max_order) {
    Scene* sc = static_cast<Scene*>(s);
    std::vector<FlatNode> fl;
    if (sc->top) sc->top->flatten(fl);
    for (size_t i = 0; i < fl.size() && (int64_t)i < max_nodes; i++) {
        float f[6] = {fl[i].box.mn.x, fl[i].box.mn.y, fl[i].box.mn.z, fl[i].box.mx.x, fl[i].box.mx.y, fl[i].box.mx.z};
        std::memcpy(nodes + i * 10, f, sizeof(f));
        nodes[i * 10 + 6] = fl[i].leaf;
        nodes[i * 10 + 7] = fl[i].axis;
        nodes[i * 10 + 8] = fl[i].first;
        nodes[i * 10 + 9] = fl[i].count;
    }
    if (order) {
        const std::vector<const Hittable*>& src = sc->top ? sc->bvh_objects : sc->objects;
        for (size_t i = 0; i < src.size() && (int64_t)i < max_order; i++) {
            int idx = -1;
            for (size_t e = 0; e < sc->entity_ptr.size(); e++)
                if (sc->entity_ptr[e] == src[i]) idx = (int)e;
            order[i] = idx;
        }
    }
    return (int64_t)fl.size();
}

// Same for the BVH of the mesh at entity index `entity`; `order` receives the
// partitioned triangle order (local indices).
int64_t or_export_mesh(void* s, int32_t entity, int32_t* nodes, int64_t max_nodes, int32_t* order, int64_t max_order) {
    Scene* sc = static_cast<Scene*>(s);
    const Mesh* m = dynamic_cast<const Mesh*>(sc->entity_ptr[entity]);
    if (!m) return -1;
    std::vector<FlatNode> fl;
    if (m->use_bvh) m->root->flatten(fl);
    for (size_t i = 0; i < fl.size() && (int64_t)i < max_nodes; i++) {
        float f[6] = {fl[i].box.mn.x, fl[i].box.mn.y, fl[i].box.mn.z, fl[i].box.mx.x, fl[i].box.mx.y, fl[i].box.mx.z};
        std::memcpy(nodes + i * 10, f, sizeof(f));
        nodes[i * 10 + 6] = fl[i].leaf;
        nodes[i * 10 + 7] = fl[i].axis;
        nodes[i * 10 + 8] = fl[i].first;
        nodes[i * 10 + 9] = fl[i].count;
    }
    if (order)
        for (size_t i = 0; i < m->bvh_input.size() && (int64_t)i < max_order; i++)
            order[i] = static_cast<const Triangle*>(m->bvh_input[i])->prim;
    return (int64_t)fl.size();
}

// Closest hit for n rays (8 floats each: o, d, pad). hits: 6 words per ray
// (t, u, v as float bits; entity, prim, hit flag). counters[3] += node visits,
// triangle tests, other primitive tests.
int or_trace_closest(void* s, const float* rays, int64_t n, float tmin, float tmax, int32_t* hits,
                     uint64_t* counters, int32_t linear) {
    Scene* sc = static_cast<Scene*>(s);
    t_cnt = Counters();
    t_counting = true;
    for (int64_t i = 0; i < n; i++) {
        const float* r = rays + i * 8;
        Ray ray(v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]));
        HitRecord rec;
        bool h;
        if (linear) {   // BvhEquivalenceTests: the same objects in a flat HittableList
            HittableList flat;
            flat.objs = sc->objects;
            h = flat.hit(ray, tmin, tmax, rec);
        } else {
            h = sc->world_hit(ray, tmin, tmax, rec);
        }
        int32_t* o = hits + i * 6;
        float f3[3] = {h ? rec.t : 0.0f, h ? rec.u : 0.0f, h ? rec.v : 0.0f};
        std::memcpy(o, f3, sizeof(f3));
        o[3] = h ? rec.entity : -1;
        o[4] = h ? rec.prim : -1;
        o[5] = h ? 1 : 0;
    }
    t_counting = false;
    if (counters) {
        counters[0] += t_cnt.node_visits;
        counters[1] += t_cnt.tri_tests;
        counters[2] += t_cnt.other_tests;
    }
    return 0;
}

// Shadow rays: 8 floats (o, d, tmin, tmax) -> transmittance rgb.
int or_trace_any(void* s, const float* rays, int64_t n, float* out) {
    Scene* sc = static_cast<Scene*>(s);
    for (int64_t i = 0; i < n; i++) {
        const float* r = rays + i * 8;
        Ray ray(v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]));
        V3 t = shadow_transmittance(*sc, ray, r[6], r[7]);
        out[i * 3 + 0] = t.x;
        out[i * 3 + 1] = t.y;
        out[i * 3 + 2] = t.z;
    }
    return 0;
}

int or_bsdf_batch(void* s, const RtBsdfQuery* q, int64_t n, RtBsdfResult* out) {
    Scene* sc = static_cast<Scene*>(s);
    for (int64_t i = 0; i < n; i++) {
        const RtBsdfQuery& qq = q[i];
        RtBsdfResult& r = out[i];
        std::memset(&r, 0, sizeof(r));
        const Material& m = sc->mats[qq.material];
        if (m.is_emissive()) {
            r.lobe = -1;
            continue;
        }
        Disney d(m);
        HitRecord rec;
        rec.n = v3(qq.n[0], qq.n[1], qq.n[2]);
        rec.tangent = v3(qq.tangent[0], qq.tangent[1], qq.tangent[2]);
        rec.bitangent = v3(qq.bitangent[0], qq.bitangent[1], qq.bitangent[2]);
        rec.p = v3(qq.point[0], qq.point[1], qq.point[2]);
        rec.front = qq.front_face != 0;
        rec.material = qq.material;
        V3 V = v3(qq.v[0], qq.v[1], qq.v[2]);
        V3 L = v3(qq.l[0], qq.l[1], qq.l[2]);
        V3 f = d.evaluate(V, L, rec);
        r.f[0] = f.x; r.f[1] = f.y; r.f[2] = f.z;
        r.pdf = d.pdf(V, L, rec);
        V3 fd = d.evaluate_direct(L, V, rec.n, rec);
        r.fd[0] = fd.x; r.fd[1] = fd.y; r.fd[2] = fd.z;
        begin_pixel_sample(qq.pixel_seed, qq.sample_index);
        t_sampler.dim = qq.dim;
        BsdfSample bs;
        int lobe;
        bool has = d.sample(V, rec, bs, lobe);
        r.dims_used = t_sampler.dim - qq.dim;
        end_pixel_sample();
        r.lobe = lobe;
        r.has_sample = has ? 1 : 0;
        if (has) {
            r.wo[0] = bs.wo.x; r.wo[1] = bs.wo.y; r.wo[2] = bs.wo.z;
            r.s_f[0] = bs.f.x; r.s_f[1] = bs.f.y; r.s_f[2] = bs.f.z;
            r.s_pdf = bs.pdf;
            r.is_delta = bs.is_delta ? 1 : 0;
            r.transition = bs.transition;
        }
    }
    return 0;
}

// The scene's global medium on one Sobol stream per query: HomogeneousMedium
// .Sample (:46-76) over [0, tmax], then HenyeyGreensteinPhase.Sample (:32-54)
// with the next two draws, as TraceRay's volumetric branch draws them
// (Renderer.cs:1704-1765); Transmittance(tmax) (:36-44) and Evaluate (:23-30)
// beside them.
int or_medium_batch(void* s, const RtMediumQuery* q, int64_t n, RtMediumResult* out) {
    Scene* sc = static_cast<Scene*>(s);
    if (!sc->has_medium) return -1;
    for (int64_t i = 0; i < n; i++) {
        const RtMediumQuery& qq = q[i];
        RtMediumResult& r = out[i];
        std::memset(&r, 0, sizeof(r));
        V3 wo = v3(qq.wo[0], qq.wo[1], qq.wo[2]);
        V3 wi = v3(qq.wi[0], qq.wi[1], qq.wi[2]);
        begin_pixel_sample(qq.pixel_seed, qq.sample_index);
        t_sampler.dim = qq.dim;
        float t = 0.0f;
        V3 beta;
        float u_ch = random_float();
        r.scattered = medium_draw(sc->sigma_t, sc->sigma_s, qq.tmax, u_ch, [] { return random_float(); }, t, beta);
        r.t = t;
        r.beta[0] = beta.x; r.beta[1] = beta.y; r.beta[2] = beta.z;
        float u1 = random_float(), u2 = random_float();
        float pdf = 0.0f;
        V3 d = hg_draw(sc->hg_g, wo, u1, u2, pdf);
        r.phase_wi[0] = d.x; r.phase_wi[1] = d.y; r.phase_wi[2] = d.z;
        r.phase_pdf = pdf;
        r.dims_used = t_sampler.dim - qq.dim;
        end_pixel_sample();
        V3 tr = medium_transmittance(sc->sigma_t, qq.tmax);
        r.tr[0] = tr.x; r.tr[1] = tr.y; r.tr[2] = tr.z;
        r.phase_eval = hg_evaluate(sc->hg_g, wo, wi);
    }
    return 0;
}

// Renderer.ToneMapToDisplay (:741-751): each pixel times the exposure scale
// 2^ev (:333), then AcesToneMap (:893-907): floor at zero, the ACES filmic fit
// x(2.51x + 0.03) / (x(2.43x + 0.59) + 0.14) per channel, clamp to [0, 1],
// gamma 1/2.2. Planar HDR in, interleaved RGB out.
int or_tonemap(const float* hdr, int32_t width, int32_t height, float exposure_ev, float* rgb) {
    if (!hdr || !rgb || width <= 0 || height <= 0) return -1;
    const float scale = std::pow(2.0f, exposure_ev);
    const float inv_gamma = 1.0f / 2.2f;
    size_t npix = (size_t)width * height;
    for (size_t i = 0; i < npix; i++) {
        V3 c = v3(hdr[i], hdr[npix + i], hdr[2 * npix + i]) * scale;
        c = vmax(c, v3(0.0f));
        V3 a = c * (2.51f * c + v3(0.03f));
        V3 b = c * (2.43f * c + v3(0.59f)) + v3(0.14f);
        V3 m = v3(a.x / b.x, a.y / b.y, a.z / b.z);
        rgb[3 * i + 0] = std::pow(std::fmin(std::fmax(m.x, 0.0f), 1.0f), inv_gamma);
        rgb[3 * i + 1] = std::pow(std::fmin(std::fmax(m.y, 0.0f), 1.0f), inv_gamma);
        rgb[3 * i + 2] = std::pow(std::fmin(std::fmax(m.z, 0.0f), 1.0f), inv_gamma);
    }
    return 0;
}

// Renders a window of the film (or the full frame) with `threads` workers over
// 16x16 tiles (Renderer.cs:530-585). out: planar 3*W*H (only the window is
// written). counters[7]: node visits, tri tests, other tests, closest rays,
// shadow rays, segments, samples.
// A capturing render (Renderer.Render with RenderCaptureOptions.Full) of the
// whole frame: out holds 23 planes of W*H floats, in the order of
// render_pixel_capture's record.
int or_render_capture(void* s, const RtRenderParams* p, float* out, int32_t threads) {
    Scene* sc = static_cast<Scene*>(s);
    int W = p->width, H = p->height;
    build_camera(*sc, sc->cam_desc, (float)W / (float)H);
    Tracer tr{*sc, {}};
    tr.cfg.max_depth = p->max_depth;
    tr.cfg.max_radiance = p->max_sample_radiance > 0.0f ? p->max_sample_radiance : 10.0f;
    float icf = p->indirect_clamp_factor >= 0.0f ? p->indirect_clamp_factor : 0.25f;
    tr.cfg.indirect_max = tr.cfg.max_radiance * std::fmax(0.0f, icf);
    tr.cfg.mis_power = p->mis_heuristic == RT_MIS_POWER;
    tr.cfg.rr_min_bounces = p->rr_min_bounces >= 0 ? p->rr_min_bounces : sc->rr_min_bounces;
    tr.cfg.rr_min_survival = p->rr_min_bounces >= 0 ? p->rr_min_survival : sc->rr_min_survival;
    tr.cfg.light_pick = p->light_strategy;
    const int T = 16;
    int tx = (W + T - 1) / T, ty = (H + T - 1) / T;
    std::atomic<int> next(0);
    size_t plane = (size_t)W * (size_t)H;
    auto worker = [&]() {
        for (;;) {
            int tile = next.fetch_add(1);
            if (tile >= tx * ty) break;
            int px0 = (tile % tx) * T, py0 = (tile / tx) * T;
            for (int j = py0; j < std::min(py0 + T, H); j++)
                for (int i = px0; i < std::min(px0 + T, W); i++) {
                    float rec[23];
                    render_pixel_capture(*sc, tr, i, j, W, H, p->spp, p->spp_offset, rec);
                    for (int k = 0; k < 23; k++) out[(size_t)k * plane + (size_t)j * W + i] = rec[k];
                }
        }
    };
    int nt = std::max(1, (int)threads);
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return 0;
}

int or_render(void* s, const RtRenderParams* p, float* out, int32_t threads, uint64_t* counters) {
    Scene* sc = static_cast<Scene*>(s);
    int W = p->width, H = p->height;
    build_camera(*sc, sc->cam_desc, (float)W / (float)H);
    Tracer tr{*sc, {}};
    tr.cfg.max_depth = p->max_depth;
    tr.cfg.max_radiance = p->max_sample_radiance > 0.0f ? p->max_sample_radiance : 10.0f;
    float icf = p->indirect_clamp_factor >= 0.0f ? p->indirect_clamp_factor : 0.25f;
    tr.cfg.indirect_max = tr.cfg.max_radiance * std::fmax(0.0f, icf);
    tr.cfg.mis_power = p->mis_heuristic == RT_MIS_POWER;
    tr.cfg.rr_min_bounces = p->rr_min_bounces >= 0 ? p->rr_min_bounces : sc->rr_min_bounces;
    tr.cfg.rr_min_survival = p->rr_min_bounces >= 0 ? p->rr_min_survival : sc->rr_min_survival;
    tr.cfg.light_pick = p->light_strategy;
    int x0 = p->pixel_x0, y0 = p->pixel_y0;
    int ww = p->window_w > 0 ? p->window_w : W;
    int wh = p->window_h > 0 ? p->window_h : H;
    const int T = 16;
    int tx = (ww + T - 1) / T, ty = (wh + T - 1) / T;
    int total = tx * ty;
    std::atomic<int> next(0);
    std::vector<Counters> cnts(std::max(1, threads));
    auto worker = [&](int wid) {
        t_counting = counters != nullptr;
        t_cnt = Counters();
        for (;;) {
            int tile = next.fetch_add(1);
            if (tile >= total) break;
            int ax = tile % tx, ay = tile / tx;
            int px0 = x0 + ax * T, py0 = y0 + ay * T;
            int px1 = std::min(px0 + T, x0 + ww), py1 = std::min(py0 + T, y0 + wh);
            for (int j = py0; j < py1; j++)
                for (int i = px0; i < px1; i++) {
                    V3 c = render_pixel(*sc, tr, i, j, W, H, p->spp, p->spp_offset);
                    V3 lin = c / (float)p->spp;   // Renderer.cs:711
                    size_t plane = (size_t)W * (size_t)H;
                    out[0 * plane + (size_t)j * W + i] = lin.x;
                    out[1 * plane + (size_t)j * W + i] = lin.y;
                    out[2 * plane + (size_t)j * W + i] = lin.z;
                }
        }
        cnts[wid] = t_cnt;
        t_counting = false;
    };
    int nt = std::max(1, threads);
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(worker, t);
    worker(0);
    for (auto& th : pool) th.join();
    if (counters) {
        for (const Counters& c : cnts) {
            counters[0] += c.node_visits;
            counters[1] += c.tri_tests;
            counters[2] += c.other_tests;
            counters[3] += c.closest_rays;
            counters[4] += c.shadow_rays;
            counters[5] += c.segments;
            counters[6] += c.samples;
        }
    }
    return 0;
}

}  // extern "C"
