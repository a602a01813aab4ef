// Device code of the bounce loop: Owen-scrambled Sobol, ordered BVH traversal
// (closest and any hit), hit-record reconstruction, the Disney BSDF, lights,
// transparent shadows, the homogeneous medium and the per-path integrator.
//
// Built with -fmad=false and IEEE div/sqrt: every decision (hit/miss, leaf
// order, lobe choice, RR gate) uses the same float operations, in the same
// order, as 3d-ray's C# (paths in comments are relative to src/RayTracer/).
// Transcendentals (cos, sin, pow, exp, log) are CUDA's own; they differ from
// glibc by a few ulps, so paths agree bit-for-bit only up to the first
// transcendental-dependent direction.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>

#include "scene_types.h"

namespace rt {

// ---------------------------------------------------------------------------
// Checked build (-DRT_CHECKED): every index that comes from scene data or from
// the wavefront's queues is tested against its array's length before the
// access. An index out of range raises a device flag, which the host turns
// into RT_ERR_BOUNDS when the call ends, and is replaced by 0 (the checked
// build gives every array at least one element), so the access stays in
// bounds and nothing traps. The product build compiles the tests away.
// ---------------------------------------------------------------------------
#ifdef RT_CHECKED
static __device__ int g_bounds_flag;
RT_D long long checked_index(long long i, long long n) {
    if (i >= 0 && i < n) return i;
    atomicExch(&g_bounds_flag, 1);
    return 0;
}
#define RT_IX(i, n) checked_index((long long)(i), (long long)(n))
#else
#define RT_IX(i, n) (i)
#endif

// ---------------------------------------------------------------------------
// Owen-scrambled Sobol (Core/Sampling/OwenSobol.cs:48-210)
// ---------------------------------------------------------------------------
__constant__ uint32_t c_dim1_dirs[32] = {
    0x80000000u, 0xc0000000u, 0xa0000000u, 0xf0000000u, 0x88000000u, 0xcc000000u, 0xaa000000u, 0xff000000u,
    0x80800000u, 0xc0c00000u, 0xa0a00000u, 0xf0f00000u, 0x88880000u, 0xcccc0000u, 0xaaaa0000u, 0xffff0000u,
    0x80008000u, 0xc000c000u, 0xa000a000u, 0xf000f000u, 0x88008800u, 0xcc00cc00u, 0xaa00aa00u, 0xff00ff00u,
    0x80808080u, 0xc0c0c0c0u, 0xa0a0a0a0u, 0xf0f0f0f0u, 0x88888888u, 0xccccccccu, 0xaaaaaaaau, 0xffffffffu,
};

RT_D uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
RT_D uint32_t lk_permute(uint32_t v, uint32_t seed) {
    v += seed;
    v ^= v * 0x6c50b47cu;
    v ^= v * 0xb82f1e52u;
    v ^= v * 0xc7afe638u;
    v ^= v * 0x8d22f6e6u;
    return v;
}
RT_D uint32_t owen_scramble(uint32_t v, uint32_t seed) { return __brev(lk_permute(__brev(v), seed)); }

RT_D float sobol_sample(uint32_t index, uint32_t dim, uint32_t pixel_seed) {
    uint32_t v;
    if (dim == 0u) {
        v = __brev(index);
    } else if (dim == 1u) {
        v = 0u;
        uint32_t i = index;
#pragma unroll 1
        for (int k = 0; i != 0u; k++, i >>= 1)
            if (i & 1u) v ^= c_dim1_dirs[k];
    } else {
        uint32_t shuffle = hash_u32(dim * 0x68bc21ebu + 0xc7afe638u);
        v = __brev(owen_scramble(index, shuffle));
    }
    uint32_t scramble = hash_u32(pixel_seed ^ hash_u32(dim * 0xa511e9b3u + 0x736f6c34u));
    v = owen_scramble(v, scramble);
    return (float)(v >> 8) * (1.0f / 16777216.0f);
}

// The per-path dimension counter of Core/Sampling/Sampler.cs:75-118.
struct Sampler {
    uint32_t seed, index, dim;
    RT_D float next() { return sobol_sample(index, dim++, seed); }
};

RT_D V3 random_unit_vector(Sampler& s) {   // Core/MathUtils.cs:104-112
    float u = s.next();
    float v = s.next();
    float z = 1.0f - 2.0f * u;
    float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float phi = 2.0f * kPi * v;
    float sn, cs;
    sincosf(phi, &sn, &cs);
    return v3(r * cs, r * sn, z);
}

// ---------------------------------------------------------------------------
// Traversal
// ---------------------------------------------------------------------------
enum : int { HIT_NONE = 0, HIT_TRI = 1, HIT_QUAD = 2, HIT_SPHERE = 3 };

struct Hit {
    float t, u, v;
    int kind;
    int slot;   // stored triangle index, or entity id for quads and spheres
};

// Work counters of the counting build (algorithmic bytes of the roofline):
// traversal work of closest-hit rays and of shadow rays kept apart.
struct TravCounters {
    uint32_t nodes, tris, others;
};
struct Counters {
    TravCounters closest, shadow;
    uint32_t closest_rays, shadow_rays;
};

RT_D V3 ld3(const float4& f) { return v3(f.x, f.y, f.z); }

// Read-only load of scene data (BVH records, triangles, entity boxes) with an
// L2 evict-last policy. The path state the wavefront streams each iteration
// (~0.6 GB at 4 M slots) is far larger than the 126 MB L2; without the hint it
// pushes the ~86 MB scene of the icosphere field out of L2 between the
// traversal kernels. A hint: results are unchanged.
#ifndef RT_L2_HINTS
#define RT_L2_HINTS 1
#endif
RT_D float4 ldg_scene(const float4* p) {
#if RT_L2_HINTS
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    float4 v;
    asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p), "l"(pol));
    return v;
#else
    return __ldg(p);
#endif
}

// Geometry/Triangle.cs:49-89 (Moller-Trumbore, |a| < 1e-7 reject, inclusive t range)
RT_D bool tri_test(const float4* tris, int i, V3 o, V3 d, float tmin, float tmax, float& t, float& u, float& v) {
    float4 a0 = ldg_scene(tris + 3 * i), a1 = ldg_scene(tris + 3 * i + 1), a2 = ldg_scene(tris + 3 * i + 2);
    V3 v0 = ld3(a0), e1 = ld3(a1), e2 = ld3(a2);
    V3 h = cross(d, e2);
    float a = dot(e1, h);
    if (fabsf(a) < 1e-7f) return false;
    float f = 1.0f / a;
    V3 s = o - v0;
    u = f * dot(s, h);
    if (u < 0.0f || u > 1.0f) return false;
    V3 q = cross(s, e1);
    v = f * dot(d, q);
    if (v < 0.0f || u + v > 1.0f) return false;
    t = f * dot(e2, q);
    if (t < tmin || t > tmax) return false;
    return true;
}

// Geometry/Quad.cs:42-86; front_only for the back-face-culled light proxy
// (Geometry/BackFaceCulledHittable.cs).
RT_D bool quad_test(const QuadData& q, V3 o, V3 d, float tmin, float tmax, bool front_only, float& t, float& a,
                    float& b) {
    float denom = dot(q.normal, d);
    if (fabsf(denom) < 1e-8f) return false;
    t = (q.d - dot(q.normal, o)) / denom;
    if (t < tmin || t > tmax) return false;
    V3 ip = o + t * d;
    V3 ph = ip - q.q;
    a = dot(q.w, cross(ph, q.v));
    b = dot(q.w, cross(q.u, ph));
    if (a < 0.0f || a > 1.0f || b < 0.0f || b > 1.0f) return false;
    if (front_only && !(dot(d, q.normal) < 0.0f)) return false;
    return true;
}

// Geometry/Sphere.cs:20-42
RT_D bool sphere_test(const SphereData& s, V3 o, V3 d, float tmin, float tmax, float& t) {
    V3 oc = o - s.c;
    float a = length_sq(d);
    float hb = dot(oc, d);
    float c = length_sq(oc) - s.r * s.r;
    float disc = hb * hb - a * c;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float root = (-hb - sq) / a;
    if (root < tmin || root > tmax) {
        root = (-hb + sq) / a;
        if (root < tmin || root > tmax) return false;
    }
    t = root;
    return true;
}

// Tests one quad/sphere entity. Returns true on an accepted hit.
RT_D bool entity_test(const SceneView& s, int e, V3 o, V3 d, float tmin, float tmax, Hit& h) {
    Entity en = s.entities[RT_IX(e, s.n_entities)];
    float t, a = 0.0f, b = 0.0f;
    if (en.kind == ENT_QUAD) {
        if (!quad_test(s.quads[RT_IX(en.index, s.n_quads)], o, d, tmin, tmax, (en.flags & ENT_BACKFACE_CULLED) != 0,
                       t, a, b))
            return false;
        h = Hit{t, a, b, HIT_QUAD, e};
        return true;
    }
    if (!sphere_test(s.spheres[RT_IX(en.index, s.n_spheres)], o, d, tmin, tmax, t)) return false;
    h = Hit{t, 0.0f, 0.0f, HIT_SPHERE, e};
    return true;
}

// Three-input min / max (PTX min.f32 and max.f32 with three sources, sm_100):
// one instruction for what fminf(a, fminf(b, c)) computes in two. Neither
// rounds, and both skip a NaN source as fminf / fmaxf do, so the value is the
// same.
RT_D float fmin3(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
RT_D float fmax3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Slab test of one child box; te receives max(tmin, entry distance).
RT_D bool box_hit_te(float lx, float ly, float lz, float hx, float hy, float hz, V3 o, V3 inv, float tmin,
                     float tmax, float& te) {   // Core/AABB.cs:28-52
    float t0x = (lx - o.x) * inv.x, t0y = (ly - o.y) * inv.y, t0z = (lz - o.z) * inv.z;
    float t1x = (hx - o.x) * inv.x, t1y = (hy - o.y) * inv.y, t1z = (hz - o.z) * inv.z;
    te = fmax3(tmin, fminf(t0x, t1x), fmaxf(fminf(t0y, t1y), fminf(t0z, t1z)));
    float tx = fmin3(tmax, fmaxf(t0x, t1x), fminf(fmaxf(t0y, t1y), fmaxf(t0z, t1z)));
    return tx >= te;
}

// Ordered depth-first traversal reproducing HittableList -> BvhNode -> Mesh ->
// BvhNode -> Triangle (Geometry/HittableList.cs:19-37, Acceleration/BvhNode.cs:157-206).
// The near child (sign of dir[split axis]) is visited first, fat leaves are
// scanned in order, a later primitive at an equal t wins (inclusive range).
// Each 64-byte node record holds both children's boxes: both are tested
// against the current closest t when the parent is visited, and a pushed far
// child keeps its entry distance so it is dropped at pop time exactly when
// BvhNode's own box test (against the closer t found meanwhile) would reject
// it. Box tests only prune, never accept, so the primitive test sequence is
// the reference's minus primitives that cannot be hit: ids and t match.
// ANY = true stops at the first accepted hit (opaque shadow rays).
// has_root restricts the walk to one mesh BVH (a light's own geometry).
// Walker holds the walk's state so that it can run in rounds; the persistent
// wavefront kernels refill finished lanes of a warp between rounds. A stack
// overflow ends the walk with ok = false and err set. traverse() below is the
// same walk as one loop.
template <bool ANY, int STACK>
struct Walker {
    static constexpr int kNone = INT_MIN;   // "pop the next entry" (no leaf code can take this value)
    V3 o, d, inv;
    float tmin, closest;
    Hit best;
    int code, sp;
    bool ok;
    int st_code[STACK];
    float st_te[STACK];

    RT_D void start(const SceneView& s, V3 o_, V3 d_, float tmin_, float tmax, TravCounters* cnt, bool has_root,
                    int root) {
        o = o_;
        d = d_;
        inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);   // Core/Ray.cs:43
        tmin = tmin_;
        closest = tmax;
        best.kind = HIT_NONE;
        sp = 0;
        ok = true;
        code = kNone;
        if (has_root) {
            code = root;
            if (cnt && root >= 0) cnt->nodes++;   // the mesh root's own BvhNode.Hit
        } else if (s.top_is_bvh) {
            code = s.top_root;
            if (cnt) cnt->nodes++;                // the world root's BvhNode.Hit
        } else {
            for (int i = s.num_top_items - 1; i >= 0; --i) {
                st_code[sp] = leaf_code(s.top_items[RT_IX(i, s.num_top_items)], LEAF_ENT1, 1);
                st_te[sp] = -kInf;
                sp++;
            }
        }
    }

    // One round: descend interior records to a leaf, test the leaf, pop the
    // next entry. Returns true when the walk is over.
    RT_D bool step(const SceneView& s, TravCounters* cnt, int* err) {
        // Descend interior records: test both children, go near, stack far.
        while (code >= 0) {
            const float4* np = s.cnodes + (size_t)RT_IX(code, s.n_cnodes) * 4;
            float4 a = ldg_scene(np), b = ldg_scene(np + 1), c = ldg_scene(np + 2), e = ldg_scene(np + 3);
            if (cnt) cnt->nodes += 2;
            float tel, ter;
            bool hl = box_hit_te(a.x, a.y, a.z, b.x, b.y, b.z, o, inv, tmin, closest, tel);
            bool hr = box_hit_te(c.x, c.y, c.z, e.x, e.y, e.z, o, inv, tmin, closest, ter);
            int axis = __float_as_int(c.w);
            float da = axis == 0 ? d.x : (axis == 1 ? d.y : d.z);
            bool left_near = da >= 0.0f;
            int lc = __float_as_int(a.w), rc = __float_as_int(b.w);
            int nc = left_near ? lc : rc, fc = left_near ? rc : lc;
            bool hn = left_near ? hl : hr, hf = left_near ? hr : hl;
            float tf = left_near ? ter : tel;
            if (hn && hf) {
                if (sp >= STACK) {
                    *err = RT_ERR_STACK;
                    ok = false;
                    return true;
                }
                st_code[sp] = fc;
                st_te[sp] = tf;
                sp++;
            }
            code = hn ? nc : (hf ? fc : kNone);
        }
        // A leaf (or nothing): primitives in order.
        if (code != kNone) {
            int v = ~code;
            int first = v >> 5;
            int kind = (v >> 3) & 3;
            int count = (v & 7) + 1;
            code = kNone;
            if (kind == LEAF_ENT1) {
                Entity en = s.entities[RT_IX(first, s.n_entities)];
                if (en.kind == ENT_MESH) {   // Mesh.Hit -> its BVH root (box test) or flat list
                    if (en.index >= 0) {
                        if (cnt) cnt->nodes++;
                        float4 lo = ldg_scene(s.ent_box + 2 * RT_IX(first, s.n_entities)),
                               hi = ldg_scene(s.ent_box + 2 * RT_IX(first, s.n_entities) + 1);
                        float te;
                        if (box_hit_te(lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, o, inv, tmin, closest, te)) {
                            code = en.index;
                            return false;
                        }
                    } else {
                        code = en.index;   // <= 4 triangles: HittableList, no box test
                        return false;
                    }
                } else {
                    if (cnt) cnt->others++;
                    Hit h;
                    if (entity_test(s, first, o, d, tmin, closest, h)) {
                        best = h;
                        closest = h.t;
                        if (ANY) return true;
                    }
                }
            } else if (kind == LEAF_ENTS) {   // top-level fat leaf: entities in order
                if (sp + count > STACK) {
                    *err = RT_ERR_STACK;
                    ok = false;
                    return true;
                }
                for (int i = count - 1; i >= 0; --i) {
                    st_code[sp] = leaf_code(s.top_items[RT_IX(first + i, s.num_top_items)], LEAF_ENT1, 1);
                    st_te[sp] = -kInf;
                    sp++;
                }
            } else {   // triangle leaf (or a mesh's flat list)
                for (int i = 0; i < count; i++) {
                    float t, u, vv;
                    if (cnt) cnt->tris++;
                    if (tri_test(s.tris, RT_IX(first + i, s.n_tris), o, d, tmin, closest, t, u, vv)) {
                        best = Hit{t, u, vv, HIT_TRI, first + i};
                        closest = t;
                        if (ANY) return true;
                    }
                }
            }
        }
        // Pop the next entry the current closest t does not prune.
        while (sp > 0) {
            --sp;
            if (!(st_te[sp] > closest)) {
                code = st_code[sp];
                break;
            }
        }
        return code == kNone;
    }
};

// One walk to the end. The same walk as Walker, in one loop (kept separate:
// the one-shot form compiles to a smaller stack frame and runs faster).
template <bool ANY, int STACK>
__device__ __forceinline__ bool traverse(const SceneView& s, V3 o, V3 d, float tmin, float tmax, Hit& best,
                                         TravCounters* cnt, int* err, bool has_root = false, int root = 0) {
    const int kNone = INT_MIN;   // "pop the next entry" (no leaf code can take this value)
    V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);   // Core/Ray.cs:43
    // (code, entry distance bits): one 8-byte access per push and pop. An
    // any-hit walk returns at its first hit, so its closest t stays tmax and no
    // entry is ever pruned at pop time: it keeps the codes alone.
    int2 st[ANY ? 1 : STACK];
    int stc[ANY ? STACK : 1];
    int sp = 0;
    auto push = [&](int c, float te) {
        if (ANY) stc[sp++] = c;
        else st[sp++] = make_int2(c, __float_as_int(te));
    };
    float closest = tmax;
    best.kind = HIT_NONE;
    int code = kNone;
    if (has_root) {
        code = root;
        if (cnt && root >= 0) cnt->nodes++;   // the mesh root's own BvhNode.Hit
    } else if (s.top_is_bvh) {
        code = s.top_root;
        if (cnt) cnt->nodes++;                // the world root's BvhNode.Hit
    } else {
        for (int i = s.num_top_items - 1; i >= 0; --i) {
            push(leaf_code(s.top_items[RT_IX(i, s.num_top_items)], LEAF_ENT1, 1), -kInf);
        }
    }
    for (;;) {
        // Descend interior records: test both children, go near, stack far.
        while (code >= 0) {
            const float4* np = s.cnodes + (size_t)RT_IX(code, s.n_cnodes) * 4;
            float4 a = ldg_scene(np), b = ldg_scene(np + 1), c = ldg_scene(np + 2), e = ldg_scene(np + 3);
            if (cnt) cnt->nodes += 2;
            float tel, ter;
            bool hl = box_hit_te(a.x, a.y, a.z, b.x, b.y, b.z, o, inv, tmin, closest, tel);
            bool hr = box_hit_te(c.x, c.y, c.z, e.x, e.y, e.z, o, inv, tmin, closest, ter);
            int axis = __float_as_int(c.w);
            float da = axis == 0 ? d.x : (axis == 1 ? d.y : d.z);
            // An opaque any-hit answer does not depend on the visit order, so
            // that walk enters the child whose box the ray meets first (an
            // occluder near the origin ends it sooner); every other walk, and
            // the counting build, keeps BvhNode's order (near child by the sign
            // of the ray along the split axis).
            bool left_near = (ANY && !cnt) ? (tel <= ter) : (da >= 0.0f);
            int lc = __float_as_int(a.w), rc = __float_as_int(b.w);
            int nc = left_near ? lc : rc, fc = left_near ? rc : lc;
            bool hn = left_near ? hl : hr, hf = left_near ? hr : hl;
            float tf = left_near ? ter : tel;
            if (hn && hf) {
                if (sp >= STACK) {
                    *err = RT_ERR_STACK;
                    return false;
                }
                push(fc, tf);
            }
            code = hn ? nc : (hf ? fc : kNone);
        }
        // A leaf (or nothing): primitives in order.
        if (code != kNone) {
            int v = ~code;
            int first = v >> 5;
            int kind = (v >> 3) & 3;
            int count = (v & 7) + 1;
            code = kNone;
            if (kind == LEAF_ENT1) {
                Entity en = s.entities[RT_IX(first, s.n_entities)];
                if (en.kind == ENT_MESH) {   // Mesh.Hit -> its BVH root (box test) or flat list
                    if (en.index >= 0) {
                        if (cnt) cnt->nodes++;
                        float4 lo = ldg_scene(s.ent_box + 2 * RT_IX(first, s.n_entities)),
                               hi = ldg_scene(s.ent_box + 2 * RT_IX(first, s.n_entities) + 1);
                        float te;
                        if (box_hit_te(lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, o, inv, tmin, closest, te)) {
                            code = en.index;
                            continue;
                        }
                    } else {
                        code = en.index;   // <= 4 triangles: HittableList, no box test
                        continue;
                    }
                } else {
                    if (cnt) cnt->others++;
                    Hit h;
                    if (entity_test(s, first, o, d, tmin, closest, h)) {
                        best = h;
                        closest = h.t;
                        if (ANY) return true;
                    }
                }
            } else if (kind == LEAF_ENTS) {   // top-level fat leaf: entities in order
                if (sp + count > STACK) {
                    *err = RT_ERR_STACK;
                    return false;
                }
                for (int i = count - 1; i >= 0; --i)
                    push(leaf_code(s.top_items[RT_IX(first + i, s.num_top_items)], LEAF_ENT1, 1), -kInf);
            } else {   // triangle leaf (or a mesh's flat list)
                for (int i = 0; i < count; i++) {
                    float t, u, vv;
                    if (cnt) cnt->tris++;
                    if (tri_test(s.tris, RT_IX(first + i, s.n_tris), o, d, tmin, closest, t, u, vv)) {
                        best = Hit{t, u, vv, HIT_TRI, first + i};
                        closest = t;
                        if (ANY) return true;
                    }
                }
            }
        }
        // Pop the next entry the current closest t does not prune.
        if (ANY) {
            if (sp > 0) code = stc[--sp];
        } else {
            while (sp > 0) {
                int2 e = st[--sp];
                if (!(__int_as_float(e.y) > closest)) {
                    code = e.x;
                    break;
                }
            }
        }
        if (code == kNone) return true;
    }
}

// The same walk over the four-wide records (SceneView::cnodes4). A record tests
// the boxes of up to four grandchildren of a binary node at once and visits
// the hit ones in the binary tree's order for this ray (near group first by
// the node's split axis, then near first within each group by the child's
// axis), pushing the others in reverse. A grandchild box lies inside its
// parent's box (the build takes exact float unions), so a hit on it implies
// the hit the binary walk would have required first; pruning at pop time is
// the same entry-distance test. The primitive test sequence, hence the hit
// and the tie-breaking, is the binary walk's.
RT_D float sel4(int j, float a, float b, float c, float d) { return j == 0 ? a : (j == 1 ? b : (j == 2 ? c : d)); }
RT_D int sel4i(int j, int a, int b, int c, int d) { return j == 0 ? a : (j == 1 ? b : (j == 2 ? c : d)); }

template <bool ANY, int STACK>
__device__ __forceinline__ bool traverse4(const SceneView& s, V3 o, V3 d, float tmin, float tmax, Hit& best,
                                          int* err) {
    const int kNone = INT_MIN;
    V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);   // Core/Ray.cs:43
    int st_code[STACK];
    float st_te[STACK];
    int sp = 0;
    float closest = tmax;
    best.kind = HIT_NONE;
    int code = kNone;
    if (s.top_is_bvh) {
        code = s.top_root4;
    } else {
        for (int i = s.num_top_items - 1; i >= 0; --i) {
            st_code[sp] = leaf_code(s.top_items[RT_IX(i, s.num_top_items)], LEAF_ENT1, 1);
            st_te[sp] = -kInf;
            sp++;
        }
    }
    for (;;) {
        while (code >= 0) {
            const float4* q = s.cnodes4 + (size_t)RT_IX(code, s.n_cnodes4) * 8;
            float4 lx = ldg_scene(q), ly = ldg_scene(q + 1), lz = ldg_scene(q + 2);
            float4 hx = ldg_scene(q + 3), hy = ldg_scene(q + 4), hz = ldg_scene(q + 5);
            float4 cc = ldg_scene(q + 6), mt = ldg_scene(q + 7);
            int c0 = __float_as_int(cc.x), c1 = __float_as_int(cc.y), c2 = __float_as_int(cc.z),
                c3 = __float_as_int(cc.w);
            float t0, t1, t2, t3;
            int hm = 0;
            if (box_hit_te(lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, o, inv, tmin, closest, t0) && c0 != kNone) hm |= 1;
            if (box_hit_te(lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, o, inv, tmin, closest, t1) && c1 != kNone) hm |= 2;
            if (box_hit_te(lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, o, inv, tmin, closest, t2) && c2 != kNone) hm |= 4;
            if (box_hit_te(lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, o, inv, tmin, closest, t3) && c3 != kNone) hm |= 8;
            code = kNone;
            if (!hm) break;
            int axn = __float_as_int(mt.x), axl = __float_as_int(mt.y), axr = __float_as_int(mt.z);
            bool ln = (axn == 0 ? d.x : (axn == 1 ? d.y : d.z)) >= 0.0f;
            bool l0 = (axl == 0 ? d.x : (axl == 1 ? d.y : d.z)) >= 0.0f;
            bool r0 = (axr == 0 ? d.x : (axr == 1 ? d.y : d.z)) >= 0.0f;
            int la = l0 ? 0 : 1, lb = l0 ? 1 : 0, ra = r0 ? 2 : 3, rb = r0 ? 3 : 2;
            // slots in visit order v0..v3; walk them backwards, pushing all but the first hit
            int v0 = ln ? la : ra, v1 = ln ? lb : rb, v2 = ln ? ra : la, v3 = ln ? rb : lb;
            int pend = -1;
#pragma unroll
            for (int k = 3; k >= 0; --k) {
                int j = k == 0 ? v0 : (k == 1 ? v1 : (k == 2 ? v2 : v3));
                if (!((hm >> j) & 1)) continue;
                if (pend >= 0) {
                    if (sp >= STACK) {
                        *err = RT_ERR_STACK;
                        return false;
                    }
                    st_code[sp] = sel4i(pend, c0, c1, c2, c3);
                    st_te[sp] = sel4(pend, t0, t1, t2, t3);
                    sp++;
                }
                pend = j;
            }
            code = sel4i(pend, c0, c1, c2, c3);
        }
        if (code != kNone) {
            int v = ~code;
            int first = v >> 5;
            int kind = (v >> 3) & 3;
            int count = (v & 7) + 1;
            code = kNone;
            if (kind == LEAF_ENT1) {
                Entity en = s.entities[RT_IX(first, s.n_entities)];
                if (en.kind == ENT_MESH) {
                    int r4 = __ldg(s.mesh_root4 + RT_IX(first, s.n_entities));
                    if (en.index >= 0) {
                        float4 lo = ldg_scene(s.ent_box + 2 * RT_IX(first, s.n_entities)),
                               hi = ldg_scene(s.ent_box + 2 * RT_IX(first, s.n_entities) + 1);
                        float te;
                        if (box_hit_te(lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, o, inv, tmin, closest, te)) {
                            code = r4;
                            continue;
                        }
                    } else {
                        code = r4;
                        continue;
                    }
                } else {
                    Hit h;
                    if (entity_test(s, first, o, d, tmin, closest, h)) {
                        best = h;
                        closest = h.t;
                        if (ANY) return true;
                    }
                }
            } else if (kind == LEAF_ENTS) {
                if (sp + count > STACK) {
                    *err = RT_ERR_STACK;
                    return false;
                }
                for (int i = count - 1; i >= 0; --i) {
                    st_code[sp] = leaf_code(s.top_items[RT_IX(first + i, s.num_top_items)], LEAF_ENT1, 1);
                    st_te[sp] = -kInf;
                    sp++;
                }
            } else {
                for (int i = 0; i < count; i++) {
                    float t, u, vv;
                    if (tri_test(s.tris, RT_IX(first + i, s.n_tris), o, d, tmin, closest, t, u, vv)) {
                        best = Hit{t, u, vv, HIT_TRI, first + i};
                        closest = t;
                        if (ANY) return true;
                    }
                }
            }
        }
        while (sp > 0) {
            --sp;
            if (!(st_te[sp] > closest)) {
                code = st_code[sp];
                break;
            }
        }
        if (code == kNone) return true;
    }
}

// Opaque any-hit over the four-wide records. The answer (is anything hit in
// [tmin, tmax]) does not depend on the visit order, so this walk keeps none:
// every hit slot of a record is taken, the first one at once and the others
// from a stack of codes, and the first accepted primitive ends the walk. A
// grandchild box holds every primitive below it, so no primitive the
// two-wide walk could hit is skipped.
template <int STACK>
__device__ __forceinline__ bool traverse4_any(const SceneView& s, V3 o, V3 d, float tmin, float tmax, Hit& best,
                                              int* err) {
    const int kNone = INT_MIN;
    V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);   // Core/Ray.cs:43
    int stc[STACK];
    int sp = 0;
    best.kind = HIT_NONE;
    int code = kNone;
    if (s.top_is_bvh) {
        code = s.top_root4;
    } else {
        for (int i = s.num_top_items - 1; i >= 0; --i) stc[sp++] = leaf_code(s.top_items[RT_IX(i, s.num_top_items)],
                                                                                LEAF_ENT1, 1);
    }
    for (;;) {
        while (code >= 0) {
            const float4* q = s.cnodes4 + (size_t)RT_IX(code, s.n_cnodes4) * 8;
            float4 lx = ldg_scene(q), ly = ldg_scene(q + 1), lz = ldg_scene(q + 2);
            float4 hx = ldg_scene(q + 3), hy = ldg_scene(q + 4), hz = ldg_scene(q + 5);
            float4 cc = ldg_scene(q + 6);
            int c[4] = {__float_as_int(cc.x), __float_as_int(cc.y), __float_as_int(cc.z), __float_as_int(cc.w)};
            float te;
            bool h[4];
            h[0] = c[0] != kNone && box_hit_te(lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, o, inv, tmin, tmax, te);
            h[1] = c[1] != kNone && box_hit_te(lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, o, inv, tmin, tmax, te);
            h[2] = c[2] != kNone && box_hit_te(lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, o, inv, tmin, tmax, te);
            h[3] = c[3] != kNone && box_hit_te(lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, o, inv, tmin, tmax, te);
            // enter the first hit slot, stack the others (entering the slot the
            // ray meets first instead: occlude 54.4 against 49.1 ms per 64-spp
            // icosphere frame; the selection costs more than earlier exits win)
            code = kNone;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (!h[j]) continue;
                if (code == kNone) {
                    code = c[j];
                } else {
                    if (sp >= STACK) {
                        *err = RT_ERR_STACK;
                        return false;
                    }
                    stc[sp++] = c[j];
                }
            }
        }
        if (code != kNone) {
            int v = ~code;
            int first = v >> 5;
            int kind = (v >> 3) & 3;
            int count = (v & 7) + 1;
            code = kNone;
            if (kind == LEAF_ENT1) {
                Entity en = s.entities[RT_IX(first, s.n_entities)];
                if (en.kind == ENT_MESH) {
                    int r4 = __ldg(s.mesh_root4 + RT_IX(first, s.n_entities));
                    if (en.index >= 0) {
                        float4 lo = ldg_scene(s.ent_box + 2 * RT_IX(first, s.n_entities)),
                               hi = ldg_scene(s.ent_box + 2 * RT_IX(first, s.n_entities) + 1);
                        float te;
                        if (box_hit_te(lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, o, inv, tmin, tmax, te)) code = r4;
                    } else {
                        code = r4;
                    }
                    if (code != kNone) continue;
                } else {
                    Hit hh;
                    if (entity_test(s, first, o, d, tmin, tmax, hh)) {
                        best = hh;
                        return true;
                    }
                }
            } else if (kind == LEAF_ENTS) {
                if (sp + count > STACK) {
                    *err = RT_ERR_STACK;
                    return false;
                }
                for (int i = count - 1; i >= 0; --i)
                    stc[sp++] = leaf_code(s.top_items[RT_IX(first + i, s.num_top_items)], LEAF_ENT1, 1);
            } else {
                for (int i = 0; i < count; i++) {
                    float t, u, vv;
                    if (tri_test(s.tris, RT_IX(first + i, s.n_tris), o, d, tmin, tmax, t, u, vv)) {
                        best = Hit{t, u, vv, HIT_TRI, first + i};
                        return true;
                    }
                }
            }
        }
        if (sp == 0) return true;
        code = stc[--sp];
    }
}

// The node layout as a template switch (counting builds use the two-wide one).
template <bool ANY, int STACK, bool L4>
__device__ __forceinline__ bool trace(const SceneView& s, V3 o, V3 d, float tmin, float tmax, Hit& best,
                                      TravCounters* cnt, int* err) {
    if (L4 && ANY) return traverse4_any<STACK>(s, o, d, tmin, tmax, best, err);
    if (L4) return traverse4<ANY, STACK>(s, o, d, tmin, tmax, best, err);
    return traverse<ANY, STACK>(s, o, d, tmin, tmax, best, cnt, err);
}

// Surface record of an accepted hit (Core/HitRecord.cs fields on the path).
struct Surface {
    V3 p, n, tangent, bitangent;
    float t;
    int front;
    int material;
    int entity;
    int prim;
};

RT_D Surface make_surface(const SceneView& s, const Hit& h, V3 o, V3 d) {
    Surface r;
    r.t = h.t;
    r.p = o + h.t * d;   // Ray.At
    if (h.kind == HIT_TRI) {
        int ti = RT_IX(h.slot, s.n_tris);
        const float4* tp = s.tris + 3 * ti;
        float4 a0 = ldg_scene(tp), a1 = ldg_scene(tp + 1), a2 = ldg_scene(tp + 2);
        V3 e1 = ld3(a1), e2 = ld3(a2);
        V3 n = v3(a0.w, a1.w, a2.w);
        r.front = dot(d, n) < 0.0f;   // HitRecord.SetFaceNormal
        r.n = r.front ? n : -n;
        int si = s.tri_smooth ? s.tri_smooth[ti] : -1;
        if (si >= 0) {   // SmoothTriangle.Hit (Geometry/SmoothTriangle.cs:166-197)
            const SmoothTri& st = s.smooth[RT_IX(si, s.n_smooth)];
            float w0 = 1.0f - h.u - h.v;
            V3 sn = normalize(w0 * st.n0 + h.u * st.n1 + h.v * st.n2);
            r.n = r.front ? sn : -sn;   // the face normal decides the side
            r.tangent = st.tangent;
            r.bitangent = st.bitangent;
        } else {
            r.tangent = length_sq(e1) > 0.0f ? normalize(e1) : v3(1.0f, 0.0f, 0.0f);
            r.bitangent = length_sq(e2) > 0.0f ? normalize(e2) : v3(0.0f, 0.0f, 1.0f);
        }
        r.entity = s.tri_entity[ti];
        r.prim = s.tri_local[ti];
    } else if (h.kind == HIT_QUAD) {
        Entity en = s.entities[RT_IX(h.slot, s.n_entities)];
        const QuadData& q = s.quads[RT_IX(en.index, s.n_quads)];
        r.front = dot(d, q.normal) < 0.0f;
        r.n = r.front ? q.normal : -q.normal;
        r.tangent = q.tangent;
        r.bitangent = q.bitangent;
        r.entity = h.slot;
        r.prim = 0;
    } else {
        Entity en = s.entities[RT_IX(h.slot, s.n_entities)];
        const SphereData& sp = s.spheres[RT_IX(en.index, s.n_spheres)];
        V3 outward = (r.p - sp.c) / sp.r;
        r.front = dot(d, outward) < 0.0f;
        r.n = r.front ? outward : -outward;
        V3 td = cross(v3(0.0f, 1.0f, 0.0f), outward);
        if (length_sq(td) < 1e-4f) td = v3(1.0f, 0.0f, 0.0f);
        r.tangent = normalize(td);
        r.bitangent = normalize(cross(outward, r.tangent));
        r.entity = h.slot;
        r.prim = 0;
    }
    r.material = RT_IX(s.entities[RT_IX(r.entity, s.n_entities)].material, s.n_materials);
    return r;
}

// ---------------------------------------------------------------------------
// Kulla-Conty LUT lookups (Materials/EnergyCompensationLut.cs:140-175)
// ---------------------------------------------------------------------------
RT_D float lut_e(const float* e, float mu, float alpha) {
    mu = clampf(mu, 0.0f, 1.0f);
    alpha = clampf(alpha, 0.001f, 1.0f);
    float fmu = mu * 32.0f - 0.5f;
    float fal = alpha * 32.0f - 0.5f;
    int m0 = min(max((int)floorf(fmu), 0), 31);
    int a0 = min(max((int)floorf(fal), 0), 31);
    int m1 = min(m0 + 1, 31);
    int a1 = min(a0 + 1, 31);
    float tu = clampf(fmu - (float)m0, 0.0f, 1.0f);
    float ta = clampf(fal - (float)a0, 0.0f, 1.0f);
    float e00 = __ldg(e + m0 * 32 + a0), e01 = __ldg(e + m0 * 32 + a1);
    float e10 = __ldg(e + m1 * 32 + a0), e11 = __ldg(e + m1 * 32 + a1);
    float x0 = e00 + (e01 - e00) * ta;
    float x1 = e10 + (e11 - e10) * ta;
    return x0 + (x1 - x0) * tu;
}

// ---------------------------------------------------------------------------
// Microfacet helpers (Materials/Microfacet.cs) and Charlie sheen
// (Materials/SheenCharlie.cs)
// ---------------------------------------------------------------------------
RT_D void tangent_frame(V3 n, V3& t, V3& b) {   // Microfacet.cs:22-37
    if (n.z < -0.999f) {
        t = v3(0.0f, -1.0f, 0.0f);
        b = v3(-1.0f, 0.0f, 0.0f);
    } else {
        float a = 1.0f / (1.0f + n.z);
        float bb = -n.x * n.y * a;
        t = v3(1.0f - n.x * n.x * a, bb, -n.x);
        b = v3(bb, 1.0f - n.y * n.y * a, -n.y);
    }
}
RT_D float d_ggx(V3 h, float ax, float ay) {   // :43-49
    float hx = h.x / ax;
    float hy = h.y / ay;
    float d = hx * hx + hy * hy + h.z * h.z;
    return 1.0f / fmaxf(kPi * ax * ay * d * d, 1e-20f);
}
RT_D float g1_ggx(V3 w, float ax, float ay) {   // :55-69
    float c2 = w.z * w.z;
    float lam;
    if (c2 < 1e-14f) {
        lam = 1e10f;
    } else {
        float num = (ax * w.x) * (ax * w.x) + (ay * w.y) * (ay * w.y);
        lam = 0.5f * (-1.0f + sqrtf(1.0f + num / c2));
    }
    return 1.0f / (1.0f + lam);
}
RT_D float smith_g1(float ndx, float alpha) {   // :75-81
    float a2 = alpha * alpha;
    float n2 = ndx * ndx;
    float denom = ndx + sqrtf(a2 + (1.0f - a2) * n2);
    return 2.0f * ndx / fmaxf(denom, 1e-7f);
}
RT_D V3 sample_vndf(V3 vl, float ax, float ay, float u1, float u2) {   // :100-124
    V3 vh = normalize(v3(ax * vl.x, ay * vl.y, vl.z));
    float lsq = vh.x * vh.x + vh.y * vh.y;
    V3 t1 = lsq > 0.0f ? v3(-vh.y, vh.x, 0.0f) / sqrtf(lsq) : v3(1.0f, 0.0f, 0.0f);
    V3 t2 = cross(vh, t1);
    float r = sqrtf(u1);
    float phi = 2.0f * kPi * u2;
    float sn, cs;
    sincosf(phi, &sn, &cs);
    float a1 = r * cs;
    float a2 = r * sn;
    float s = 0.5f * (1.0f + vh.z);
    a2 = (1.0f - s) * sqrtf(fmaxf(0.0f, 1.0f - a1 * a1)) + s * a2;
    V3 nh = a1 * t1 + a2 * t2 + sqrtf(fmaxf(0.0f, 1.0f - a1 * a1 - a2 * a2)) * vh;
    return normalize(v3(ax * nh.x, ay * nh.y, fmaxf(0.0f, nh.z)));
}
RT_D float sheen_lambda_log(float c, bool smooth) {   // SheenCharlie.cs:40-65
    float a, b, cc, d, e;
    if (smooth) {
        a = 25.3245f; b = 3.32435f; cc = 0.16801f; d = -1.27393f; e = -4.85967f;
    } else {
        a = 21.5473f; b = 3.82987f; cc = 0.19823f; d = -1.97760f; e = -4.32054f;
    }
    return a / (1.0f + b * powf(c, cc)) + d * c + e;
}
RT_D float sheen_lambda(float c, float alpha) {   // :71-85
    c = clampf(c, 1e-4f, 1.0f);
    if (alpha <= 0.25f - 0.05f) return expf(sheen_lambda_log(c, true));
    if (alpha >= 0.25f + 0.05f) return expf(sheen_lambda_log(c, false));
    float t = (alpha - (0.25f - 0.05f)) / (2.0f * 0.05f);
    float lo = expf(sheen_lambda_log(c, true));
    float hi = expf(sheen_lambda_log(c, false));
    return lo + (hi - lo) * t;
}
RT_D float sheen_brdf(float ndv, float ndl, float ndh, float alpha) {   // :24-34, :92-121
    float denom = 4.0f * fmaxf(ndv, 1e-6f) * fmaxf(ndl, 1e-6f);
    float g = 1.0f / ((1.0f + sheen_lambda(ndv, alpha)) * (1.0f + sheen_lambda(ndl, alpha)));
    float al = fmaxf(alpha, 0.04f);
    float inv = 1.0f / al;
    float c2 = ndh * ndh;
    float s2 = fmaxf(1.0f - c2, 0.0f);
    float sp = powf(s2, 0.5f * inv);
    float D = (2.0f + inv) * sp / (2.0f * kPi);
    return D * g / denom;
}
RT_D float schlick_weight(float c) {   // DisneyBsdf.cs:1994-1999
    float x = clampf(1.0f - c, 0.0f, 1.0f);
    float x2 = x * x;
    return x2 * x2 * x;
}
RT_D V3 fresnel_schlick(float c, V3 f0) {   // :1963-1967 (thin film off)
    float w = schlick_weight(c);
    return f0 + (v3(1.0f) - f0) * w;
}
RT_D float fresnel_dielectric(float ci, float eta) {   // Core/MathUtils.cs:191-201
    ci = clampf(ci, 0.0f, 1.0f);
    float s2i = fmaxf(0.0f, 1.0f - ci * ci);
    float s2t = eta * eta * s2i;
    if (s2t >= 1.0f) return 1.0f;
    float ct = sqrtf(1.0f - s2t);
    float rpa = (ci - eta * ct) / (ci + eta * ct);
    float rpe = (eta * ci - ct) / (eta * ci + ct);
    return 0.5f * (rpa * rpa + rpe * rpe);
}
RT_D V3 refract(V3 uv, V3 n, float eta) {   // Core/MathUtils.cs:160-166
    float ct = fminf(dot(-uv, n), 1.0f);
    V3 perp = eta * (uv + ct * n);
    V3 par = -sqrtf(fabsf(1.0f - length_sq(perp))) * n;
    return perp + par;
}

// ---------------------------------------------------------------------------
// Disney BSDF (Materials/DisneyBsdf.cs) on host-precomputed material constants
// ---------------------------------------------------------------------------
struct Frame {
    V3 t, b, n;
    RT_D V3 to_local(V3 w) const { return v3(dot(w, t), dot(w, b), dot(w, n)); }
    RT_D V3 to_world(V3 w) const { return w.x * t + w.y * b + w.z * n; }
};

RT_D Frame shading_frame(const Surface& rec, const Material& m) {   // :1840-1877
    V3 n = rec.n, t, b;
    if (length_sq(rec.tangent) > 1e-10f && length_sq(rec.bitangent) > 1e-10f) {
        t = rec.tangent - dot(rec.tangent, n) * n;
        float tl = length_sq(t);
        if (tl > 1e-10f) {
            t = t / sqrtf(tl);
            b = cross(n, t);
        } else {
            tangent_frame(n, t, b);
        }
    } else {
        tangent_frame(n, t, b);
    }
    if (m.has_rotation) {
        float c = m.rot_cos, s = m.rot_sin;
        V3 tr = c * t + s * b;
        V3 br = -s * t + c * b;
        t = tr;
        b = br;
    }
    return Frame{t, b, n};
}

RT_D V3 multiscatter_weight(const SceneView& s, const Material& m, float ndv, float ndl) {   // :1906-1926
    float e_out = lut_e(s.lut_e, ndv, m.alpha_iso);
    float e_in = lut_e(s.lut_e, ndl, m.alpha_iso);
    float e_avg = m.e_avg;
    float one_m = fmaxf(1.0f - e_avg, 1e-6f);
    V3 f_avg = m.f0 + (v3(1.0f) - m.f0) * (1.0f / 21.0f);
    V3 den = v3(1.0f) - f_avg * (1.0f - e_avg);
    den = v3(fmaxf(den.x, 1e-6f), fmaxf(den.y, 1e-6f), fmaxf(den.z, 1e-6f));
    V3 f_ms = f_avg * f_avg * e_avg / den;
    return f_ms * ((1.0f - e_out) * (1.0f - e_in) / one_m);
}

// EvaluateDirect (:418-535): f(V,L) * max(N.L, 0), the NEE integrand.
RT_D V3 bsdf_eval_direct(const SceneView& s, const Material& m, const Surface& rec, V3 L, V3 V, V3 N) {
    float ndl = fmaxf(dot(N, L), 0.0f);
    if (ndl <= 0.0f) return v3(0.0f);
    float ndv = fmaxf(dot(N, V), 0.001f);
    V3 H = normalize(L + V);
    float ndh = fmaxf(dot(N, H), 0.0f);
    float vdh = fmaxf(dot(V, H), 0.0f);
    float ldh = fmaxf(dot(L, H), 0.0f);
    V3 bc = m.base;
    V3 diffuse = v3(0.0f);
    if (m.diffuse_w > 0.0f) {
        float fd90 = 0.5f + 2.0f * m.roughness * ldh * ldh;
        float fi = schlick_weight(ndv), fo = schlick_weight(ndl);
        float fd = (1.0f + (fd90 - 1.0f) * fi) * (1.0f + (fd90 - 1.0f) * fo);
        diffuse = bc * fd * (m.diffuse_w * ndl / kPi);
    }
    V3 specular = v3(0.0f);
    if (m.alpha > kDeltaAlpha) {
        Frame fr = shading_frame(rec, m);
        V3 vl = fr.to_local(V), ll = fr.to_local(L), hl = fr.to_local(H);
        float D = d_ggx(hl, m.alpha_x, m.alpha_y);
        float G = g1_ggx(vl, m.alpha_x, m.alpha_y) * g1_ggx(ll, m.alpha_x, m.alpha_y);
        V3 F = fresnel_schlick(vdh, m.f0);
        specular = D * G * F / fmaxf(4.0f * ndv, 1e-6f);
    }
    V3 clearcoat = v3(0.0f);
    if (m.clearcoat > 0.0f && m.cc_alpha > kDeltaAlpha) {
        V3 cn = rec.n;
        float cndv = fmaxf(dot(cn, V), 0.001f);
        float cndl = dot(cn, L);
        if (cndl > 0.0f) {
            float cndh = fmaxf(dot(cn, H), 0.0f);
            float cvdh = fmaxf(dot(V, H), 0.0f);
            float ca2 = m.cc_alpha * m.cc_alpha;
            float cden = cndh * cndh * (ca2 - 1.0f) + 1.0f;
            float cD = ca2 / (kPi * cden * cden);
            float cG = smith_g1(cndv, m.cc_alpha) * smith_g1(cndl, m.cc_alpha);
            float cF = m.cc_f0 + (1.0f - m.cc_f0) * schlick_weight(cvdh);
            clearcoat = v3(m.clearcoat * 0.25f * cD * cG * cF / fmaxf(4.0f * cndv, 1e-6f));
        }
    }
    V3 sheen = v3(0.0f);
    if (m.sheen > 0.0f && m.diffuse_w > 0.0f) {
        float sb = sheen_brdf(ndv, ndl, ndh, m.sheen_roughness);
        sheen = m.sheen * sb * m.sheen_col * ndl;
    }
    V3 ms = multiscatter_weight(s, m, ndv, ndl) * (1.0f / kPi) * ndl;
    return diffuse + sheen + specular + ms + clearcoat;
}

// Evaluate (:649-771): f(V, L) without the cosine.
RT_D V3 bsdf_eval(const SceneView& s, const Material& m, const Surface& rec, V3 V, V3 L) {
    V3 N = rec.n;
    float ndl = dot(N, L);
    float ndv = dot(N, V);
    if (ndv <= 0.0f) return v3(0.0f);
    V3 bc = m.base;
    if (ndl <= 0.0f) {
        if (m.diff_all <= 0.0f || m.diff_trans <= 0.0f) return v3(0.0f);
        return bc * (m.diff_all * m.diff_trans / kPi);
    }
    V3 hraw = V + L;
    float hl2 = length_sq(hraw);
    if (hl2 < 1e-14f) return v3(0.0f);
    V3 H = hraw / sqrtf(hl2);
    float ndh = fmaxf(dot(N, H), 0.0f);
    float vdh = fmaxf(dot(V, H), 0.0f);
    float ldh = fmaxf(dot(L, H), 0.0f);
    V3 diffuse = v3(0.0f);
    if (m.diffuse_w > 0.0f) {
        float fd90 = 0.5f + 2.0f * m.roughness * ldh * ldh;
        float fi = schlick_weight(ndv), fo = schlick_weight(ndl);
        float fd = (1.0f + (fd90 - 1.0f) * fi) * (1.0f + (fd90 - 1.0f) * fo);
        diffuse = bc * fd * (m.diffuse_w / kPi);
    }
    V3 sheen = v3(0.0f);
    if (m.sheen > 0.0f && m.diffuse_w > 0.0f) {
        float sb = sheen_brdf(ndv, ndl, ndh, m.sheen_roughness);
        sheen = m.sheen * sb * m.sheen_col;
    }
    Frame fr = shading_frame(rec, m);
    V3 vl = fr.to_local(V), ll = fr.to_local(L), hl = fr.to_local(H);
    float D = d_ggx(hl, m.alpha_x, m.alpha_y);
    float G = g1_ggx(vl, m.alpha_x, m.alpha_y) * g1_ggx(ll, m.alpha_x, m.alpha_y);
    V3 F = fresnel_schlick(vdh, m.f0);
    V3 specular = D * G / fmaxf(4.0f * ndv * ndl, 1e-7f) * F;
    V3 clearcoat = v3(0.0f);
    if (m.clearcoat > 0.0f) {
        V3 cn = rec.n;
        float cndv = dot(cn, V), cndl = dot(cn, L);
        if (cndv > 0.0f && cndl > 0.0f) {
            float cndh = fmaxf(dot(cn, H), 0.0f);
            float cvdh = fmaxf(dot(V, H), 0.0f);
            float ca2 = m.cc_alpha * m.cc_alpha;
            float cden = cndh * cndh * (ca2 - 1.0f) + 1.0f;
            float cD = ca2 / (kPi * cden * cden);
            float cG = smith_g1(cndv, m.cc_alpha) * smith_g1(cndl, m.cc_alpha);
            float cF = m.cc_f0 + (1.0f - m.cc_f0) * schlick_weight(cvdh);
            float cc = m.clearcoat * 0.25f * cD * cG * cF / fmaxf(4.0f * cndv * cndl, 1e-7f);
            clearcoat = v3(cc);
        }
    }
    V3 ms = multiscatter_weight(s, m, ndv, ndl) * (1.0f / kPi);
    return diffuse + sheen + specular + ms + clearcoat;
}

// Pdf (:783-870): the one-sample mixture density of Sample.
RT_D float bsdf_pdf(const Material& m, const Surface& rec, V3 V, V3 L) {
    V3 N = rec.n;
    float ndl = dot(N, L);
    float ndv = dot(N, V);
    if (ndv <= 0.0f) return 0.0f;
    float cos_pdf = ndl > 0.0f ? ndl / kPi : 0.0f;
    float dt_pdf = ndl < 0.0f ? -ndl / kPi : 0.0f;
    float spec_pdf = 0.0f, cc_pdf = 0.0f;
    V3 hraw = V + L;
    float hl2 = length_sq(hraw);
    if (hl2 >= 1e-14f) {
        V3 H = hraw / sqrtf(hl2);
        float ndh = dot(N, H);
        if (ndh > 0.0f && m.alpha > kDeltaAlpha) {
            float sndv = fmaxf(ndv, 1e-7f);
            Frame fr = shading_frame(rec, m);
            V3 vl = fr.to_local(V), hl = fr.to_local(H);
            float D = d_ggx(hl, m.alpha_x, m.alpha_y);
            float g1v = g1_ggx(vl, m.alpha_x, m.alpha_y);
            spec_pdf = g1v * D / (4.0f * sndv);
        }
        if (m.cc_alpha > kDeltaAlpha) {
            V3 cn = rec.n;
            float cndv = dot(cn, V), cndh = dot(cn, H);
            if (cndv > 0.0f && cndh > 0.0f) {
                float sc = fmaxf(cndv, 1e-7f);
                float ca2 = m.cc_alpha * m.cc_alpha;
                float cden = cndh * cndh * (ca2 - 1.0f) + 1.0f;
                float cD = ca2 / (kPi * cden * cden);
                float cg1 = smith_g1(cndv, m.cc_alpha);
                cc_pdf = cg1 * cD / (4.0f * sc);
            }
        }
    }
    return m.p_d * cos_pdf + m.p_sh * cos_pdf + m.p_ms * cos_pdf + m.p_s * spec_pdf + m.p_c * cc_pdf +
           m.p_dt * dt_pdf;
}

enum : int { LOBE_DIFFUSE = 0, LOBE_SPECULAR, LOBE_TRANSMISSION, LOBE_SHEEN, LOBE_MULTISCATTER, LOBE_DIFFTRANS,
             LOBE_CLEARCOAT };

RT_D bool any_nonfinite(V3 a) { return !isfinite(a.x) || !isfinite(a.y) || !isfinite(a.z); }

// ScatterInternal (:1176-1248) with the lobe samplers (:1263-1709). ray_dir is
// the incoming ray direction; V = normalize(-ray_dir). When a reflection lobe
// fails, *tried (if given) receives the direction it drew.
// TRANSMIT = false compiles the specular-transmission lobe out, for batches in
// which no material has specTrans > 0: there p_t is exactly 0, so the lobe is
// never picked and subtracting p_t leaves the draw unchanged.
template <bool TRANSMIT = true>
RT_D bool bsdf_scatter(const SceneView& s, const Material& m, const Surface& rec, V3 ray_dir, float relative_eta,
                       Sampler& rng, V3& att, V3& dir, int& lobe, V3* tried = nullptr) {
    V3 bc = m.base;
    V3 N = rec.n;
    V3 V = normalize(-ray_dir);
    float rnd = rng.next();
    bool ok = true;
    if (rnd < m.p_d) {   // ScatterDiffuse (:1263-1306)
        lobe = LOBE_DIFFUSE;
        V3 sd = N + random_unit_vector(rng);
        if (near_zero(sd)) sd = N;
        sd = normalize(sd);
        dir = sd;
        float ndv = fmaxf(dot(N, V), 0.001f);
        float ndl = fmaxf(dot(N, sd), 0.001f);
        V3 hraw = V + sd;
        float hl2 = length_sq(hraw);
        V3 H = hl2 > 1e-7f ? hraw / sqrtf(hl2) : N;
        float ldh = fmaxf(dot(sd, H), 0.0f);
        float fd90 = 0.5f + 2.0f * m.roughness * ldh * ldh;
        float fi = schlick_weight(ndv), fo = schlick_weight(ndl);
        float fd = (1.0f + (fd90 - 1.0f) * fi) * (1.0f + (fd90 - 1.0f) * fo);
        att = bc * fd;
        att = att * (1.0f - m.diff_trans);
        att = att / fmaxf(m.p_d, 0.1f);
    } else if ((rnd -= m.p_d) < m.p_s) {   // ScatterSpecular (:1399-1444)
        lobe = LOBE_SPECULAR;
        Frame fr = shading_frame(rec, m);
        V3 vl = fr.to_local(V);
        float u1 = rng.next();
        float u2 = rng.next();
        V3 hl = sample_vndf(vl, m.alpha_x, m.alpha_y, u1, u2);
        V3 H = fr.to_world(hl);
        V3 L = reflect(-V, H);
        if (dot(L, N) <= 0.0f) {
            att = v3(0.0f);
            dir = N;
            ok = false;
            if (tried) *tried = L;
        } else {
            dir = L;
            float vdh = fmaxf(dot(V, H), 1e-4f);
            V3 fres = fresnel_schlick(vdh, m.f0);
            float g1l = g1_ggx(fr.to_local(L), m.alpha_x, m.alpha_y);
            att = fres * g1l;
            att = att / fmaxf(m.p_s, 0.1f);
        }
    } else if ((rnd -= m.p_s), TRANSMIT && rnd < m.p_t) {   // ScatterTransmission (:1473-1608)
        lobe = LOBE_TRANSMISSION;
        bool thin = m.thin_walled != 0;
        float eta = thin ? (1.0f / m.ior) : (relative_eta > 0.0f ? relative_eta : (rec.front ? (1.0f / m.ior) : m.ior));
        V3 unit = normalize(ray_dir);
        Frame fr = shading_frame(rec, m);
        bool rough = m.roughness > 0.01f;
        V3 Ht;
        if (rough) {
            V3 vl = fr.to_local(V);
            float u1 = rng.next();
            float u2 = rng.next();
            Ht = fr.to_world(sample_vndf(vl, m.alpha_x, m.alpha_y, u1, u2));
        } else {
            Ht = N;
        }
        if (dot(Ht, unit) > 0.0f) Ht = -Ht;
        float ct = fminf(dot(-unit, Ht), 1.0f);
        float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        bool cannot = !thin && eta * st > 1.0f;
        float frs = cannot ? 1.0f : fresnel_dielectric(ct, eta);
        V3 d;
        bool is_refl;
        if (frs > rng.next()) {
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
        att = is_refl ? v3(1.0f) : m.trans_tint;
        if (rough) {
            V3 ll = fr.to_local(dir);
            ll.z = fabsf(ll.z);
            att = att * g1_ggx(ll, m.alpha_x, m.alpha_y);
        }
        att = att / fmaxf(m.p_t, 0.1f);
    } else if ((rnd -= m.p_t) < m.p_sh) {   // ScatterSheen (:1354-1388)
        lobe = LOBE_SHEEN;
        V3 sd = N + random_unit_vector(rng);
        if (near_zero(sd)) sd = N;
        sd = normalize(sd);
        dir = sd;
        float ndv = fmaxf(dot(N, V), 1e-4f);
        float ndl = fmaxf(dot(N, sd), 1e-4f);
        V3 hraw = V + sd;
        float hl2 = length_sq(hraw);
        V3 H = hl2 > 1e-7f ? hraw / sqrtf(hl2) : N;
        float ndh = fmaxf(dot(N, H), 0.0f);
        float sb = sheen_brdf(ndv, ndl, ndh, m.sheen_roughness);
        att = m.sheen * kPi * sb * m.sheen_col;
        att = att / fmaxf(m.p_sh, 0.1f);
    } else if ((rnd -= m.p_sh) < m.p_ms) {   // ScatterMultiscatter (:1688-1709)
        lobe = LOBE_MULTISCATTER;
        V3 sd = N + random_unit_vector(rng);
        if (near_zero(sd)) sd = N;
        sd = normalize(sd);
        dir = sd;
        float ndv = fmaxf(dot(N, V), 1e-3f);
        float ndl = fmaxf(dot(N, sd), 1e-3f);
        att = multiscatter_weight(s, m, ndv, ndl) / fmaxf(m.p_ms, 0.05f);
    } else if ((rnd -= m.p_ms) < m.p_dt) {   // ScatterDiffTrans (:1321-1338)
        lobe = LOBE_DIFFTRANS;
        V3 sd = -N + random_unit_vector(rng);
        if (near_zero(sd)) sd = -N;
        sd = normalize(sd);
        dir = sd;
        att = bc * m.diff_trans;
        att = att / fmaxf(m.p_dt, 0.05f);
    } else {   // ScatterClearcoat (:1623-1678)
        lobe = LOBE_CLEARCOAT;
        V3 cn = rec.n;
        V3 ct_, cb_;
        tangent_frame(cn, ct_, cb_);
        Frame fr{ct_, cb_, cn};
        if (dot(cn, V) <= 0.0f) {
            att = v3(0.0f);
            dir = N;
            ok = false;
        } else {
            V3 vl = fr.to_local(V);
            float u1 = rng.next();
            float u2 = rng.next();
            V3 H = fr.to_world(sample_vndf(vl, m.cc_alpha, m.cc_alpha, u1, u2));
            V3 L = reflect(-V, H);
            if (dot(L, N) <= 0.0f || dot(L, cn) <= 0.0f) {
                att = v3(0.0f);
                dir = N;
                ok = false;
            } else {
                dir = L;
                float cndl = fmaxf(dot(cn, L), 1e-4f);
                float cvdh = fmaxf(dot(V, H), 1e-4f);
                float fres = m.cc_f0 + (1.0f - m.cc_f0) * schlick_weight(cvdh);
                float g1l = smith_g1(cndl, m.cc_alpha);
                att = v3(fres * g1l);
                att = att / fmaxf(m.p_c, 0.1f);
            }
        }
    }
    if (any_nonfinite(att)) att = bc;
    return ok;
}

struct BsdfSample {
    V3 wo, f;
    float pdf;
    int is_delta;
    int lobe;
    int transition;            // 0 none, 1 enter, 2 exit
    int has_next_absorption;
    V3 next_absorption;
    V3 tried;                  // a null sample: the direction its lobe drew
};

// The rest of Sample (:893-997) once ScatterInternal has drawn (att, wo) with
// `lobe`. Returns false for a null sample.
template <bool TRANSMIT = true>
RT_D bool bsdf_sample_finish(const SceneView& s, const Material& m, const Surface& rec, V3 V, V3 att, V3 wo, int lobe,
                             BsdfSample& out) {
    float ndwo = dot(rec.n, wo);
    out.wo = wo;
    // Diffuse transmission and the non-delta reflection lobes both end in
    // Evaluate + Pdf; one call site serves both (the code is long).
    bool dt = lobe == LOBE_DIFFTRANS;
    if (!dt) {
        if (TRANSMIT && lobe == LOBE_TRANSMISSION) {
            if (ndwo < 0.0f && !m.thin_walled) {
                V3 sg = m.trans_sigma;
                bool has_sigma = sg.x > 0.0f || sg.y > 0.0f || sg.z > 0.0f;
                if (rec.front && has_sigma) {
                    out.has_next_absorption = 1;
                    out.next_absorption = sg;
                } else if (!rec.front) {
                    out.has_next_absorption = 1;
                    out.next_absorption = v3(0.0f);
                }
                out.transition = rec.front ? 1 : 2;
            }
            out.f = att;
            out.pdf = 1.0f;
            out.is_delta = 1;
            return true;
        }
        if (ndwo <= 0.0f) {
            out.tried = wo;
            return false;
        }
        bool nd_spec = lobe == LOBE_SPECULAR && m.alpha <= kDeltaAlpha;
        bool nd_coat = lobe == LOBE_CLEARCOAT && m.cc_alpha <= kDeltaAlpha;
        if (nd_spec || nd_coat) {
            out.f = att;
            out.pdf = 1.0f;
            out.is_delta = 1;
            return true;
        }
    }
    V3 fb = bsdf_eval(s, m, rec, V, wo);
    float pb = bsdf_pdf(m, rec, V, wo);
    if (dt && pb <= 0.0f) {   // a diffuse-transmission direction of zero density: a delta with its weight
        out.f = att;
        out.pdf = 1.0f;
        out.is_delta = 1;
        return true;
    }
    out.f = fb;
    out.pdf = pb;
    out.is_delta = 0;
    return true;
}

// Sample (:893-997). Returns false for a null sample.
template <bool TRANSMIT = true>
RT_D bool bsdf_sample(const SceneView& s, const Material& m, const Surface& rec, V3 V, float relative_eta,
                      Sampler& rng, BsdfSample& out) {
    V3 att, wo;
    int lobe = -1;
    out.transition = 0;
    out.has_next_absorption = 0;
    out.tried = rec.n;
    bool ok = bsdf_scatter<TRANSMIT>(s, m, rec, -V, relative_eta, rng, att, wo, lobe, &out.tried);
    out.lobe = lobe;
    if (!ok) return false;
    return bsdf_sample_finish<TRANSMIT>(s, m, rec, V, att, wo, lobe, out);
}

// ShadeSampleBounce's draw: Sample, and when it returns null the legacy
// Scatter draw the renderer falls back to (Renderer.cs:1127-1225), with fresh
// random numbers and the ray direction itself. Both draws go through one
// bsdf_scatter call site, so its long lobe samplers are compiled once.
// Returns 1 with `out` filled (a sample), 2 with (latt, ldir, llobe) (the
// legacy draw; out.lobe and out.tried describe the null sample), 0 when both
// fail.
template <bool TRANSMIT = true>
RT_D int bsdf_sample_or_scatter(const SceneView& s, const Material& m, const Surface& rec, V3 V, V3 ray_dir,
                                float relative_eta, Sampler& rng, BsdfSample& out, V3& latt, V3& ldir, int& llobe) {
    out.transition = 0;
    out.has_next_absorption = 0;
    out.tried = rec.n;
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
        V3 att, wo;
        int lobe = -1;
        bool ok = bsdf_scatter<TRANSMIT>(s, m, rec, pass == 0 ? -V : ray_dir, relative_eta, rng, att, wo, lobe,
                                         pass == 0 ? &out.tried : nullptr);
        if (pass == 1) {
            if (!ok) return 0;
            latt = att;
            ldir = wo;
            llobe = lobe;
            return 2;
        }
        out.lobe = lobe;
        if (ok && bsdf_sample_finish<TRANSMIT>(s, m, rec, V, att, wo, lobe, out)) return 1;
    }
    return 0;
}

// ShadowTransmittance (:560-584) and ShadowAbsorption (:609-614).
RT_D V3 bsdf_shadow_transmittance(const Material& m, V3 wi, const Surface& rec) {
    if (m.type != 0) return v3(0.0f);   // Emissive: IMaterial default (opaque)
    float st = m.spec_trans_raw;
    if (st <= 0.0f) return v3(0.0f);
    float eta = 1.0f / m.ior_raw;
    float c = fminf(fabsf(dot(wi, rec.n)), 1.0f);
    float fr = fresnel_dielectric(c, eta);
    return st * (1.0f - fr) * m.trans_tint;
}

// ---------------------------------------------------------------------------
// Lights (Lights/*.cs)
// ---------------------------------------------------------------------------
struct LightSample {
    int occluded;     // early "in shadow" (no shadow ray needed)
    int has_ray;      // a shadow ray must decide visibility
    V3 color;         // contribution before the shadow transmittance
    V3 dir;
    float dist;
    V3 ray_o;
    float ray_tmax;
};

// A direction in the cone of half-angle acos(cos_max) around w, uniform in
// solid angle (Sphere.SampleSolidAngleCore, Sphere.cs:160-169; SphereLight
// :87-96), through LocalToWorld (Sphere.cs:230-246).
RT_D V3 cone_dir(V3 w, float cos_max, float xi1, float xi2) {
    float ct = 1.0f - xi1 * (1.0f - cos_max);
    float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float phi = 2.0f * kPi * xi2;
    V3 loc = v3(st * cosf(phi), st * sinf(phi), ct);
    V3 uu, vv;
    tangent_frame(w, uu, vv);
    V3 res = loc.x * uu + loc.y * vv + loc.z * w;
    float l2 = length_sq(res);
    return l2 > 1e-8f ? res / sqrtf(l2) : w;
}

// Sphere.SolidAnglePdf (Sphere.cs:205-226) and SphereLight.PdfSolidAngle
// (SphereLight.cs:179-200), the same function of the cone.
RT_D float sphere_cone_pdf(V3 center, float radius, V3 p, V3 wi) {
    V3 tc = center - p;
    float d2 = length_sq(tc);
    float r2 = radius * radius;
    if (d2 <= r2) return 1.0f / (4.0f * kPi);   // observer inside: uniform sphere
    float cmax = sqrtf(fmaxf(0.0f, 1.0f - r2 / d2));
    float wl = length(wi);
    if (wl < kEps) return 0.0f;
    V3 wd = tc / sqrtf(d2);
    float ct = dot(wi, wd) / wl;
    if (ct < cmax) return 0.0f;
    float sa = 2.0f * kPi * (1.0f - cmax);
    return sa > kEps ? 1.0f / sa : 0.0f;
}

// The sphere and sky samplers of light_sample, out of line: most scenes have
// none of these lights, and the shade kernel is bound by instruction fetch.
__device__ __noinline__ LightSample light_sample_sphere_env(const SceneView& s, const Light& l, V3 p, V3 sn, int si,
                                                         Sampler& rng) {
    LightSample r;
    r.occluded = 0;
    r.has_ray = 0;
    r.color = v3(0.0f);
    r.dist = 0.0f;
    if (l.type == LIGHT_GEOM_SPHERE) {   // GeometryLight.ComputeSolidAngleSample (:202-238)
        int su = si % l.sqrt_samples, sv = si / l.sqrt_samples;
        float xi1 = ((float)su + rng.next()) * l.inv_sqrt;   // Sphere.SampleSolidAngleStratified
        float xi2 = ((float)sv + rng.next()) * l.inv_sqrt;
        V3 tc = l.center - p;
        float d2c = length_sq(tc);
        float r2 = l.radius * l.radius;
        V3 sp, ln;
        float pdf;
        if (d2c <= r2) {   // observer inside: uniform sphere (two more draws)
            V3 pu = random_unit_vector(rng);
            sp = l.center + pu * l.radius;
            ln = pu;
            pdf = 1.0f / (4.0f * kPi);
        } else {
            float dc = sqrtf(d2c);
            V3 wd = tc / dc;
            float cmax = sqrtf(fmaxf(0.0f, 1.0f - r2 / d2c));
            V3 dw = cone_dir(wd, cmax, xi1, xi2);
            V3 oc = p - l.center;
            float b = dot(oc, dw);
            float c = length_sq(oc) - r2;
            float disc = b * b - c;
            float t;
            if (disc <= 0.0f) {
                t = -b;   // tangent ray: the foot of the perpendicular
            } else {
                float sq = sqrtf(disc);
                t = -b - sq;
                if (t < kEps) t = -b + sq;
            }
            sp = p + t * dw;
            ln = normalize(sp - l.center);
            float sa = 2.0f * kPi * (1.0f - cmax);
            pdf = sa > kEps ? 1.0f / sa : 0.0f;
        }
        if (pdf <= 0.0f) {
            r.occluded = 1;
            r.dir = v3(0.0f, 1.0f, 0.0f);
            return r;
        }
        V3 tl = sp - p;
        float d2 = length_sq(tl);
        if (d2 < kEps * kEps) {
            r.occluded = 1;
            r.dir = v3(0.0f, 1.0f, 0.0f);
            return r;
        }
        float dist = sqrtf(d2);
        V3 dir = tl / dist;
        r.dir = dir;
        r.dist = dist;
        float cl = fmaxf(0.0f, dot(-dir, ln));
        if (cl <= 0.0f) return r;   // not in shadow, zero colour
        V3 so = offset_origin(p, sn);
        r.has_ray = 1;
        r.ray_o = so;
        r.ray_tmax = length(sp - so) - kEps;
        float atten = 1.0f / (pdf * (float)l.shadow_samples);
        r.color = l.emission * atten;
        return r;
    }
    if (l.type == LIGHT_SPHERE) {   // SphereLight.IlluminateAndTestStratified (:72-141)
        V3 tc = l.center - p;
        float d2c = length_sq(tc);
        if (d2c < kEps * kEps) {
            r.occluded = 1;
            r.dir = v3(0.0f, 1.0f, 0.0f);
            return r;
        }
        float dc = sqrtf(d2c);
        V3 wd = tc / dc;
        float s2 = l.radius * l.radius / d2c;
        float cmax = s2 >= 1.0f ? -1.0f : sqrtf(1.0f - s2);
        int su = si % l.sqrt_samples, sv = si / l.sqrt_samples;
        float xi1 = ((float)su + rng.next()) * l.inv_sqrt;
        float xi2 = ((float)sv + rng.next()) * l.inv_sqrt;
        V3 dw = cone_dir(wd, cmax, xi1, xi2);
        V3 oc = p - l.center;
        float b = dot(oc, dw);
        float c = length_sq(oc) - l.radius * l.radius;
        float disc = b * b - c;
        r.dir = dw;
        if (disc < 0.0f) {
            r.occluded = 1;
            r.dist = length(l.center + normalize(dw) * l.radius - p);
            return r;
        }
        float sq = sqrtf(disc);
        float t = -b - sq;
        if (t < kEps) t = -b + sq;
        if (t < kEps) {
            r.occluded = 1;
            return r;
        }
        V3 sp = p + t * dw;
        r.dist = t;
        V3 ln = (sp - l.center) / l.radius;
        float cl = fmaxf(0.0f, dot(-dw, ln));
        if (cl <= 0.0f) return r;   // not in shadow, zero colour
        V3 so = offset_origin(p, sn);
        r.has_ray = 1;
        r.ray_o = so;
        r.ray_tmax = length(sp - so) - kEps;
        float sa = 2.0f * kPi * (1.0f - cmax);
        float atten = l.intensity * sa / (float)l.shadow_samples;
        r.color = l.color * atten;
        return r;
    }
    if (l.type == LIGHT_ENV) {   // EnvironmentLight.IlluminateAndTest (:54-90) over FlatSky.ImportanceSample
        V3 dir = random_unit_vector(rng);
        const float pdf = 1.0f / (4.0f * kPi);
        r.dir = dir;
        r.dist = kInf;
        if (length_sq(sn) > 0.0f && dot(sn, dir) <= 0.0f) {   // below a surface's horizon
            r.occluded = 1;
            return r;
        }
        r.has_ray = 1;
        r.ray_o = offset_origin(p, sn);
        r.ray_tmax = kInf;
        r.color = l.color / (pdf * (float)l.shadow_samples);
        return r;
    }
    return r;   // not reached: the caller passes only these three types
}

// Draws the light sample (all RNG draws happen here, before any shadow test):
// GeometryLight.ComputeAreaSample (GeometryLight.cs:149-190),
// AreaLight.IlluminateAndTestStratified (AreaLight.cs:129-178),
// DirectionalLight.IlluminateAndTestStratified (DirectionalLight.cs:102-160).
RT_D LightSample light_sample(const SceneView& s, const Light& l, V3 p, V3 sn, int si, Sampler& rng) {
    LightSample r;
    r.occluded = 0;
    r.has_ray = 0;
    r.color = v3(0.0f);
    r.dist = 0.0f;
    if (l.type == LIGHT_GEOM_QUAD || l.type == LIGHT_GEOM_MESH) {
        V3 sp, ln;
        float area;
        if (l.type == LIGHT_GEOM_QUAD) {   // Quad.SampleStratified (Quad.cs:99-109)
            const QuadData& q = s.quads[RT_IX(l.quad, s.n_quads)];
            int su = si % l.sqrt_samples, sv = si / l.sqrt_samples;
            float inv = 1.0f / (float)l.sqrt_samples;
            float uu = ((float)su + rng.next()) * inv;
            float vv = ((float)sv + rng.next()) * inv;
            sp = q.q + uu * q.u + vv * q.v;
            ln = q.normal;
            area = q.area;
        } else {   // Mesh.SampleStratified (Mesh.cs:151-178) + Triangle.Sample
            int total = max(1, l.sqrt_samples * l.sqrt_samples);
            float stratum = 1.0f / (float)total;
            float jit = ((float)si + rng.next()) * stratum;
            float target = clampf(jit, 0.0f, 0.9999999f) * l.rep_area;
            int lo = 0, hi = l.mesh_count;   // lower_bound over the cumulative areas
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (s.light_tris[RT_IX(l.mesh_first + mid, s.n_light_tris)].cum_area < target) lo = mid + 1;
                else hi = mid;
            }
            int idx = min(max(lo, 0), l.mesh_count - 1);
            const LightTri& t = s.light_tris[RT_IX(l.mesh_first + idx, s.n_light_tris)];
            float x1 = rng.next();
            float x2 = rng.next();
            float r1 = sqrtf(x1);
            float u = 1.0f - r1;
            float v = x2 * r1;
            if (t.smooth >= 0) {   // SmoothTriangle.SampleAt (:219-230)
                const SmoothTri& st = s.smooth[RT_IX(t.smooth, s.n_smooth)];
                float w0 = 1.0f - u - v;
                sp = w0 * t.v0 + u * st.v1 + v * st.v2;
                ln = normalize(w0 * st.n0 + u * st.n1 + v * st.n2);
            } else {
                sp = t.v0 + u * t.e1 + v * t.e2;
                ln = t.normal;
            }
            area = l.rep_area;
        }
        V3 tl = sp - p;
        float d2 = length_sq(tl);
        if (d2 < kEps * kEps) {
            r.occluded = 1;
            r.dir = v3(0.0f, 1.0f, 0.0f);
            return r;
        }
        float dist = sqrtf(d2);
        V3 dir = tl / dist;
        r.dir = dir;
        r.dist = dist;
        float cl = fmaxf(0.0f, dot(-dir, ln));
        if (cl <= 0.0f) {
            r.occluded = 1;
            return r;
        }
        V3 so = offset_origin(p, sn);
        r.has_ray = 1;
        r.ray_o = so;
        r.ray_tmax = length(sp - so) - kEps;
        float atten = area * cl / (d2 * (float)l.shadow_samples);
        r.color = l.emission * atten;
        return r;
    }
    if (l.type == LIGHT_GEOM_SPHERE || l.type == LIGHT_SPHERE || l.type == LIGHT_ENV)
        return light_sample_sphere_env(s, l, p, sn, si, rng);
    if (l.type == LIGHT_AREA) {
        int su = si % l.sqrt_samples, sv = si / l.sqrt_samples;
        float ru = ((float)su + rng.next()) * l.inv_sqrt;
        float rv = ((float)sv + rng.next()) * l.inv_sqrt;
        V3 sp = l.corner + ru * l.u + rv * l.v;
        V3 tl = sp - p;
        float d2 = length_sq(tl);
        if (d2 < kEps * kEps) {
            r.occluded = 1;
            r.dir = v3(0.0f, 1.0f, 0.0f);
            return r;
        }
        float dist = sqrtf(d2);
        V3 dir = tl / dist;
        r.dir = dir;
        r.dist = dist;
        float cl = fmaxf(0.0f, dot(-dir, l.normal));
        if (cl <= 0.0f) return r;   // not in shadow, zero colour
        V3 so = offset_origin(p, sn);
        r.has_ray = 1;
        r.ray_o = so;
        r.ray_tmax = length(sp - so) - kEps;
        float ad2 = d2;
        if (l.soft_radius > 0.0f) ad2 = fmaxf(ad2, l.soft_radius * l.soft_radius);
        float atten = l.intensity * l.area * cl / (ad2 * (float)l.shadow_samples);
        r.color = l.color * atten;
        return r;
    }
    // Directional
    V3 tl;
    if (l.angular_radius > 0.0f) {
        int su = si % l.sqrt_samples, sv = si / l.sqrt_samples;
        float xi1 = ((float)su + rng.next()) * l.inv_sqrt;
        float xi2 = ((float)sv + rng.next()) * l.inv_sqrt;
        float ct = 1.0f - xi1 * (1.0f - l.cos_angular);
        float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        float phi = 2.0f * kPi * xi2;
        float sn2, cs2;
        sincosf(phi, &sn2, &cs2);
        V3 w = -l.direction;
        V3 loc = v3(st * cs2, st * sn2, ct);
        V3 uu, vv;
        tangent_frame(w, uu, vv);   // DirectionalLight.LocalToWorld (:192-213)
        V3 res = loc.x * uu + loc.y * vv + loc.z * w;
        float l2 = length_sq(res);
        tl = l2 > 1e-8f ? res / sqrtf(l2) : w;
    } else {
        tl = -l.direction;
    }
    r.dir = tl;
    r.dist = kInf;
    r.has_ray = 1;
    r.ray_o = offset_origin(p, sn);
    r.ray_tmax = kInf;
    float e = l.intensity / (float)l.shadow_samples;
    r.color = l.color * e;
    return r;
}

// GeometryLight.PdfSolidAngle for an emissive mesh: a ray cast against the
// emitter mesh alone (a whole BVH walk), out of line like the cold samplers.
__device__ __noinline__ float mesh_light_pdf(const SceneView& s, const Light& l, V3 p, V3 wi) {
    Hit h;
    int err = 0;
    traverse<false, 64>(s, p, wi, kEps, kInf, h, nullptr, &err, true, l.mesh_root);
    if (err || h.kind == HIT_NONE) return 0.0f;
    int ti = RT_IX(h.slot, s.n_tris);
    const float4* tp = s.tris + 3 * ti;
    V3 n = v3(ldg_scene(tp).w, ldg_scene(tp + 1).w, ldg_scene(tp + 2).w);
    int si = s.tri_smooth ? s.tri_smooth[ti] : -1;
    if (si >= 0) {   // the hit record's normal is the interpolated one
        const SmoothTri& st = s.smooth[RT_IX(si, s.n_smooth)];
        float w0 = 1.0f - h.u - h.v;
        n = normalize(w0 * st.n0 + h.u * st.n1 + h.v * st.n2);
    }
    float cl = fabsf(dot(-wi, n));
    if (cl < 1e-6f) return 0.0f;
    float d2 = h.t * h.t;
    if (l.rep_area < 1e-12f) return 0.0f;
    return d2 / (l.rep_area * cl);
}

// ILight.PdfSolidAngle (GeometryLight.cs:254-279, AreaLight.cs:189-226,
// DirectionalLight.cs:169-181).
RT_D float light_pdf(const SceneView& s, const Light& l, V3 p, V3 wi) {
    if (l.type == LIGHT_GEOM_QUAD) {
        const QuadData& q = s.quads[RT_IX(l.quad, s.n_quads)];
        float t, a, b;
        if (!quad_test(q, p, wi, kEps, kInf, false, t, a, b)) return 0.0f;
        float cl = fabsf(dot(-wi, q.normal));   // |.| makes the face flip irrelevant
        if (cl < 1e-6f) return 0.0f;
        float d2 = t * t;
        if (l.rep_area < 1e-12f) return 0.0f;
        return d2 / (l.rep_area * cl);
    }
    if (l.type == LIGHT_GEOM_SPHERE || l.type == LIGHT_SPHERE) return sphere_cone_pdf(l.center, l.radius, p, wi);
    if (l.type == LIGHT_ENV) return 1.0f / (4.0f * kPi);   // FlatSky.Pdf
    if (l.type == LIGHT_GEOM_MESH) return mesh_light_pdf(s, l, p, wi);
    if (l.type == LIGHT_AREA) {
        float denom = dot(l.normal, wi);
        if (fabsf(denom) < 1e-7f) return 0.0f;
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
        float cl = fabsf(denom);
        if (cl < 1e-6f) return 0.0f;
        return (t * t) / (l.area * cl);
    }
    if (l.angular_radius <= 0.0f || l.solid_angle <= 0.0f) return 0.0f;
    float wl = length(wi);
    if (wl < kEps) return 0.0f;
    float ct = dot(wi / wl, -l.direction);
    if (ct < l.cos_angular) return 0.0f;
    return 1.0f / l.solid_angle;
}

RT_D float mis_weight(float p, float q, int power) {   // Renderer.cs:1534-1543
    if (power) {
        float p2 = p * p, q2 = q * q;
        return p2 / (p2 + q2 + 1e-30f);
    }
    return p / (p + q + 1e-30f);
}

// Geometry/ShadowRay.cs:59-157. Opaque scenes take the any-hit fast path: with
// no transmissive material the walk returns 0 at the first hit, so "any hit in
// [tmin, tmax]" decides it exactly.
template <int STACK, bool L4 = false>
__device__ __forceinline__ V3 shadow_transmittance(const SceneView& s, int opaque_scene, V3 o, V3 d, float tmin,
                                                   float tmax, Counters* cnt, int* err) {
    Hit h;
    TravCounters* tc = cnt ? &cnt->shadow : nullptr;
    if (cnt) cnt->shadow_rays++;
    if (opaque_scene && !cnt) {   // the counting build walks like ShadowRay.Transmittance
        trace<true, STACK, L4>(s, o, d, tmin, tmax, h, tc, err);
        return h.kind == HIT_NONE ? v3(1.0f) : v3(0.0f);
    }
    V3 thr = v3(1.0f);
    float remaining = tmax;
    V3 sigma = v3(0.0f), entry = v3(0.0f);
    bool in_med = false;
    for (int i = 0; i < 8; i++) {
        trace<false, STACK, L4>(s, o, d, tmin, remaining, h, tc, err);
        if (h.kind == HIT_NONE) return thr;
        Surface rec = make_surface(s, h, o, d);
        const Material& m = s.materials[rec.material];
        if (in_med) {
            float dd = length(rec.p - entry);
            thr = v3(thr.x * expf(-sigma.x * dd), thr.y * expf(-sigma.y * dd), thr.z * expf(-sigma.z * dd));
            in_med = false;
            if (near_zero(thr)) return v3(0.0f);
        }
        V3 t = bsdf_shadow_transmittance(m, d, rec);
        if (near_zero(t)) return v3(0.0f);
        thr = thr * t;
        if (near_zero(thr)) return v3(0.0f);
        if (rec.front && m.type == 0) {
            V3 sg = m.trans_sigma;
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
// Homogeneous medium + Henyey-Greenstein (Volumetrics/HomogeneousMedium.cs,
// Volumetrics/HenyeyGreensteinPhase.cs)
// ---------------------------------------------------------------------------
RT_D V3 medium_tr(const SceneView& s, float t) {
    float d = fminf(fmaxf(t, 0.0f), 1e30f);
    return v3(expf(-s.sigma_t.x * d), expf(-s.sigma_t.y * d), expf(-s.sigma_t.z * d));
}
RT_D float hg_eval(float g, V3 wo, V3 wi) {
    float mu = dot(wo, wi);
    float den = 1.0f + g * g - 2.0f * g * mu;
    return kInv4Pi * (1.0f - g * g) / (den * sqrtf(den));
}
RT_D V3 hg_sample(float g, V3 wo, Sampler& rng, float& pdf) {
    float u1 = rng.next(), u2 = rng.next();
    float ct;
    if (fabsf(g) < 1e-3f) {
        ct = 1.0f - 2.0f * u1;
    } else {
        float sqr = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
        ct = (1.0f + g * g - sqr * sqr) / (2.0f * g);
    }
    float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float phi = 2.0f * kPi * u2;
    float sn, cs;
    sincosf(phi, &sn, &cs);
    V3 w = wo;
    V3 a = fabsf(w.x) > 0.9f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    V3 v = normalize(cross(w, a));
    V3 u = cross(w, v);
    V3 wi = st * cs * u + st * sn * v + ct * w;
    wi = normalize(wi);
    pdf = hg_eval(g, wo, wi);
    return wi;
}
RT_D bool medium_sample(const SceneView& s, float tmax, Sampler& rng, float& t, V3& beta) {
    int ch = (int)(rng.next() * 3.0f);
    if (ch > 2) ch = 2;
    float st = ch == 0 ? s.sigma_t.x : (ch == 1 ? s.sigma_t.y : s.sigma_t.z);
    if (st <= 0.0f) {
        t = tmax;
        beta = v3(1.0f);
        return false;
    }
    float dist = -logf(1.0f - rng.next()) / st;
    bool sc = dist < tmax;
    t = sc ? dist : tmax;
    V3 tr = medium_tr(s, t);
    V3 dens = sc ? s.sigma_t * tr : tr;
    float pdf = (dens.x + dens.y + dens.z) / 3.0f;
    if (pdf < 1e-20f) pdf = 1.0f;
    beta = sc ? (tr * s.sigma_s / pdf) : (tr / pdf);
    return sc;
}

RT_D V3 sanitize(V3 c) {   // Renderer.cs:917-923
    if (!isfinite(c.x)) c.x = 0.0f;
    if (!isfinite(c.y)) c.y = 0.0f;
    if (!isfinite(c.z)) c.z = 0.0f;
    return vmax(c, v3(0.0f));
}
RT_D V3 clamp_lum(V3 c, float mx) {   // ClampRadiance / ClampRadianceIndirect (:931-972)
    c = sanitize(c);
    float lum = luminance(c);
    if (lum > mx && lum > 0.0f) c = c * (mx / lum);
    return c;
}
RT_D V3 beer_lambert(V3 rad, V3 sigma, float t) {   // Renderer.cs:1791-1800
    if (sigma.x <= 0.0f && sigma.y <= 0.0f && sigma.z <= 0.0f) return rad;
    if (isinf(t) && t > 0.0f) return v3(0.0f);
    if (t <= 0.0f) return rad;
    return rad * v3(sigma.x > 0.0f ? expf(-sigma.x * t) : 1.0f, sigma.y > 0.0f ? expf(-sigma.y * t) : 1.0f,
                    sigma.z > 0.0f ? expf(-sigma.z * t) : 1.0f);
}

}  // namespace rt
