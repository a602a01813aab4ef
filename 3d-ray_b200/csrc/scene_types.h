// Flattened scene layout in HBM, shared by the host builder and the kernels.
//
// BVH nodes (32 B, two 16-byte loads):
//   lo = (bmin.x, bmin.y, bmin.z, a)   hi = (bmax.x, bmax.y, bmax.z, b)
//   interior : a >= 0 is the left child, b = right child | axis << 30
//   leaf     : a = ~first, b = count | kind << 16
//              kind LEAF_TRIS  -> triangles [first, first+count) of the triangle SoA
//              kind LEAF_ENTS  -> entity ids top_items[first .. first+count)
//              kind LEAF_LIST  -> a mesh of <= 4 triangles held in a flat list:
//                                 no box test (Geometry/Mesh.cs:93-96)
// Nodes of the top-level tree and of every mesh BVH share one array, each
// tree laid out in depth-first pre-order (a parent precedes its left subtree).
//
// Triangles (48 B, three 16-byte loads): (v0, n.x) (e1, n.y) (e2, n.z) with
// e1 = v1 - v0, e2 = v2 - v0 and n the unit geometric normal, exactly as
// Geometry/Triangle.cs:35-47 precomputes them; tri_entity / tri_local map a
// stored triangle back to its entity and its index in the source mesh.
#pragma once

#include <stdint.h>
#include <vector_types.h>

#include "vec.cuh"

namespace rt {

enum : int { LEAF_TRIS = 0, LEAF_ENTS = 1, LEAF_LIST = 2, LEAF_ENT1 = 3 };

// Traversal layout (what the kernels read): one 64-byte record per interior
// node holding both children's boxes, so a single fetch tests two boxes.
//   (lmin.xyz, lcode) (lmax.xyz, rcode) (rmin.xyz, axis) (rmax.xyz, -)
// A child code >= 0 is an interior record index; a negative code is a leaf:
//   ~code = first << 5 | kind << 3 | (count - 1)
// kind LEAF_TRIS / LEAF_LIST: triangles [first, first+count); LEAF_ENTS:
// entity ids top_items[first .. first+count); LEAF_ENT1: the single entity
// `first` (traversal-stack entries for pending top-level leaf items).
RT_HD int leaf_code(int first, int kind, int count) { return ~((first << 5) | (kind << 3) | (count - 1)); }
enum : int { ENT_QUAD = 0, ENT_SPHERE = 1, ENT_MESH = 2 };
enum : int { ENT_BACKFACE_CULLED = 1 };

struct alignas(16) NodeF {
    float lo[4];
    float hi[4];
};

struct Entity {
    int kind;
    int material;
    int flags;
    int index;   // quad / sphere index, or the mesh root child code
};

struct QuadData {   // Geometry/Quad.cs:26-40 precomputed constants
    V3 q, u, v, normal, w, tangent, bitangent;
    float d, area;
};

struct SphereData {
    V3 c;
    float r;
};

// Disney material with every per-shading-point constant precomputed once on
// the host (constant textures make ShadingParams, the lobe probabilities and
// F0 per-material constants; DisneyBsdf.cs:213-293, 1104-1139, 1943-1959).
struct Material {
    int type;          // RT_MAT_DISNEY / RT_MAT_EMISSIVE
    int thin_walled;
    int has_tc;
    int has_rotation;
    V3 base;           // baseColor (Disney) or colour (Emissive)
    V3 emission;       // Emissive: colour * intensity
    float metallic, roughness, specular, specular_tint, sheen, sheen_tint, sheen_roughness;
    float clearcoat, clearcoat_gloss, spec_trans, ior, anisotropic, aniso_rotation, diff_trans;
    float alpha, alpha_x, alpha_y, cc_alpha, cc_f0;
    float rot_cos, rot_sin;            // cos/sin(2*pi*rotation)
    float spec_trans_raw, ior_raw;     // unclamped texture values (ShadowTransmittance)
    V3 f0;                             // ComputeF0
    V3 sheen_col;                      // lerp(1, tint, sheenTint)
    V3 trans_tint, trans_sigma;        // ResolveTransmission
    float p_d, p_s, p_t, p_sh, p_ms, p_dt, p_c;   // lobe selection probabilities
    float diffuse_w;                   // (1-metallic)(1-specTrans)(1-diffTrans)
    float diff_all;                    // (1-metallic)(1-specTrans)
    float alpha_iso, e_avg;            // sqrt(ax*ay), E_avg(alpha_iso)
};

enum : int {
    LIGHT_GEOM_QUAD = 0,
    LIGHT_GEOM_MESH = 1,
    LIGHT_GEOM_SPHERE = 2,   // an emissive sphere: GeometryLight with cone sampling
    LIGHT_AREA = 3,
    LIGHT_DIRECTIONAL = 4,
    LIGHT_SPHERE = 5,        // SphereLight
    LIGHT_ENV = 6,           // EnvironmentLight over a flat sky
};

struct Light {
    int type;
    int shadow_samples;
    int sqrt_samples;
    int is_delta;
    int emissive_material;
    int quad;            // geometry-quad light: quad index
    int mesh_first;      // geometry-mesh light: first triangle in light_tris (source order)
    int mesh_count;
    int mesh_root;       // mesh BVH root child code (PdfSolidAngle ray cast)
    int mesh_entity;
    float inv_sqrt;
    float rep_area;      // ISamplable.SurfaceArea
    V3 emission;         // GeometryLight: Emissive colour * intensity
    V3 corner, u, v, color, normal;
    float intensity, area, soft_radius;
    V3 direction;
    float angular_radius, cos_angular, solid_angle;
    V3 center;           // sphere lights (geometry or SphereLight)
    float radius;
};

// Emissive-mesh triangles in source order with the area CDF (Mesh.cs:98-107).
struct LightTri {
    V3 v0, e1, e2, normal;
    float cum_area;
    int smooth;   // index into SceneView::smooth, or -1 (flat)
};

// Shading data of a smooth triangle (Geometry/SmoothTriangle.cs:67-138): the
// normalised vertex normals, the UV-gradient tangent frame, the vertex UVs and
// the original v1, v2 (SampleAt weights the vertices themselves, not v0 plus
// the edges).
struct SmoothTri {
    V3 n0, n1, n2;
    V3 tangent, bitangent;
    V3 v1, v2;
    float uv[6];
};

struct Camera {
    V3 origin, llc, horizontal, vertical;
};

// Four-wide traversal layout: one 128-byte record per node of the binary tree
// at even depth, holding the boxes of its (up to) four grandchildren
// {LL, LR, RL, RR} as SoA float4s and their codes:
//   q[0..2] lo.x/y/z of the four slots, q[3..5] hi.x/y/z, q[6] child codes,
//   q[7] (axis of the node, axis of L, axis of R, -).
// A slot whose binary child is a leaf holds that leaf in its first position
// (LL or RL) and an empty box in the second. A code >= 0 is another record;
// a leaf code as in the two-wide layout; an empty slot is INT_MIN.
// The three axes give the binary tree's visit order for a ray, so the
// traversal tests the same primitives in the same order as the two-wide one.
struct SceneView {
    const float4* cnodes;       // 4 float4 per interior node (child-box layout)
    const float4* cnodes4;      // 8 float4 per four-wide record
    const int* mesh_root4;      // per entity: a mesh's root code in cnodes4
    const int* top_items;
    const float4* tris;
    const int* tri_entity;
    const int* tri_local;
    const Entity* entities;
    const float4* ent_box;      // 2 per entity: the entity's AABB (a mesh's root box)
    const QuadData* quads;
    const SphereData* spheres;
    const Material* materials;
    const Light* lights;
    const LightTri* light_tris;
    const SmoothTri* smooth;
    const int* tri_smooth;      // per triangle: index into smooth or -1; null when no triangle is smooth
    const int* emitter_light;   // material -> light index or -1
    const float* pick_cdf;      // 2 * num_lights: the power then the uniform LightDistribution CDF
    const float* pick_pdf;      // 2 * num_lights: their pdfs
    const float* lut_e;         // 32 x 32, mu-major
    const float* lut_eavg;      // 32
    int num_lights;
    int top_is_bvh;             // 0: the world is a flat list of top_items
    int top_root;               // child code of the top-level root (top_is_bvh only)
    int top_root4;              // the same in the four-wide layout
    int num_top_items;          // flat list: entity count
    int has_medium;
    V3 sigma_a, sigma_s, sigma_t;
    float hg_g;
    V3 sky;                     // flat sky radiance (black: no sky term)
    int sky_on;                 // sky is not black
    int env_light;              // index of the EnvironmentLight, or -1
    // Box of the wavefront's bounce-ray sort: origins map to cells of
    // (o - sort_lo) * sort_scale in [0, 1) (clamped); sort_scale 0 on a flat axis.
    V3 sort_lo, sort_scale;
    // Lengths of the arrays above, in elements; the checked build tests every
    // index into them.
    int n_cnodes, n_cnodes4, n_tris, n_entities, n_quads, n_spheres, n_materials, n_light_tris, n_smooth;
};

}  // namespace rt
