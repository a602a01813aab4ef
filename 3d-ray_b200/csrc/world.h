// Host-side world assembly: what 3d-ray's .NET host does before the bounce
// loop (SceneLoader world assembly + the binned-SAH build), producing the
// flattened SoA the kernels read. Without .NET in this environment the SAH
// build is restated here in C++ (Acceleration/BvhNode.cs:91-364); a .NET host
// would instead read its own BvhNode tree out into the same arrays.
#pragma once

#include <string>
#include <vector>

#include "../../include/rt3d.h"
#include "scene_types.h"

namespace rt {

struct HostScene {
    std::vector<NodeF> nodes;      // build layout (pre-order), kept for export and tests
    std::vector<float4> cnodes;    // traversal layout: 4 float4 per interior node
    std::vector<float4> cnodes4;   // four-wide traversal layout: 8 float4 per record
    std::vector<int> mesh_root4;   // per entity: mesh root code in cnodes4 (else 0)
    int top_root4 = 0;             // four-wide code of the top-level root (top_is_bvh only)
    int max_stack4 = 0;            // worst-case traversal stack in the four-wide layout
    std::vector<int> top_items;
    std::vector<float4> tris;      // 3 per triangle
    std::vector<int> tri_entity;
    std::vector<int> tri_local;
    std::vector<Entity> entities;
    std::vector<float4> ent_box;   // 2 per entity
    std::vector<QuadData> quads;
    std::vector<SphereData> spheres;
    std::vector<Material> materials;
    std::vector<Light> lights;
    std::vector<LightTri> light_tris;
    std::vector<SmoothTri> smooth;
    std::vector<int> tri_smooth;   // per triangle (traversal order); empty when no triangle is smooth
    std::vector<int> emitter_light;
    std::vector<float> pick_cdf, pick_pdf;   // LightDistribution: power, then uniform (2 * lights each)
    std::vector<float> lut_e, lut_eavg;
    RtCameraDesc camera{};
    int top_root = -1;             // build layout
    int top_root_code = 0;         // traversal layout (top_is_bvh only)
    int top_is_bvh = 0;
    int max_stack = 0;
    int rr_min_bounces = 3;
    float rr_min_survival = 0.1f;
    float mean_irradiance = 0.0f;
    int has_medium = 0;
    V3 sigma_a{}, sigma_s{}, sigma_t{};
    float hg_g = 0.0f;
    V3 sky{};
    int sky_on = 0;
    int env_light = -1;
    int bvh_on_device = 0;         // the mesh BVHs came from the device build
    double bvh_build_ms = 0.0;     // wall time of the mesh-BVH phase
};

// One mesh's BVH in the build layout (pre-order, node indices local to the
// mesh, leaf `first` an offset into `order`), as BvhNode's constructor makes
// it for a mesh of more than 4 triangles (Geometry/Mesh.cs:93-96).
struct MeshBvh {
    std::vector<NodeF> nodes;
    std::vector<int> order;        // mesh-local triangle ids in leaf order
    V3 box_mn{}, box_mx{};
    int max_depth = 0;             // interior nodes on the longest root-leaf path
};

// Builds the BVHs of `n` meshes whose triangles are tri_verts[first[i]*9 ...]
// (count[i] > 4 each), exactly as the host build does. Returns RT_OK, or an
// error code with a message; build_world then builds those meshes on the host.
using MeshBvhBuilder = int (*)(const float* tri_verts, const int64_t* first, const int64_t* count, int n,
                               MeshBvh* out, std::string& err);

// The device build (bvh_build.cu): a MeshBvhBuilder on the current device.
int device_build_meshes(const float* tri_verts, const int64_t* first, const int64_t* count, int n, MeshBvh* out,
                        std::string& err);

// Where build_world builds the mesh BVHs.
struct BuildOptions {
    MeshBvhBuilder device_builder = nullptr;   // null: host threads
    int64_t device_min_tris = 0;               // use the device when the meshes hold at least this many
};

// Returns RT_OK or an RT_ERR_* code with a message in err.
int build_world(const RtWorldDesc* w, HostScene& out, std::string& err, const BuildOptions& opt = BuildOptions{});

// Kulla-Conty E(mu, alpha) / E_avg(alpha) tables
// (Materials/EnergyCompensationLut.cs:48-74), built with the host libm.
void build_energy_lut(float* e1024, float* eavg32);

// Pinhole camera basis (Camera/Camera.cs:26-51) for the given aspect ratio.
Camera make_camera(const RtCameraDesc& c, float aspect);

// Material constants (DisneyBsdf.cs:213-293, 1104-1139, 1943-1959, 1016-1049).
Material make_material(const RtMaterialDesc& d, const float* lut_eavg);

}  // namespace rt
