/*
 * rt3d.h — C-ABI of the B200 path-tracing core for 3d-ray.
 *
 * The library replaces 3d-ray's per-pixel bounce loop (Sobol camera rays,
 * closest-hit and shadow traversal of the host-built SAH BVH, Disney BSDF,
 * NEE with MIS and Russian roulette, HDR film accumulation). Everything above
 * that loop — YAML scene loading, the camera description, the CLI and the
 * `Renderer` API — stays in the host. All entry points take plain pointers and
 * sizes; no torch or .NET types cross this boundary.
 *
 * Conventions
 *   - Every function returns 0 (RT_OK) or a negative RT_ERR_* code and never
 *     aborts or traps. rt_last_error() returns a thread-local message.
 *   - The caller owns every host pointer for the duration of a call; nothing
 *     is retained after return. The library owns device memory behind the
 *     opaque RtScene handle.
 *   - Calls on one RtScene are serialised internally (one CUDA stream per
 *     scene); distinct scenes may be used from different host threads.
 *   - Films are planar linear-HDR fp32, channel-major: value (c, x, y) lives
 *     at out[c*W*H + y*W + x], the layout of 3d-ray's FrameBuffer
 *     (src/RayTracer/Rendering/FrameBuffer.cs:38).
 *
 * Reference seams (file:line in fiorenzobrioni/3d-ray):
 *   rt_scene_build / rt_scene_create : SceneLoader.Load world assembly
 *       (src/RayTracer/Scene/SceneLoader.cs:446-485, 805-887) and the SAH
 *       build (src/RayTracer/Acceleration/BvhNode.cs:91-153)
 *   rt_render          : Renderer.Render (src/RayTracer/Rendering/Renderer.cs:522-733)
 *   rt_render_batch    : N independent Renderer.Render calls in one launch
 *   rt_adjoint         : no counterpart (gradient of an image loss w.r.t.
 *                        Disney parameters and emitter radiance)
 *   rt_trace_closest   : IHittable.Hit on the world (Renderer.cs:1624-1647,
 *                        HittableList.cs:19-37, BvhNode.cs:157-206)
 *   rt_trace_any       : ShadowRay.Transmittance (Geometry/ShadowRay.cs:59-157)
 *   rt_bsdf_batch      : DisneyBsdf.Sample/Evaluate/Pdf/EvaluateDirect
 *                        (Materials/DisneyBsdf.cs:418-997)
 *   rt_medium_batch    : HomogeneousMedium.Sample/Transmittance and
 *                        HenyeyGreensteinPhase.Sample/Evaluate
 *                        (Volumetrics/HomogeneousMedium.cs:36-76,
 *                        Volumetrics/HenyeyGreensteinPhase.cs:23-54)
 *   rt_sobol_batch     : OwenSobol.Sample (Core/Sampling/OwenSobol.cs:48-89)
 *   rt_tonemap         : Renderer.AcesToneMap (Rendering/Renderer.cs:893-907)
 */
#ifndef RT3D_H
#define RT3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RT3D_ABI_VERSION 2   /* 2: RtRenderParams gained the two test-only limits */

/* ---- status codes -------------------------------------------------------- */
#define RT_OK                  0
#define RT_ERR_INVALID_ARG    -1   /* null pointer, bad size, bad enum */
#define RT_ERR_OOM            -2   /* device or host allocation failed */
#define RT_ERR_CUDA           -3   /* a CUDA runtime call failed */
#define RT_ERR_TIMEOUT        -4   /* a bounded device wait expired */
#define RT_ERR_BOUNDS         -5   /* a checked kernel saw an out-of-range index */
#define RT_ERR_UNSUPPORTED    -6   /* scene feature outside the GPU path */
#define RT_ERR_STACK          -7   /* traversal stack bound exceeded */
#define RT_ERR_NO_DEVICE      -8   /* no CUDA device / extension not usable */

/* ---- scene description (what the host's loader produces) ---------------- */

/* Material kinds (IMaterial implementations on the path). */
#define RT_MAT_DISNEY   0   /* Materials/DisneyBsdf.cs */
#define RT_MAT_EMISSIVE 1   /* Materials/Emissive.cs   */

/* One material with constant parameters. Field meanings and defaults follow
 * the DisneyBsdf constructor (Materials/DisneyBsdf.cs:172-215) and the
 * Emissive constructor (Materials/Emissive.cs:43-53). */
typedef struct RtMaterialDesc {
    int32_t type;                 /* RT_MAT_* */
    int32_t is_light_proxy;       /* Emissive backing an area light's proxy quad */
    int32_t thin_walled;          /* DisneyBsdf.ThinWalled */
    int32_t has_transmission_color;
    float base_color[3];          /* Disney baseColor, or Emissive colour */
    float intensity;              /* Emissive intensity (clamped >= 0 by the library) */
    float metallic, roughness, specular, specular_tint;
    float sheen, sheen_tint, sheen_roughness;
    float clearcoat, clearcoat_gloss;
    float spec_trans, ior;
    float anisotropic, anisotropic_rotation;
    float diff_trans;
    float coat_ior, coat_roughness;   /* coat_roughness < 0 selects the clearcoat_gloss path */
    float thin_film_thickness, thin_film_ior;
    float transmission_color[3];
    float transmission_depth;
} RtMaterialDesc;

/* Entity kinds (IHittable leaves the world list holds). */
#define RT_ENT_QUAD   0   /* Geometry/Quad.cs          p[0..2]=Q, p[3..5]=U, p[6..8]=V */
#define RT_ENT_SPHERE 1   /* Geometry/Sphere.cs        p[0..2]=centre, p[3]=radius     */
#define RT_ENT_MESH   2   /* Geometry/Mesh.cs of flat Geometry/Triangle.cs,
                             triangles [first, first+count) of tri_verts          */

#define RT_ENT_FLAG_BACKFACE_CULLED 1  /* Geometry/BackFaceCulledHittable.cs wrapper */

typedef struct RtEntityDesc {
    int32_t kind;
    int32_t material;
    int32_t flags;
    int32_t pad;
    int64_t first;
    int64_t count;
    float p[12];
} RtEntityDesc;

#define RT_LIGHT_AREA        0   /* Lights/AreaLight.cs        */
#define RT_LIGHT_DIRECTIONAL 1   /* Lights/DirectionalLight.cs */
#define RT_LIGHT_SPHERE      2   /* Lights/SphereLight.cs      */

/* Explicit lights in YAML order. Geometry lights (Lights/GeometryLight.cs) are
 * derived by the library from emissive, non-proxy entities in entity order and
 * appended after these, as SceneLoader.ExtractGeometryLights does
 * (Scene/SceneLoader.cs:516-522). */
typedef struct RtLightDesc {
    int32_t type;
    int32_t shadow_samples;       /* <= 0: the light type's default */
    int32_t proxy_material;       /* area / sphere light: material index of its proxy, or -1 */
    int32_t pad;
    float corner[3], u[3], v[3];  /* area light parallelogram */
    float color[3];
    float intensity;
    float soft_radius;
    float direction[3];           /* directional light travel direction */
    float angular_radius_deg;     /* directional disc; 0 = delta light */
    float center[3];              /* sphere light */
    float radius;
} RtLightDesc;

/* Camera/Camera.cs:26-51 (pinhole when aperture == 0). */
typedef struct RtCameraDesc {
    float look_from[3], look_at[3], vup[3];
    float vfov_deg;
    float aperture;
    float focus_dist;
} RtCameraDesc;

/* Global homogeneous medium (Volumetrics/HomogeneousMedium.cs) with a
 * Henyey-Greenstein phase (Volumetrics/HenyeyGreensteinPhase.cs). */
typedef struct RtMediumDesc {
    int32_t enabled;
    int32_t pad;
    float sigma_a[3];
    float sigma_s[3];
    float g;
} RtMediumDesc;

typedef struct RtWorldDesc {
    const RtMaterialDesc* materials;  int32_t num_materials;
    const RtEntityDesc*   entities;   int32_t num_entities;
    const float*          tri_verts;  int64_t num_tris;   /* 9 floats: v0, v1, v2 */
    const RtLightDesc*    lights;     int32_t num_lights;
    int32_t geometry_light_samples;   /* ShadowSamples of derived geometry lights */
    RtCameraDesc camera;
    RtMediumDesc medium;
    /* Smooth triangles (Geometry/SmoothTriangle.cs, what ObjLoader.cs:355-395
     * builds for faces with vertex normals): null, or 9 floats per triangle,
     * the vertex normals n0, n1, n2 (normalised on load). All nine zero marks
     * a flat Triangle. */
    const float*          tri_normals;
    /* null, or 6 floats per triangle: uv0, uv1, uv2 of a smooth triangle, for
     * its UV-gradient tangent frame (null: (0,0), (1,0), (0,1)). */
    const float*          tri_uvs;
    /* Flat sky colour (Rendering/Sky/FlatSky.cs): the radiance of every ray
     * that leaves the scene. Unless it is black (luminance <= 1e-6) the
     * library appends an EnvironmentLight after the geometry lights, as
     * SceneLoader does (:524-528). */
    float                 sky_color[3];
    int32_t               sky_light_samples;  /* its ShadowSamples (the -S override, else 1); <= 0: 1 */
} RtWorldDesc;

/* ---- render parameters: the Renderer constructor (Renderer.cs:300-319) --- */

#define RT_MIS_BALANCE 0
#define RT_MIS_POWER   1
#define RT_LIGHTS_ALL     0   /* every light, every shadow sample */
#define RT_LIGHTS_POWER   1   /* one light per vertex, picked by ApproximatePower (LightDistribution.cs) */
#define RT_LIGHTS_UNIFORM 2   /* one light per vertex, picked uniformly */

#define RT_KERNEL_MEGAKERNEL 0   /* one thread per sample, whole path in registers */
#define RT_KERNEL_WAVEFRONT  1   /* raygen/extend/shade/occlude/resolve queues     */

typedef struct RtRenderParams {
    int32_t width, height;
    int32_t spp;
    int32_t max_depth;
    int32_t spp_offset;             /* first Sobol sample index (progressive resume) */
    int32_t rr_min_bounces;         /* < 0: the reference's scene classifier decides */
    float   rr_min_survival;        /* used only when rr_min_bounces >= 0 */
    float   max_sample_radiance;    /* <= 0: default 10 (Renderer.cs:202) */
    float   indirect_clamp_factor;  /* < 0: default 0.25 (Renderer.cs:214) */
    float   exposure_ev;
    int32_t mis_heuristic;          /* RT_MIS_* */
    int32_t light_strategy;         /* RT_LIGHTS_* (LightSamplingStrategy) */
    int32_t kernel;                 /* RT_KERNEL_* */
    int32_t block_size;             /* wavefront: 64, 128 or 256; 0: autotuned / default */
    int32_t wavefront_size;         /* wavefront: path slots; 0: autotuned / default */
    int32_t sort_materials;         /* wavefront: 1 sort hits by material, 0 no, -1 autotuned / default */
    int32_t pixel_x0, pixel_y0;     /* render window (0,0,0,0 = full frame) */
    int32_t window_w, window_h;
    int32_t count_work;             /* 1: counting build, fills the work fields of RtStats */
    int32_t profile_kernels;        /* 1: wavefront without the graph, per-kernel events in RtStats */
    int32_t node_layout;            /* BVH records the wavefront's extend/occlude read: 2 two-wide,
                                       4 four-wide, 0 the autotuned choice (else two-wide) */
    int32_t ray_fetch;              /* wavefront extend/occlude on two-wide records: 1 one ray per
                                       thread, 2 persistent warps refilling finished lanes from a
                                       global counter, 0 the autotuned choice (else 1) */
    int32_t trace_block_size;       /* block of the wavefront's extend/occlude: 64, 128 or 256;
                                       0 the autotuned choice (else block_size) */
    int32_t ray_groups;             /* wavefront extend/occlude on one ray per thread: 1 rays in slot
                                       order, 2 each block regroups its rays by kind (camera rays,
                                       then bounce and shadow rays by direction octant), 3 extend
                                       walks the bounce rays sorted by origin cell and direction,
                                       then the camera rays in pixel order, 4 as 3 and occlude walks
                                       the shadow rays sorted the same way; 0 the autotuned choice
                                       (else 4, or 1 when a scene has a participating medium) */
    /* Test-only limits of the wavefront, for exercising its failure paths.
     * Both are 0 in production: the host then sizes the queue and bounds the
     * iterations itself, and neither limit is ever reached. */
    int32_t iteration_limit;        /* > 0: the wavefront gives up after this many iterations and
                                       returns RT_ERR_TIMEOUT (the host-side bound on its poll loop) */
    int32_t shadow_queue_limit;     /* > 0: the shadow queue holds at most this many records; a fuller
                                       queue is refused by the kernel and the call returns RT_ERR_BOUNDS */
} RtRenderParams;

/* Counters and timings of one call. */
typedef struct RtStats {
    double   kernel_ms;             /* device time of the render kernels (CUDA events) */
    double   total_ms;              /* host wall time of the call */
    uint64_t samples;               /* camera samples traced */
    uint64_t closest_rays;          /* closest-hit rays (count_work only) */
    uint64_t shadow_rays;           /* any-hit rays (count_work only) */
    uint64_t node_visits;           /* BVH node box tests of closest rays (count_work only) */
    uint64_t prim_tests;            /* triangle tests of closest rays (count_work only) */
    uint64_t other_tests;           /* quad / sphere tests of closest rays (count_work only) */
    uint64_t shadow_node_visits;    /* the same three for shadow rays (count_work only) */
    uint64_t shadow_prim_tests;
    uint64_t shadow_other_tests;
    double   regen_ms, extend_ms, shade_ms, occlude_ms, sort_ms;   /* profile_kernels only; sort_ms holds
                                       the material sort and the ray sorts' scans and scatter */
    int32_t  iterations;            /* wavefront iterations */
    int32_t  kernel_launches;       /* kernels launched by the call */
    int32_t  rr_min_bounces;        /* the RR knobs the call used */
    float    rr_min_survival;
} RtStats;

typedef struct RtScene RtScene;

/* ---- version / errors ---------------------------------------------------- */
int         rt_abi_version(void);
/* 1 in the checked build (librt3d_checked.so), 0 in the product build. The
 * checked build tests every index its kernels take from scene data or from
 * the wavefront's queues against the array's length; an index out of range is
 * replaced by 0 (no trap) and the call returns RT_ERR_BOUNDS. It is a
 * diagnostic build for the test suite: its flag is one word per device,
 * shared by all scenes, so concurrent calls may report each other's error. */
int         rt_checked_build(void);
const char* rt_last_error(void);
/* Number of visible CUDA devices; < 0 on error. Loads no kernels. */
int         rt_device_count(void);

/* ---- scene lifetime ------------------------------------------------------ */
/* Runs the world assembly (SAH BVH build, flattening into SoA, geometry-light
 * extraction, Kulla-Conty LUT build) and uploads the result to the current
 * device. The mesh BVHs are built as by rt_scene_create_ex with RT_BVH_AUTO. */
int rt_scene_create(const RtWorldDesc* world, RtScene** out_scene);
int rt_scene_destroy(RtScene* scene);

/* Where the mesh BVHs (BvhNode's constructor for every mesh of more than 4
 * triangles, Geometry/Mesh.cs:93-96) are built. Both builds give the same
 * nodes, boxes and leaf order, bit for bit. */
#define RT_BVH_AUTO   0   /* the device when the meshes hold >= RT_BVH_AUTO_MIN_TRIS triangles */
#define RT_BVH_HOST   1   /* host threads */
#define RT_BVH_DEVICE 2   /* the current device (the host when the device build fails) */
#define RT_BVH_AUTO_MIN_TRIS 65536

typedef struct RtSceneOptions {
    int32_t bvh_build;            /* RT_BVH_* */
    int32_t reserved[7];          /* zero */
} RtSceneOptions;

/* rt_scene_create with options (null: the defaults, all zero). */
int rt_scene_create_ex(const RtWorldDesc* world, const RtSceneOptions* options, RtScene** out_scene);

/* Scene summary for tests and logs. */
typedef struct RtSceneInfo {
    int64_t num_nodes;            /* flattened BVH nodes (top level + all meshes) */
    int64_t num_tris;
    int32_t num_entities;
    int32_t num_lights;           /* explicit + derived geometry lights */
    int32_t top_is_bvh;           /* 0: the world is a flat list (<= 4 objects) */
    int32_t max_stack_depth;      /* traversal stack entries the scene needs */
    int32_t rr_min_bounces;       /* the reference's classifier result */
    float   rr_min_survival;
    float   mean_irradiance;      /* classifier input, Renderer.cs:361-372 */
    int32_t bvh_on_device;        /* 1: the mesh BVHs came from the device build */
    int64_t device_bytes;
    double  bvh_build_ms;         /* wall time of the mesh-BVH build */
} RtSceneInfo;
int rt_scene_info(const RtScene* scene, RtSceneInfo* info);

/* Copies the flattened BVH: nodes as 8 x int32 words each (bmin xyz as float
 * bits, a, bmax xyz as float bits, b), and the item arrays. Any pointer may be
 * null to skip that array. Used to compare against the oracle's build. */
int rt_scene_export_bvh(const RtScene* scene, int32_t* nodes, int64_t max_nodes,
                        int32_t* top_items, int64_t max_top_items,
                        int32_t* tri_order, int64_t max_tris);

/* Host-only world assembly without a device: runs the same build as
 * rt_scene_create and returns the summary and the flattened BVH (same export
 * layout as rt_scene_export_bvh). Lets a host without a GPU inspect the
 * build; no device memory is touched. */
int rt_world_inspect(const RtWorldDesc* world, RtSceneInfo* info, int32_t* nodes, int64_t max_nodes,
                     int32_t* top_items, int64_t max_top_items, int32_t* tri_order, int64_t max_tris);

/* ---- rendering ----------------------------------------------------------- */
/* Renders into a caller-owned planar fp32 buffer of 3*W*H floats (host memory).
 * The linear-HDR mean of the clamped per-sample radiance, before exposure. */
int rt_render(RtScene* scene, const RtRenderParams* params, float* hdr_rgb_planar,
              RtStats* stats);

/* Same, with the film left in caller-owned DEVICE memory (3*W*H floats); no
 * host copies. The call still synchronises before returning. */
int rt_render_device(RtScene* scene, const RtRenderParams* params, float* d_hdr_rgb_planar,
                     RtStats* stats);

/* Allocation-free variant of rt_render_device (megakernel only). No
 * counterpart in the reference. For hosts that cannot allocate device memory
 * while rendering — a host whose device-memory budget is fixed at start-up,
 * or one rendering from a latency-critical thread where cudaMalloc/cudaFree
 * (which synchronise the device) are not allowed. The caller passes the scene
 * and a device film of 3*W*H floats; the kernel's scratch (partial sums and
 * the error word) lives in one fixed 32 MiB array inside the library, so the
 * call makes no allocation. Limits and rules:
 *   - the render window may hold at most 2 796 181 pixels (3 floats each in
 *     8 Mi floats minus a 256-byte header); larger windows return
 *     RT_ERR_INVALID_ARG; count_work is rejected, and so is any
 *     params->kernel other than RT_KERNEL_MEGAKERNEL;
 *   - the first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress); make that first call before any stream capture;
 *   - every call shares the array: calls that overlap on the GPU (any scenes,
 *     any threads) race and must be serialised by the caller. */
int rt_render_device_noalloc(RtScene* scene, const RtRenderParams* params, float* d_hdr_rgb_planar,
                             RtStats* stats);

/* One request of a batch. */
typedef struct RtRequest {
    int32_t scene;                /* index into the scenes array */
    int32_t width, height, spp, max_depth;
    int32_t pad;
    RtCameraDesc camera;          /* per-request camera (overrides the scene's) */
} RtRequest;

/* Renders n requests of uneven size in one persistent wavefront launch.
 * outs[i] is a host buffer of 3*W_i*H_i floats. Every distinct scene of the
 * batch is locked for the duration of the call, like a single-scene call. */
int rt_render_batch(RtScene* const* scenes, int32_t num_scenes,
                    const RtRequest* requests, int32_t n,
                    const RtRenderParams* common, float* const* outs, RtStats* stats);

/* Capture planes of a capturing render (Rendering/RenderBuffers.cs): the
 * linear-HDR even/odd sample halves the denoiser's variance estimate needs,
 * and the first-non-delta-hit AOVs, each split the same way. A holds the
 * ceil(n/2) even samples of the call, B the floor(n/2) odd ones (B mirrors A
 * when n == 1); each is a mean. Colour planes are 3*W*H floats (planar),
 * depth W*H (world-space distance; -1 where no sample of the half hit
 * geometry). Host pointers, each null to skip its plane. */
typedef struct RtCapture {
    float* beauty_a;
    float* beauty_b;
    float* albedo_a;
    float* albedo_b;
    float* normal_a;
    float* normal_b;
    float* depth_a;
    float* depth_b;
} RtCapture;

/* Renderer.Render(w, h, RenderCaptureOptions.Full) (Renderer.cs:522-733 with
 * the AOV probe :755-856): the beauty film as rt_render plus the planes of
 * `capture`. It always runs the plain megakernel (params->kernel is ignored)
 * over the whole frame; a render window or count_work is RT_ERR_INVALID_ARG.
 * The capture draws nothing from the sampler, so the beauty film equals
 * rt_render's megakernel film up to the order of the per-pixel sums. */
int rt_render_capture(RtScene* scene, const RtRenderParams* params, float* hdr_rgb_planar,
                      const RtCapture* capture, RtStats* stats);

/* Autotuner: times the wavefront over wavefront size {256K, 1M, 4M} x block
 * {64, 128, 256} x material sort {off, on} x node layout {two-wide,
 * four-wide}, then, on the winner, the extend/occlude block {64, 128, 256},
 * the ray order {block-local regrouping, sorted bounce rays, sorted bounce
 * and shadow rays} and the persistent dynamic-fetch kernels, on a bounded
 * slice of `params` (the full window at the spp giving ~16 M samples), keeps
 * the fastest for this scene (used when those params fields are 0 / -1) and
 * returns it. */
int rt_autotune(RtScene* scene, const RtRenderParams* params, RtRenderParams* best);

/* ---- differentiation ----------------------------------------------------- */
/* The differentiable parameter vector of a scene: 16 floats per material, in
 * material order, then 6 floats of the global medium. Total
 * RT_ADJ_PARAMS_PER_MATERIAL * num_materials + RT_ADJ_GLOBAL_PARAMS.
 * Disney material slots (the RtMaterialDesc fields, before the constructor's
 * clamps; a clamped-out value has zero derivative): */
#define RT_ADJ_BASE_COLOR      0   /* [3] baseColor                                   */
#define RT_ADJ_ROUGHNESS       3
#define RT_ADJ_METALLIC        4
#define RT_ADJ_SPECULAR        5
#define RT_ADJ_SPECULAR_TINT   6
#define RT_ADJ_SHEEN           7
#define RT_ADJ_SHEEN_TINT      8
#define RT_ADJ_CLEARCOAT       9
#define RT_ADJ_SPEC_TRANS     10
#define RT_ADJ_ANISOTROPIC    11
#define RT_ADJ_ABSORPTION     12   /* [3] interior Beer-Lambert sigma_a per unit length:
                                      -ln(transmission_color) / transmission_depth     */
/* Emissive material slots: */
#define RT_ADJ_RADIANCE        0   /* [3] emitted radiance, colour * intensity         */
#define RT_ADJ_PARAMS_PER_MATERIAL 16
/* Global slots after the materials: homogeneous medium sigma_a[3], sigma_s[3]. */
#define RT_ADJ_MEDIUM_SIGMA_A  0
#define RT_ADJ_MEDIUM_SIGMA_S  3
#define RT_ADJ_GLOBAL_PARAMS   6

/* Path-replay adjoint. dL_dimage_planar is the host gradient of a scalar
 * loss with respect to the 3*H*W planar HDR film that rt_render returns for
 * the same params (same spp and spp_offset). Every sample is traced twice from
 * its Sobol indices: a primal pass for the sample radiance, then a replay that
 * accumulates the gradient; nothing is stored per bounce. Sampling decisions
 * (directions, lobe choice, light samples, MIS weights, Russian roulette) are
 * held fixed, with score terms for the two discrete events whose probability
 * the reference's estimator keeps (a lobe weight divided by max(p, floor), and
 * a null Sample followed by the legacy Scatter draw) and, for the samples the
 * luminance clamps saturate, for the medium's free-flight draws and Russian
 * roulette (with respect to the medium's slots); geometry and visibility
 * edges are not differentiated. Writes the gradient (float, host) in the
 * parameter-vector layout above; count is that layout's length. mask (count
 * bytes, or NULL for all) selects the slots to differentiate; unselected slots
 * come back 0 and cost nothing (a material with no selected BSDF slot skips
 * the dual-number BSDF evaluations). params->kernel selects the form:
 * RT_KERNEL_MEGAKERNEL traces both passes of a sample in one thread;
 * RT_KERNEL_WAVEFRONT renders runs of at most 2^24 samples with the wavefront
 * kernels, keeping each sample's end state (64 B, device memory for one run),
 * then replays them on the wavefront with the gradient hooks and the shadow
 * rays inline. Both give the same gradient up to the order of the float sums.
 * count_work must be 0. */
int rt_adjoint(RtScene* scene, const RtRenderParams* params,
               const float* dL_dimage_planar, const uint8_t* mask,
               float* dL_dparams, int32_t count, RtStats* stats);
/* Reads / overwrites the parameter vector (count floats, layout above). Set
 * rebuilds the scene's materials, lights and Russian-roulette classifier from
 * the stored world description, exactly as rt_scene_create would from a world
 * with those values; the BVH is untouched. A slot equal to what get reports
 * leaves its field untouched, so set(get()) changes nothing. */
int rt_scene_get_params(const RtScene* scene, float* params, int32_t count);
int rt_scene_set_params(RtScene* scene, const float* params, int32_t count);

/* ---- test-only entry points --------------------------------------------- */
/* Ray in: origin[3], dir[3] (8 floats per ray, last two ignored).
 * Closest hit out per ray: t, u, v as float, entity id, local primitive id
 * (int32 bits), and a hit flag: 6 words. node_layout: 2 (two-wide records)
 * or 4 (four-wide), the layouts the wavefront can run on. */
int rt_trace_closest(RtScene* scene, const float* rays, int64_t n, float tmin, float tmax,
                     int32_t* hits, int32_t node_layout);
/* Shadow rays in: origin[3], dir[3], tmin, tmax. Out: transmittance rgb. */
int rt_trace_any(RtScene* scene, const float* rays, int64_t n, float* transmittance, int32_t node_layout);

/* BSDF batch. Each record (RtBsdfQuery) carries the shading inputs; the
 * results are the Sample outcome and Evaluate/Pdf/EvaluateDirect values. */
typedef struct RtBsdfQuery {
    int32_t material;
    int32_t front_face;
    uint32_t pixel_seed, sample_index;   /* Sobol stream for the sample draws */
    uint32_t dim;                        /* first dimension the sample consumes */
    int32_t pad;
    float n[3], tangent[3], bitangent[3];
    float v[3];                          /* view direction (toward the eye)     */
    float l[3];                          /* direction for Evaluate/Pdf/Direct   */
    float point[3];
} RtBsdfQuery;
typedef struct RtBsdfResult {
    float f[3];  float pdf;              /* Evaluate(V, L), Pdf(V, L) */
    float fd[3]; float pad0;             /* EvaluateDirect(L, V, N)   */
    float wo[3]; float s_pdf;            /* Sample: direction, pdf    */
    float s_f[3];
    int32_t lobe;                        /* 0..6 (Diffuse..Clearcoat), -1 none */
    int32_t is_delta;
    int32_t has_sample;
    uint32_t dims_used;
    int32_t transition;                  /* Sample's BsdfSample.Transition: 0 none, 1 enter, 2 exit */
} RtBsdfResult;
int rt_bsdf_batch(RtScene* scene, const RtBsdfQuery* q, int64_t n, RtBsdfResult* out);

/* Medium batch: the scene's global homogeneous medium and its
 * Henyey-Greenstein phase on one Sobol stream per query. In this order:
 *   HomogeneousMedium.Sample over a segment of length tmax (hero channel, then
 *   the distance draw when that channel's sigma_t > 0;
 *   Volumetrics/HomogeneousMedium.cs:46-76), then
 *   HenyeyGreensteinPhase.Sample(wo) with the next two draws
 *   (Volumetrics/HenyeyGreensteinPhase.cs:32-54), plus
 *   Transmittance(tmax) (HomogeneousMedium.cs:36-44) and Evaluate(wo, wi)
 *   (HenyeyGreensteinPhase.cs:23-30). wo is the incoming ray direction, as
 *   the renderer passes it (Renderer.cs:1750-1765). A scene without a medium
 *   is RT_ERR_INVALID_ARG. */
typedef struct RtMediumQuery {
    uint32_t pixel_seed, sample_index, dim;
    float tmax;
    float wo[3];
    float wi[3];
} RtMediumQuery;
typedef struct RtMediumResult {
    int32_t scattered;                   /* Sample: a scattering event before tmax */
    uint32_t dims_used;                  /* Sobol dimensions both samples consumed */
    float t;                             /* Sample: the event's distance (tmax when it passed) */
    float phase_eval;                    /* Evaluate(wo, wi) */
    float beta[3];                       /* Sample: the segment's weight */
    float tr[3];                         /* Transmittance(tmax) */
    float phase_wi[3];                   /* phase Sample: direction */
    float phase_pdf;                     /* phase Sample: pdf */
} RtMediumResult;
int rt_medium_batch(RtScene* scene, const RtMediumQuery* q, int64_t n, RtMediumResult* out);

/* Owen-scrambled Sobol draws: out[i] = Sample(idx[i], dim[i], seed[i]). */
int rt_sobol_batch(const uint32_t* sample_index, const uint32_t* dim, const uint32_t* pixel_seed,
                   int64_t n, float* out);

/* Display transform: exposure gain 2^ev, ACES filmic fit, gamma 1/2.2
 * (Renderer.AcesToneMap, Rendering/Renderer.cs:893-907). Planar HDR in
 * (3*W*H host floats), interleaved RGB out (W*H*3 host floats in [0, 1]).
 * It takes no scene, so it runs on the calling thread's current device. */
int rt_tonemap(const float* hdr_rgb_planar, int32_t width, int32_t height, float exposure_ev, float* rgb_out);

/* Kulla-Conty tables the scene uses: E (32x32, mu-major) then E_avg (32). */
int rt_energy_lut(float* e_1024, float* eavg_32);
/* L2 read bandwidth of a device in GB/s: `passes` streams over a `bytes`
 * buffer (choose it to fit L2) through L2-only loads. The L2 roofline's peak;
 * no counterpart in the reference. */
int rt_probe_l2_bandwidth(int32_t device, int64_t bytes, int32_t passes, double* gbs);

#ifdef __cplusplus
}
#endif
#endif /* RT3D_H */
