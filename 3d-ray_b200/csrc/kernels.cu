// Kernels and the C-ABI (include/rt3d.h) of the B200 path-tracing core.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rt3d.h"
#include "integrator.cuh"
#include "world.h"

using rt::V3;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CUDA_TRY(x)                                                                            \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) return fail(RT_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int kStack = 64;       // traversal stack entries per thread
constexpr int kBlock = 128;      // 16 x 8 pixel tiles

}  // namespace

struct RtScene {
    rt::HostScene host;
    rt::SceneView view{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::mutex mu;
    std::vector<void*> allocs;
    int opaque = 1;
    int dielectrics = 0;
    size_t bytes = 0;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    int* d_err = nullptr;
};

namespace {

template <typename T>
int upload(RtScene* sc, const std::vector<T>& v, const T** out) {
    if (v.empty()) {
        *out = nullptr;
        return RT_OK;
    }
    void* p = nullptr;
    size_t n = v.size() * sizeof(T);
    if (cudaMalloc(&p, n) != cudaSuccess) return fail(RT_ERR_OOM, "cudaMalloc of " + std::to_string(n) + " bytes failed");
    sc->allocs.push_back(p);
    sc->bytes += n;
    CUDA_TRY(cudaMemcpy(p, v.data(), n, cudaMemcpyHostToDevice));
    *out = static_cast<const T*>(p);
    return RT_OK;
}

int ensure_scratch(RtScene* sc, size_t bytes) {
    if (sc->scratch_bytes >= bytes) return RT_OK;
    if (sc->scratch) cudaFree(sc->scratch);
    sc->scratch = nullptr;
    sc->scratch_bytes = 0;
    if (cudaMalloc(&sc->scratch, bytes) != cudaSuccess) return fail(RT_ERR_OOM, "scratch allocation failed");
    sc->scratch_bytes = bytes;
    return RT_OK;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// Plain megakernel: one thread per (pixel, sample chunk), the whole path of
// each sample in registers. Chunks write partial sums; k_resolve adds them.
template <int STACK, bool COUNT>
__global__ void __launch_bounds__(kBlock) k_render_mega(rt::SceneView s, rt::RenderConst rc, int x0, int y0, int ww,
                                                         int wh, int spp0, int per_chunk, int spp, float* partial,
                                                         unsigned long long* work, int* err) {
    int lx = blockIdx.x * 16 + (threadIdx.x & 15);
    int ly = blockIdx.y * 8 + (threadIdx.x >> 4);
    int chunk = blockIdx.z;
    if (lx >= ww || ly >= wh) return;
    int sb = chunk * per_chunk;
    int se = min(sb + per_chunk, spp);
    V3 sum = rt::v3(0.0f);
    rt::Counters cnt{0u, 0u, 0u, 0u, 0u};
    for (int si = sb; si < se; si++)
        sum = sum + rt::trace_sample<STACK, COUNT>(s, rc, x0 + lx, y0 + ly, (uint32_t)(spp0 + si), &cnt, err);
    if (COUNT) {
        atomicAdd(work + 0, (unsigned long long)cnt.nodes);
        atomicAdd(work + 1, (unsigned long long)cnt.tris);
        atomicAdd(work + 2, (unsigned long long)cnt.others);
        atomicAdd(work + 3, (unsigned long long)cnt.closest_rays);
        atomicAdd(work + 4, (unsigned long long)cnt.shadow_rays);
    }
    size_t plane = (size_t)ww * wh;
    float* out = partial + (size_t)chunk * 3 * plane + (size_t)ly * ww + lx;
    out[0] = sum.x;
    out[plane] = sum.y;
    out[2 * plane] = sum.z;
}

// Mean over the chunks (Renderer.cs:711: cumulativeColor / actualSamples).
__global__ void k_resolve(const float* partial, int nchunks, int ww, int wh, int W, int H, int x0, int y0, int spp,
                          float* film) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int plane = ww * wh;
    if (i >= plane) return;
    int lx = i % ww, ly = i / ww;
    size_t fplane = (size_t)W * H;
    size_t fi = (size_t)(y0 + ly) * W + (x0 + lx);
    for (int c = 0; c < 3; c++) {
        float a = partial[(size_t)c * plane + i];
        for (int k = 1; k < nchunks; k++) a += partial[(size_t)k * 3 * plane + (size_t)c * plane + i];
        film[c * fplane + fi] = a / (float)spp;
    }
}

template <int STACK>
__global__ void k_trace_closest(rt::SceneView s, const float* rays, int64_t n, float tmin, float tmax, int* hits,
                                int* err) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + i * 8;
    V3 o = rt::v3(r[0], r[1], r[2]), d = rt::v3(r[3], r[4], r[5]);
    rt::Hit h;
    rt::traverse<false, STACK>(s, o, d, tmin, tmax, h, nullptr, err);
    int* out = hits + i * 6;
    if (h.kind == rt::HIT_NONE) {
        out[0] = out[1] = out[2] = 0;
        out[3] = out[4] = -1;
        out[5] = 0;
        return;
    }
    rt::Surface rec = rt::make_surface(s, h, o, d);
    out[0] = __float_as_int(h.t);
    out[1] = __float_as_int(h.u);
    out[2] = __float_as_int(h.v);
    out[3] = rec.entity;
    out[4] = rec.prim;
    out[5] = 1;
}

template <int STACK>
__global__ void k_trace_any(rt::SceneView s, int opaque, const float* rays, int64_t n, float* out, int* err) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + i * 8;
    V3 t = rt::shadow_transmittance<STACK>(s, opaque, rt::v3(r[0], r[1], r[2]), rt::v3(r[3], r[4], r[5]), r[6], r[7],
                                           nullptr, err);
    out[i * 3] = t.x;
    out[i * 3 + 1] = t.y;
    out[i * 3 + 2] = t.z;
}

__global__ void k_bsdf(rt::SceneView s, const RtBsdfQuery* q, int64_t n, RtBsdfResult* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    RtBsdfQuery qq = q[i];
    RtBsdfResult r;
    memset(&r, 0, sizeof(r));
    const rt::Material& m = s.materials[qq.material];
    if (m.type != 0) {
        r.lobe = -1;
        out[i] = r;
        return;
    }
    rt::Surface rec;
    rec.n = rt::v3(qq.n[0], qq.n[1], qq.n[2]);
    rec.tangent = rt::v3(qq.tangent[0], qq.tangent[1], qq.tangent[2]);
    rec.bitangent = rt::v3(qq.bitangent[0], qq.bitangent[1], qq.bitangent[2]);
    rec.p = rt::v3(qq.point[0], qq.point[1], qq.point[2]);
    rec.front = qq.front_face;
    rec.material = qq.material;
    V3 V = rt::v3(qq.v[0], qq.v[1], qq.v[2]);
    V3 L = rt::v3(qq.l[0], qq.l[1], qq.l[2]);
    V3 f = rt::bsdf_eval(s, m, rec, V, L);
    r.f[0] = f.x; r.f[1] = f.y; r.f[2] = f.z;
    r.pdf = rt::bsdf_pdf(m, rec, V, L);
    V3 fd = rt::bsdf_eval_direct(s, m, rec, L, V, rec.n);
    r.fd[0] = fd.x; r.fd[1] = fd.y; r.fd[2] = fd.z;
    rt::Sampler rng{qq.pixel_seed, qq.sample_index, qq.dim};
    rt::BsdfSample bs;
    bool has = rt::bsdf_sample(s, m, rec, V, 0.0f, rng, bs);
    r.dims_used = rng.dim - qq.dim;
    r.lobe = bs.lobe;
    r.has_sample = has ? 1 : 0;
    if (has) {
        r.wo[0] = bs.wo.x; r.wo[1] = bs.wo.y; r.wo[2] = bs.wo.z;
        r.s_f[0] = bs.f.x; r.s_f[1] = bs.f.y; r.s_f[2] = bs.f.z;
        r.s_pdf = bs.pdf;
        r.is_delta = bs.is_delta;
    }
    out[i] = r;
}

__global__ void k_sobol(const uint32_t* idx, const uint32_t* dim, const uint32_t* seed, int64_t n, float* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = rt::sobol_sample(idx[i], dim[i], seed[i]);
}

int check_err(RtScene* sc) {
    int e = 0;
    CUDA_TRY(cudaMemcpyAsync(&e, sc->d_err, sizeof(int), cudaMemcpyDeviceToHost, sc->stream));
    CUDA_TRY(cudaStreamSynchronize(sc->stream));
    if (e == RT_ERR_STACK) return fail(RT_ERR_STACK, "traversal stack bound exceeded");
    if (e != 0) return fail(RT_ERR_BOUNDS, "device error " + std::to_string(e));
    return RT_OK;
}

int validate_params(const RtScene* sc, const RtRenderParams* p) {
    if (!p) return fail(RT_ERR_INVALID_ARG, "null params");
    if (p->width <= 0 || p->height <= 0 || p->spp <= 0 || p->max_depth < 0)
        return fail(RT_ERR_INVALID_ARG, "width, height and spp must be positive, max_depth non-negative");
    if ((int64_t)p->width * p->height > (int64_t)1 << 28) return fail(RT_ERR_INVALID_ARG, "image too large");
    if (p->light_strategy != RT_LIGHTS_ALL)
        return fail(RT_ERR_UNSUPPORTED, "only the 'all' light strategy is on the GPU path");
    int ww = p->window_w > 0 ? p->window_w : p->width;
    int wh = p->window_h > 0 ? p->window_h : p->height;
    if (p->pixel_x0 < 0 || p->pixel_y0 < 0 || p->pixel_x0 + ww > p->width || p->pixel_y0 + wh > p->height)
        return fail(RT_ERR_INVALID_ARG, "render window outside the image");
    if (sc->host.max_stack > kStack)
        return fail(RT_ERR_STACK, "scene needs a traversal stack of " + std::to_string(sc->host.max_stack));
    return RT_OK;
}

rt::RenderConst make_rc(const RtScene* sc, const RtRenderParams* p, const RtCameraDesc& cam) {
    rt::RenderConst rc;
    rc.cam = rt::make_camera(cam, (float)p->width / (float)p->height);
    rc.width = p->width;
    rc.height = p->height;
    rc.max_depth = p->max_depth;
    rc.max_rad = p->max_sample_radiance > 0.0f ? p->max_sample_radiance : 10.0f;
    float icf = p->indirect_clamp_factor >= 0.0f ? p->indirect_clamp_factor : 0.25f;
    rc.ind_max = rc.max_rad * std::fmax(0.0f, icf);
    rc.mis_power = p->mis_heuristic == RT_MIS_POWER;
    rc.rr_min_bounces = p->rr_min_bounces >= 0 ? p->rr_min_bounces : sc->host.rr_min_bounces;
    rc.rr_min_survival = p->rr_min_bounces >= 0 ? p->rr_min_survival : sc->host.rr_min_survival;
    rc.opaque = sc->opaque;
    rc.dielectrics = sc->dielectrics;
    return rc;
}

// Renders into a device film (3*W*H, planar). Caller holds sc->mu.
int render_to_device(RtScene* sc, const RtRenderParams* p, const RtCameraDesc& cam, float* d_film, RtStats* st) {
    auto t0 = std::chrono::steady_clock::now();
    int rc_ = validate_params(sc, p);
    if (rc_ != RT_OK) return rc_;
    CUDA_TRY(cudaSetDevice(sc->device));
    rt::RenderConst rc = make_rc(sc, p, cam);
    int ww = p->window_w > 0 ? p->window_w : p->width;
    int wh = p->window_h > 0 ? p->window_h : p->height;
    int64_t npix = (int64_t)ww * wh;
    // Enough (pixel, chunk) threads to fill 148 SMs several times over.
    int64_t target = 148LL * 2048 * 2;
    int nchunks = (int)std::min<int64_t>(p->spp, std::max<int64_t>(1, (target + npix - 1) / npix));
    int per_chunk = (p->spp + nchunks - 1) / nchunks;
    nchunks = (p->spp + per_chunk - 1) / per_chunk;
    size_t partial_bytes = (size_t)nchunks * 3 * npix * sizeof(float);
    rc_ = ensure_scratch(sc, partial_bytes + 8 * sizeof(unsigned long long));
    if (rc_ != RT_OK) return rc_;
    float* partial = static_cast<float*>(sc->scratch);
    auto* work = reinterpret_cast<unsigned long long*>(static_cast<char*>(sc->scratch) + partial_bytes);
    bool count = p->count_work != 0;
    if (count) CUDA_TRY(cudaMemsetAsync(work, 0, 8 * sizeof(unsigned long long), sc->stream));
    CUDA_TRY(cudaMemsetAsync(sc->d_err, 0, sizeof(int), sc->stream));
    if (p->window_w > 0 || p->window_h > 0)
        CUDA_TRY(cudaMemsetAsync(d_film, 0, (size_t)3 * p->width * p->height * sizeof(float), sc->stream));
    dim3 grid((ww + 15) / 16, (wh + 7) / 8, nchunks);
    CUDA_TRY(cudaEventRecord(sc->ev0, sc->stream));
    if (count)
        k_render_mega<kStack, true><<<grid, kBlock, 0, sc->stream>>>(sc->view, rc, p->pixel_x0, p->pixel_y0, ww, wh,
                                                                     p->spp_offset, per_chunk, p->spp, partial, work,
                                                                     sc->d_err);
    else
        k_render_mega<kStack, false><<<grid, kBlock, 0, sc->stream>>>(sc->view, rc, p->pixel_x0, p->pixel_y0, ww, wh,
                                                                      p->spp_offset, per_chunk, p->spp, partial, work,
                                                                      sc->d_err);
    k_resolve<<<(unsigned)((npix + 255) / 256), 256, 0, sc->stream>>>(partial, nchunks, ww, wh, p->width, p->height,
                                                                     p->pixel_x0, p->pixel_y0, p->spp, d_film);
    CUDA_TRY(cudaEventRecord(sc->ev1, sc->stream));
    CUDA_TRY(cudaGetLastError());
    rc_ = check_err(sc);
    if (rc_ != RT_OK) return rc_;
    if (st) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, sc->ev0, sc->ev1);
        st->kernel_ms = ms;
        st->samples = (uint64_t)npix * (uint64_t)p->spp;
        st->kernel_launches = 2;
        st->rr_min_bounces = rc.rr_min_bounces;
        st->rr_min_survival = rc.rr_min_survival;
        if (count) {
            unsigned long long w[8];
            CUDA_TRY(cudaMemcpy(w, work, sizeof(w), cudaMemcpyDeviceToHost));
            st->node_visits = w[0];
            st->prim_tests = w[1];
            st->other_tests = w[2];
            st->closest_rays = w[3];
            st->shadow_rays = w[4];
        }
        st->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return RT_OK;
}

}  // namespace

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

int rt_abi_version(void) { return RT3D_ABI_VERSION; }

const char* rt_last_error(void) { return g_err.c_str(); }

int rt_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return fail(RT_ERR_NO_DEVICE, "no CUDA device");
    return n;
}

int rt_scene_create(const RtWorldDesc* world, RtScene** out) {
    if (!world || !out) return fail(RT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(RT_ERR_NO_DEVICE, "no CUDA device");
    auto* sc = new RtScene();
    std::string err;
    int rc = rt::build_world(world, sc->host, err);
    if (rc != RT_OK) {
        delete sc;
        return fail(rc, err);
    }
    cudaGetDevice(&sc->device);
    const rt::HostScene& h = sc->host;
    rt::SceneView& v = sc->view;
    int r = RT_OK;
    r = r ? r : upload(sc, h.nodes, &v.nodes);
    r = r ? r : upload(sc, h.top_items, &v.top_items);
    r = r ? r : upload(sc, h.tris, &v.tris);
    r = r ? r : upload(sc, h.tri_entity, &v.tri_entity);
    r = r ? r : upload(sc, h.tri_local, &v.tri_local);
    r = r ? r : upload(sc, h.entities, &v.entities);
    r = r ? r : upload(sc, h.quads, &v.quads);
    r = r ? r : upload(sc, h.spheres, &v.spheres);
    r = r ? r : upload(sc, h.materials, &v.materials);
    r = r ? r : upload(sc, h.lights, &v.lights);
    r = r ? r : upload(sc, h.light_tris, &v.light_tris);
    r = r ? r : upload(sc, h.emitter_light, &v.emitter_light);
    r = r ? r : upload(sc, h.lut_e, &v.lut_e);
    r = r ? r : upload(sc, h.lut_eavg, &v.lut_eavg);
    if (r != RT_OK) {
        rt_scene_destroy(sc);
        return r;
    }
    v.num_lights = (int)h.lights.size();
    v.top_root = h.top_root;
    v.num_top_items = (int)h.top_items.size();
    v.has_medium = h.has_medium;
    v.sigma_a = h.sigma_a;
    v.sigma_s = h.sigma_s;
    v.sigma_t = h.sigma_t;
    v.hg_g = h.hg_g;
    sc->opaque = 1;
    sc->dielectrics = 0;
    for (const rt::Material& m : h.materials) {
        if (m.type == 0 && m.spec_trans_raw > 0.0f) {
            sc->opaque = 0;
            if (!m.thin_walled) sc->dielectrics = 1;
        }
    }
    if (cudaStreamCreateWithFlags(&sc->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&sc->ev0) != cudaSuccess || cudaEventCreate(&sc->ev1) != cudaSuccess ||
        cudaMalloc(&sc->d_err, sizeof(int)) != cudaSuccess) {
        rt_scene_destroy(sc);
        return fail(RT_ERR_CUDA, "stream/event/flag creation failed");
    }
    *out = sc;
    return RT_OK;
}

int rt_scene_destroy(RtScene* sc) {
    if (!sc) return RT_OK;
    cudaSetDevice(sc->device);
    if (sc->stream) cudaStreamSynchronize(sc->stream);
    for (void* p : sc->allocs) cudaFree(p);
    if (sc->scratch) cudaFree(sc->scratch);
    if (sc->d_err) cudaFree(sc->d_err);
    if (sc->ev0) cudaEventDestroy(sc->ev0);
    if (sc->ev1) cudaEventDestroy(sc->ev1);
    if (sc->stream) cudaStreamDestroy(sc->stream);
    delete sc;
    return RT_OK;
}

int rt_scene_info(const RtScene* sc, RtSceneInfo* info) {
    if (!sc || !info) return fail(RT_ERR_INVALID_ARG, "null argument");
    const rt::HostScene& h = sc->host;
    info->num_nodes = (int64_t)h.nodes.size();
    info->num_tris = (int64_t)h.tri_entity.size();
    info->num_entities = (int32_t)h.entities.size();
    info->num_lights = (int32_t)h.lights.size();
    info->top_is_bvh = h.top_is_bvh;
    info->max_stack_depth = h.max_stack;
    info->rr_min_bounces = h.rr_min_bounces;
    info->rr_min_survival = h.rr_min_survival;
    info->mean_irradiance = h.mean_irradiance;
    info->device_bytes = (int64_t)sc->bytes;
    return RT_OK;
}

int rt_scene_export_bvh(const RtScene* sc, int32_t* nodes, int64_t max_nodes, int32_t* top_items,
                        int64_t max_top_items, int32_t* tri_order, int64_t max_tris) {
    if (!sc) return fail(RT_ERR_INVALID_ARG, "null scene");
    const rt::HostScene& h = sc->host;
    if (nodes) {
        int64_t n = std::min<int64_t>(max_nodes, (int64_t)h.nodes.size());
        std::memcpy(nodes, h.nodes.data(), (size_t)n * sizeof(rt::NodeF));
    }
    if (top_items) {
        int64_t n = std::min<int64_t>(max_top_items, (int64_t)h.top_items.size());
        std::memcpy(top_items, h.top_items.data(), (size_t)n * sizeof(int));
    }
    if (tri_order) {
        int64_t n = std::min<int64_t>(max_tris, (int64_t)h.tri_local.size());
        std::memcpy(tri_order, h.tri_local.data(), (size_t)n * sizeof(int));
    }
    return RT_OK;
}

int rt_world_inspect(const RtWorldDesc* world, RtSceneInfo* info, int32_t* nodes, int64_t max_nodes,
                     int32_t* top_items, int64_t max_top_items, int32_t* tri_order, int64_t max_tris) {
    if (!world) return fail(RT_ERR_INVALID_ARG, "null world");
    rt::HostScene h;
    std::string err;
    int rc = rt::build_world(world, h, err);
    if (rc != RT_OK) return fail(rc, err);
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->num_nodes = (int64_t)h.nodes.size();
        info->num_tris = (int64_t)h.tri_entity.size();
        info->num_entities = (int32_t)h.entities.size();
        info->num_lights = (int32_t)h.lights.size();
        info->top_is_bvh = h.top_is_bvh;
        info->max_stack_depth = h.max_stack;
        info->rr_min_bounces = h.rr_min_bounces;
        info->rr_min_survival = h.rr_min_survival;
        info->mean_irradiance = h.mean_irradiance;
    }
    if (nodes) std::memcpy(nodes, h.nodes.data(), (size_t)std::min<int64_t>(max_nodes, (int64_t)h.nodes.size()) * sizeof(rt::NodeF));
    if (top_items)
        std::memcpy(top_items, h.top_items.data(),
                    (size_t)std::min<int64_t>(max_top_items, (int64_t)h.top_items.size()) * sizeof(int));
    if (tri_order)
        std::memcpy(tri_order, h.tri_local.data(), (size_t)std::min<int64_t>(max_tris, (int64_t)h.tri_local.size()) * sizeof(int));
    return RT_OK;
}

int rt_render_device(RtScene* sc, const RtRenderParams* p, float* d_film, RtStats* st) {
    if (!sc || !d_film) return fail(RT_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(sc->mu);
    return render_to_device(sc, p, sc->host.camera, d_film, st);
}

int rt_render(RtScene* sc, const RtRenderParams* p, float* out, RtStats* st) {
    if (!sc || !out || !p) return fail(RT_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(sc->mu);
    auto t0 = std::chrono::steady_clock::now();
    size_t film_bytes = (size_t)3 * p->width * p->height * sizeof(float);
    float* d_film = nullptr;
    if (p->width <= 0 || p->height <= 0) return fail(RT_ERR_INVALID_ARG, "bad image size");
    CUDA_TRY(cudaSetDevice(sc->device));
    if (cudaMalloc(&d_film, film_bytes) != cudaSuccess) return fail(RT_ERR_OOM, "film allocation failed");
    int rc = render_to_device(sc, p, sc->host.camera, d_film, st);
    if (rc == RT_OK) {
        if (cudaMemcpyAsync(out, d_film, film_bytes, cudaMemcpyDeviceToHost, sc->stream) != cudaSuccess ||
            cudaStreamSynchronize(sc->stream) != cudaSuccess)
            rc = fail(RT_ERR_CUDA, "film copy failed");
    }
    cudaFree(d_film);
    if (st && rc == RT_OK)
        st->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int rt_render_batch(RtScene* const* scenes, int32_t num_scenes, const RtRequest* reqs, int32_t n,
                    const RtRenderParams* common, float* const* outs, RtStats* st) {
    if (!scenes || !reqs || !outs || !common || n < 0 || num_scenes <= 0)
        return fail(RT_ERR_INVALID_ARG, "null argument");
    RtStats total{};
    for (int i = 0; i < n; i++) {
        const RtRequest& q = reqs[i];
        if (q.scene < 0 || q.scene >= num_scenes || !scenes[q.scene] || !outs[i])
            return fail(RT_ERR_INVALID_ARG, "request " + std::to_string(i) + ": bad scene or output");
        RtScene* sc = scenes[q.scene];
        RtRenderParams p = *common;
        p.width = q.width;
        p.height = q.height;
        p.spp = q.spp;
        p.max_depth = q.max_depth;
        p.pixel_x0 = p.pixel_y0 = p.window_w = p.window_h = 0;
        std::lock_guard<std::mutex> lk(sc->mu);
        size_t film_bytes = (size_t)3 * q.width * q.height * sizeof(float);
        float* d_film = nullptr;
        if (cudaMalloc(&d_film, film_bytes) != cudaSuccess) return fail(RT_ERR_OOM, "film allocation failed");
        RtStats s1{};
        int rc = render_to_device(sc, &p, q.camera, d_film, &s1);
        if (rc == RT_OK && cudaMemcpy(outs[i], d_film, film_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(RT_ERR_CUDA, "film copy failed");
        cudaFree(d_film);
        if (rc != RT_OK) return rc;
        total.kernel_ms += s1.kernel_ms;
        total.samples += s1.samples;
        total.kernel_launches += s1.kernel_launches;
    }
    if (st) *st = total;
    return RT_OK;
}

int rt_adjoint(RtScene*, const RtRenderParams*, const float*, float*, RtStats*) {
    return fail(RT_ERR_UNSUPPORTED, "adjoint not built yet");
}

int rt_scene_set_params(RtScene*, const float*, int32_t) { return fail(RT_ERR_UNSUPPORTED, "adjoint not built yet"); }

int rt_trace_closest(RtScene* sc, const float* rays, int64_t n, float tmin, float tmax, int32_t* hits) {
    if (!sc || !rays || !hits || n < 0) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (n == 0) return RT_OK;
    std::lock_guard<std::mutex> lk(sc->mu);
    CUDA_TRY(cudaSetDevice(sc->device));
    if (sc->host.max_stack > kStack) return fail(RT_ERR_STACK, "scene stack bound exceeded");
    size_t rb = (size_t)n * 8 * sizeof(float), hb = (size_t)n * 6 * sizeof(int);
    int rc = ensure_scratch(sc, rb + hb);
    if (rc != RT_OK) return rc;
    float* d_r = static_cast<float*>(sc->scratch);
    int* d_h = reinterpret_cast<int*>(static_cast<char*>(sc->scratch) + rb);
    CUDA_TRY(cudaMemsetAsync(sc->d_err, 0, sizeof(int), sc->stream));
    CUDA_TRY(cudaMemcpyAsync(d_r, rays, rb, cudaMemcpyHostToDevice, sc->stream));
    k_trace_closest<kStack><<<(unsigned)((n + 127) / 128), 128, 0, sc->stream>>>(sc->view, d_r, n, tmin, tmax, d_h,
                                                                                 sc->d_err);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(hits, d_h, hb, cudaMemcpyDeviceToHost, sc->stream));
    return check_err(sc);
}

int rt_trace_any(RtScene* sc, const float* rays, int64_t n, float* out) {
    if (!sc || !rays || !out || n < 0) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (n == 0) return RT_OK;
    std::lock_guard<std::mutex> lk(sc->mu);
    CUDA_TRY(cudaSetDevice(sc->device));
    size_t rb = (size_t)n * 8 * sizeof(float), ob = (size_t)n * 3 * sizeof(float);
    int rc = ensure_scratch(sc, rb + ob);
    if (rc != RT_OK) return rc;
    float* d_r = static_cast<float*>(sc->scratch);
    float* d_o = reinterpret_cast<float*>(static_cast<char*>(sc->scratch) + rb);
    CUDA_TRY(cudaMemsetAsync(sc->d_err, 0, sizeof(int), sc->stream));
    CUDA_TRY(cudaMemcpyAsync(d_r, rays, rb, cudaMemcpyHostToDevice, sc->stream));
    k_trace_any<kStack><<<(unsigned)((n + 127) / 128), 128, 0, sc->stream>>>(sc->view, sc->opaque, d_r, n, d_o,
                                                                             sc->d_err);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, d_o, ob, cudaMemcpyDeviceToHost, sc->stream));
    return check_err(sc);
}

int rt_bsdf_batch(RtScene* sc, const RtBsdfQuery* q, int64_t n, RtBsdfResult* out) {
    if (!sc || !q || !out || n < 0) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (n == 0) return RT_OK;
    for (int64_t i = 0; i < n; i++)
        if (q[i].material < 0 || q[i].material >= (int)sc->host.materials.size())
            return fail(RT_ERR_INVALID_ARG, "query material out of range");
    std::lock_guard<std::mutex> lk(sc->mu);
    CUDA_TRY(cudaSetDevice(sc->device));
    size_t qb = (size_t)n * sizeof(RtBsdfQuery), ob = (size_t)n * sizeof(RtBsdfResult);
    int rc = ensure_scratch(sc, qb + ob);
    if (rc != RT_OK) return rc;
    auto* d_q = static_cast<RtBsdfQuery*>(sc->scratch);
    auto* d_o = reinterpret_cast<RtBsdfResult*>(static_cast<char*>(sc->scratch) + qb);
    CUDA_TRY(cudaMemcpyAsync(d_q, q, qb, cudaMemcpyHostToDevice, sc->stream));
    k_bsdf<<<(unsigned)((n + 127) / 128), 128, 0, sc->stream>>>(sc->view, d_q, n, d_o);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, d_o, ob, cudaMemcpyDeviceToHost, sc->stream));
    CUDA_TRY(cudaStreamSynchronize(sc->stream));
    return RT_OK;
}

int rt_sobol_batch(const uint32_t* idx, const uint32_t* dim, const uint32_t* seed, int64_t n, float* out) {
    if (!idx || !dim || !seed || !out || n < 0) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (n == 0) return RT_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(RT_ERR_NO_DEVICE, "no CUDA device");
    size_t b = (size_t)n * 4;
    char* d = nullptr;
    if (cudaMalloc(&d, 4 * b) != cudaSuccess) return fail(RT_ERR_OOM, "allocation failed");
    int rc = RT_OK;
    if (cudaMemcpy(d, idx, b, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d + b, dim, b, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d + 2 * b, seed, b, cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = fail(RT_ERR_CUDA, "copy failed");
    } else {
        k_sobol<<<(unsigned)((n + 255) / 256), 256>>>(reinterpret_cast<uint32_t*>(d), reinterpret_cast<uint32_t*>(d + b),
                                                     reinterpret_cast<uint32_t*>(d + 2 * b), n,
                                                     reinterpret_cast<float*>(d + 3 * b));
        if (cudaGetLastError() != cudaSuccess || cudaMemcpy(out, d + 3 * b, b, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(RT_ERR_CUDA, "sobol kernel failed");
    }
    cudaFree(d);
    return rc;
}

int rt_energy_lut(float* e, float* eavg) {
    std::vector<float> a(1024), b(32);
    rt::build_energy_lut(a.data(), b.data());
    if (e) std::memcpy(e, a.data(), 1024 * sizeof(float));
    if (eavg) std::memcpy(eavg, b.data(), 32 * sizeof(float));
    return RT_OK;
}

}  // extern "C"
