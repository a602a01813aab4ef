// Kernels and the C-ABI (include/rt3d.h) of the B200 path-tracing core.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rt3d.h"
#include "adjoint.cuh"
#include "integrator.cuh"
#include "wavefront.cuh"
#include "wf_adjoint.cuh"
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

static_assert(sizeof(RtMaterialDesc) == 120, "ABI layout");
static_assert(sizeof(RtEntityDesc) == 80, "ABI layout");
static_assert(sizeof(RtLightDesc) == 104, "ABI layout");
static_assert(sizeof(RtCameraDesc) == 48, "ABI layout");
static_assert(sizeof(RtMediumDesc) == 36, "ABI layout");
static_assert(sizeof(RtRenderParams) == 112, "ABI layout");
static_assert(sizeof(RtStats) == 144, "ABI layout");
static_assert(sizeof(RtBsdfQuery) == 96, "ABI layout");
static_assert(sizeof(RtBsdfResult) == 80, "ABI layout");
static_assert(sizeof(RtRequest) == 72, "ABI layout");
static_assert(sizeof(RtWorldDesc) == 184, "ABI layout");
static_assert(sizeof(RtCapture) == 64, "ABI layout");
static_assert(sizeof(RtSceneInfo) == 64, "ABI layout");
static_assert(sizeof(RtSceneOptions) == 32, "ABI layout");
static_assert(sizeof(RtMediumQuery) == 40, "ABI layout");
static_assert(sizeof(RtMediumResult) == 56, "ABI layout");

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
    float* film = nullptr;         // rt_render's device film, kept between calls
    size_t film_bytes = 0;
    int tuned = 0;                 // rt_autotune ran: use the fields below
    int tuned_slots = 0, tuned_block = 0, tuned_sort = 0, tuned_layout = 2, tuned_fetch = 1, tuned_tblock = 0, tuned_groups = 0;
    // Copy of the world description: rt_scene_set_params rebuilds from it.
    std::vector<RtMaterialDesc> w_materials;
    std::vector<RtEntityDesc> w_entities;
    std::vector<float> w_tris, w_normals, w_uvs;
    std::vector<RtLightDesc> w_lights;
    RtWorldDesc w{};
};

namespace {

// The bounce-ray sort's box: per axis the 1st to 99th percentile of the
// primitive centroids (triangles, quads, spheres), so that one large primitive
// such as a ground plane does not stretch the cells over empty space.
void ray_sort_box(const rt::HostScene& h, rt::SceneView& v) {
    std::vector<float> c[3];
    size_t ntri = h.tris.size() / 3;
    for (int k = 0; k < 3; k++) c[k].reserve(ntri + h.quads.size() + h.spheres.size());
    for (size_t i = 0; i < ntri; i++) {
        const float4 &p0 = h.tris[3 * i], &e1 = h.tris[3 * i + 1], &e2 = h.tris[3 * i + 2];
        c[0].push_back(p0.x + (e1.x + e2.x) / 3.0f);
        c[1].push_back(p0.y + (e1.y + e2.y) / 3.0f);
        c[2].push_back(p0.z + (e1.z + e2.z) / 3.0f);
    }
    for (const rt::QuadData& q : h.quads) {
        rt::V3 m = q.q + 0.5f * (q.u + q.v);
        c[0].push_back(m.x);
        c[1].push_back(m.y);
        c[2].push_back(m.z);
    }
    for (const rt::SphereData& sp : h.spheres) {
        c[0].push_back(sp.c.x);
        c[1].push_back(sp.c.y);
        c[2].push_back(sp.c.z);
    }
    float lo[3] = {0, 0, 0}, scale[3] = {0, 0, 0};
    for (int k = 0; k < 3; k++) {
        std::vector<float>& a = c[k];
        if (a.empty()) continue;
        size_t i0 = a.size() / 100, i1 = a.size() - 1 - a.size() / 100;
        std::nth_element(a.begin(), a.begin() + i0, a.end());
        float l = a[i0];
        std::nth_element(a.begin(), a.begin() + i1, a.end());
        float hgh = a[i1];
        lo[k] = l;
        scale[k] = hgh > l ? 1.0f / (hgh - l) : 0.0f;
    }
    v.sort_lo = rt::v3(lo[0], lo[1], lo[2]);
    v.sort_scale = rt::v3(scale[0], scale[1], scale[2]);
}

// `null_when_empty`: the kernels read a null pointer as "absent" (tri_smooth).
// The checked build gives every other array at least one zeroed element, so
// the index it substitutes for an out-of-range one can always be read.
template <typename T>
int upload(RtScene* sc, const std::vector<T>& v, const T** out, bool null_when_empty = false) {
#ifdef RT_CHECKED
    if (v.empty() && !null_when_empty) return upload(sc, std::vector<T>(1, T{}), out);
#endif
    if (v.empty()) {
        *out = nullptr;
        return RT_OK;
    }
    (void)null_when_empty;
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
    // The chunk's sum in double: a float sum of tens of thousands of samples
    // drifts by ~1e-3 of its value through the rounding of every addition.
    double sx = 0.0, sy = 0.0, sz = 0.0;
    rt::Counters cnt{{0u, 0u, 0u}, {0u, 0u, 0u}, 0u, 0u};
    for (int si = sb; si < se; si++) {
        V3 l = rt::trace_sample<STACK, COUNT>(s, rc, x0 + lx, y0 + ly, (uint32_t)(spp0 + si), &cnt, err);
        sx += l.x;
        sy += l.y;
        sz += l.z;
    }
    V3 sum = rt::v3((float)sx, (float)sy, (float)sz);
    if (COUNT) {
        atomicAdd(work + 0, (unsigned long long)cnt.closest.nodes);
        atomicAdd(work + 1, (unsigned long long)cnt.closest.tris);
        atomicAdd(work + 2, (unsigned long long)cnt.closest.others);
        atomicAdd(work + 3, (unsigned long long)cnt.closest_rays);
        atomicAdd(work + 4, (unsigned long long)cnt.shadow_rays);
        atomicAdd(work + 5, (unsigned long long)cnt.shadow.nodes);
        atomicAdd(work + 6, (unsigned long long)cnt.shadow.tris);
        atomicAdd(work + 7, (unsigned long long)cnt.shadow.others);
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

// Capturing megakernel (Renderer.Render with RenderCaptureOptions.Full): the
// megakernel plus the AOV probe and the even/odd sample halves of
// CaptureAccumulator (Renderer.cs:817-856). Per chunk and pixel it writes
// kCapSums partial sums, plane after plane: beauty, beauty A, beauty B,
// albedo A, albedo B, normal A, normal B (3 each), then depth A, depth B and
// the A and B depth counts.
constexpr int kCapSums = 25;
template <int STACK>
__global__ void __launch_bounds__(kBlock) k_render_capture(rt::SceneView s, rt::RenderConst rc, int ww, int wh,
                                                            int spp0, int per_chunk, int spp, float* partial,
                                                            int* err) {
    int lx = blockIdx.x * 16 + (threadIdx.x & 15);
    int ly = blockIdx.y * 8 + (threadIdx.x >> 4);
    int chunk = blockIdx.z;
    if (lx >= ww || ly >= wh) return;
    int sb = chunk * per_chunk;
    int se = min(sb + per_chunk, spp);
    V3 sum = rt::v3(0.0f), sa = rt::v3(0.0f), sbv = rt::v3(0.0f);
    V3 aa = rt::v3(0.0f), ab = rt::v3(0.0f), na = rt::v3(0.0f), nb = rt::v3(0.0f);
    float da = 0.0f, db = 0.0f, ca = 0.0f, cb = 0.0f;
    rt::AovProbe probe;
    for (int si = sb; si < se; si++) {
        V3 l = rt::trace_capture<STACK>(s, rc, lx, ly, (uint32_t)(spp0 + si), &probe, err);
        sum = sum + l;
        if ((si & 1) == 0) {   // A: even samples of the call
            sa = sa + l;
            aa = aa + probe.albedo;
            na = na + probe.normal;
            if (probe.have_depth) {
                da += probe.depth;
                ca += 1.0f;
            }
        } else {
            sbv = sbv + l;
            ab = ab + probe.albedo;
            nb = nb + probe.normal;
            if (probe.have_depth) {
                db += probe.depth;
                cb += 1.0f;
            }
        }
    }
    size_t plane = (size_t)ww * wh;
    float* out = partial + (size_t)chunk * kCapSums * plane + (size_t)ly * ww + lx;
    const V3 v[7] = {sum, sa, sbv, aa, ab, na, nb};
    for (int k = 0; k < 7; k++) {
        out[(3 * k) * plane] = v[k].x;
        out[(3 * k + 1) * plane] = v[k].y;
        out[(3 * k + 2) * plane] = v[k].z;
    }
    out[21 * plane] = da;
    out[22 * plane] = db;
    out[23 * plane] = ca;
    out[24 * plane] = cb;
}

// The capture's means (RenderBuffers: CaptureAccumulator.Store, Renderer.cs:
// 858-882): A holds ceil(n/2) samples, B floor(n/2), and B mirrors A when
// n == 1; a depth half with no hit is -1. Writes 23 planes: beauty, beauty A,
// beauty B, albedo A, albedo B, normal A, normal B (3 each), depth A, depth B.
__global__ void k_resolve_capture(const float* partial, int nchunks, int ww, int wh, int spp, float* outp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int plane = ww * wh;
    if (i >= plane) return;
    float acc[kCapSums];
    for (int k = 0; k < kCapSums; k++) {
        float a = partial[(size_t)k * plane + i];
        for (int c = 1; c < nchunks; c++) a += partial[(size_t)c * kCapSums * plane + (size_t)k * plane + i];
        acc[k] = a;
    }
    int n_a = (spp + 1) / 2, n_b = spp / 2;
    auto put = [&](int p, float x) { outp[(size_t)p * plane + i] = x; };
    for (int c = 0; c < 3; c++) {
        put(c, acc[c] / (float)spp);   // cumulativeColor / actualSamples
        for (int q = 0; q < 3; q++) {  // beauty, albedo, normal halves
            float ma = acc[3 + 6 * q + c] / (float)n_a;
            float mb = n_b > 0 ? acc[6 + 6 * q + c] / (float)n_b : ma;
            put(3 + 6 * q + c, ma);
            put(6 + 6 * q + c, mb);
        }
    }
    float dA = acc[23] > 0.0f ? acc[21] / acc[23] : -1.0f;
    float dB = n_b > 0 ? (acc[24] > 0.0f ? acc[22] / acc[24] : -1.0f) : dA;
    put(21, dA);
    put(22, dB);
}

// Path-replay adjoint: one thread per (pixel, sample) work item, samples
// outermost, grid-stride. Gradients gather per thread (when the parameter
// vector fits kAdjLocal) or in shared memory per block, and go to the global
// double accumulators once per block.
struct AdjArgs {
    int x0, y0, ww, wh, W, H, spp, spp0;
    const float* dimg;     // 3*H*W planar dLoss/dfilm
    const float* params;   // raw parameter vector
    const unsigned* mmask; // per material slot masks
    unsigned gmask;        // global slot mask
    double* grad;          // accumulators, nparams
    int nparams;
    int medium_base;
    int use_shared;
    int use_local;
    int any4;              // opaque shadow rays may walk the four-wide records
};

// Build knobs of the adjoint kernel: a register cap (0: the compiler's
// choice) and whether gradients may gather in per-thread local arrays (1) or
// always in shared memory (0).
#ifndef RT_ADJ_MAX_REGS
#define RT_ADJ_MAX_REGS 0
#endif
#ifndef RT_ADJ_LOCAL_ACC
#define RT_ADJ_LOCAL_ACC 1
#endif
#if RT_ADJ_MAX_REGS > 0
#define RT_ADJ_BOUNDS __maxnreg__(RT_ADJ_MAX_REGS)
#else
#define RT_ADJ_BOUNDS __launch_bounds__(kBlock)
#endif

template <int STACK>
__global__ void RT_ADJ_BOUNDS k_adjoint(rt::SceneView s, rt::RenderConst rc, AdjArgs a, int* err) {
    extern __shared__ float sacc[];
    if (a.use_shared)
        for (int i = threadIdx.x; i < a.nparams; i += blockDim.x) sacc[i] = 0.0f;
    __syncthreads();
    float loc[rt::kAdjLocal];
    if (a.use_local)
        for (int i = 0; i < a.nparams; i++) loc[i] = 0.0f;
    long long npix = (long long)a.ww * a.wh;
    long long total = npix * a.spp;
    size_t plane = (size_t)a.W * a.H;
    float inv_spp = 1.0f / (float)a.spp;
    // The loops run warp-synchronously: every loop of the 32 lanes continues
    // while any lane has work and re-converges at its head, so the lanes walk
    // the primal and the replay (two large code regions) together instead of
    // each lane drifting into a different phase, which left 3 of 32 lanes
    // active per instruction and the warps waiting on instruction fetch.
    const unsigned full = 0xffffffffu;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;; idx += stride) {
        bool has = idx < total;
        if (!__any_sync(full, has)) break;
        int pix = has ? (int)(idx % npix) : 0;
        int si = has ? (int)(idx / npix) : 0;
        int px = a.x0 + pix % a.ww, py = a.y0 + pix / a.ww;
        size_t fi = (size_t)py * a.W + px;
        V3 delta = rt::v3(0.0f);
        if (has) delta = rt::v3(a.dimg[fi], a.dimg[plane + fi], a.dimg[2 * plane + fi]) * inv_spp;
        bool work = has && !rt::is_zero(delta);
        uint32_t sidx = (uint32_t)(a.spp0 + si);
        // primal pass (its own state: the replay's is read by the hooks)
        rt::PathState pp;
        rt::path_init(pp, rc, px, py, sidx);
        rt::InlineShadows<STACK> fwd{{}, &s, rc.opaque, nullptr, err};
        bool alive = work && rt::path_alive(pp);
        while (__any_sync(full, alive)) {
            if (alive) {
                rt::Hit h;
                rt::traverse<false, STACK>(s, pp.o, pp.d, rt::kEps, rt::kInf, h, nullptr, err);
                alive = rt::shade_vertex(s, rc, pp, h, fwd);
            }
        }
        // adjoints of the resolve (path_resolve)
        rt::AdjointReplay<STACK> adj;
        adj.s = &s;
        adj.params = a.params;
        adj.mmask = a.mmask;
        adj.gmask = a.gmask;
        adj.loc = a.use_local ? loc : nullptr;
        adj.acc = a.use_shared ? sacc : nullptr;
        adj.gacc = a.grad;
        adj.medium_base = a.medium_base;
        adj.opaque = rc.opaque;
        adj.any4 = a.any4;
        adj.err = err;
        adj.abs_mat = -1;
        adj.max_rad = rc.max_rad;
        adj.ind_max = rc.ind_max;
        adj.clear_log_beta();
        adj.sh_added = 0;
        adj.sh_n = 0;
        adj.set_resolve(rt::adjoint_resolve(rc, pp.lp, pp.la, pp.pre, pp.att0, pp.clamp_mode, delta));
        // replay
        rt::PathState ps;
        rt::path_init(ps, rc, px, py, sidx);
        alive = work && !rt::is_zero(adj.g_a) && rt::path_alive(ps);
        while (__any_sync(full, alive)) {
            if (alive) {
                rt::Hit h;
                rt::traverse<false, STACK>(s, ps.o, ps.d, rt::kEps, rt::kInf, h, nullptr, err);
                alive = rt::shade_vertex(s, rc, ps, h, adj);
            }
        }
    }
    if (a.use_local) {   // warp sums of the per-thread accumulators
        int lane = threadIdx.x & 31;
        for (int i = 0; i < a.nparams; i++) {
            float v = loc[i];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0 && v != 0.0f) {
                if (a.use_shared) atomicAdd(sacc + i, v);
                else atomicAdd(a.grad + i, (double)v);
            }
        }
    }
    __syncthreads();
    if (a.use_shared)
        for (int i = threadIdx.x; i < a.nparams; i += blockDim.x)
            if (sacc[i] != 0.0f) atomicAdd(a.grad + i, (double)sacc[i]);
}

template <int STACK, bool L4>
__global__ void k_trace_closest(rt::SceneView s, const float* rays, int64_t n, float tmin, float tmax, int* hits,
                                int* err) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + i * 8;
    V3 o = rt::v3(r[0], r[1], r[2]), d = rt::v3(r[3], r[4], r[5]);
    rt::Hit h;
    rt::trace<false, STACK, L4>(s, o, d, tmin, tmax, h, nullptr, err);
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

template <int STACK, bool L4>
__global__ void k_trace_any(rt::SceneView s, int opaque, const float* rays, int64_t n, float* out, int* err) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + i * 8;
    V3 t = rt::shadow_transmittance<STACK, L4>(s, opaque, rt::v3(r[0], r[1], r[2]), rt::v3(r[3], r[4], r[5]), r[6],
                                               r[7], nullptr, err);
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
        r.transition = bs.transition;
    }
    out[i] = r;
}

// Medium batch: HomogeneousMedium.Sample over [0, tmax], then
// HenyeyGreensteinPhase.Sample(wo), on one Sobol stream per query, with
// Transmittance(tmax) and Evaluate(wo, wi) beside them.
__global__ void k_medium(rt::SceneView s, const RtMediumQuery* q, int64_t n, RtMediumResult* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    RtMediumQuery qq = q[i];
    RtMediumResult r;
    memset(&r, 0, sizeof(r));
    V3 wo = rt::v3(qq.wo[0], qq.wo[1], qq.wo[2]);
    V3 wi = rt::v3(qq.wi[0], qq.wi[1], qq.wi[2]);
    rt::Sampler rng{qq.pixel_seed, qq.sample_index, qq.dim};
    float t = 0.0f;
    V3 beta;
    r.scattered = rt::medium_sample(s, qq.tmax, rng, t, beta) ? 1 : 0;
    r.t = t;
    r.beta[0] = beta.x; r.beta[1] = beta.y; r.beta[2] = beta.z;
    float pdf = 0.0f;
    V3 d = rt::hg_sample(s.hg_g, wo, rng, pdf);
    r.phase_wi[0] = d.x; r.phase_wi[1] = d.y; r.phase_wi[2] = d.z;
    r.phase_pdf = pdf;
    r.dims_used = rng.dim - qq.dim;
    V3 tr = rt::medium_tr(s, qq.tmax);
    r.tr[0] = tr.x; r.tr[1] = tr.y; r.tr[2] = tr.z;
    r.phase_eval = rt::hg_eval(s.hg_g, wo, wi);
    out[i] = r;
}

// AcesToneMap (Renderer.cs:893-907) after the exposure gain, planar HDR in,
// interleaved display RGB out.
__global__ void k_tonemap(const float* hdr, int npix, float scale, float* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    for (int c = 0; c < 3; c++) {
        float x = fmaxf(hdr[(size_t)c * npix + i] * scale, 0.0f);
        float a = x * (2.51f * x + 0.03f);
        float b = x * (2.43f * x + 0.59f) + 0.14f;
        float m = rt::clampf(a / b, 0.0f, 1.0f);
        out[(size_t)i * 3 + c] = powf(m, 1.0f / 2.2f);
    }
}

__global__ void k_sobol(const uint32_t* idx, const uint32_t* dim, const uint32_t* seed, int64_t n, float* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = rt::sobol_sample(idx[i], dim[i], seed[i]);
}

// The checked build's out-of-range flag (one per device, shared by every
// scene): read and cleared once the stream's work is done.
int checked_flag(cudaStream_t stream) {
#ifdef RT_CHECKED
    int flag = 0, zero = 0;
    CUDA_TRY(cudaMemcpyFromSymbolAsync(&flag, rt::g_bounds_flag, sizeof(int), 0, cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaMemcpyToSymbolAsync(rt::g_bounds_flag, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    if (flag) return fail(RT_ERR_BOUNDS, "checked build: a kernel met an index out of its array's range");
#else
    (void)stream;
#endif
    return RT_OK;
}

int check_err(RtScene* sc) {
    int e = 0;
    CUDA_TRY(cudaMemcpyAsync(&e, sc->d_err, sizeof(int), cudaMemcpyDeviceToHost, sc->stream));
    CUDA_TRY(cudaStreamSynchronize(sc->stream));
    if (e == RT_ERR_STACK) return fail(RT_ERR_STACK, "traversal stack bound exceeded");
    if (e != 0) return fail(RT_ERR_BOUNDS, "device error " + std::to_string(e));
    return checked_flag(sc->stream);
}

int validate_params(const RtScene* sc, const RtRenderParams* p) {
    if (!p) return fail(RT_ERR_INVALID_ARG, "null params");
    if (p->width <= 0 || p->height <= 0 || p->spp <= 0 || p->max_depth < 0)
        return fail(RT_ERR_INVALID_ARG, "width, height and spp must be positive, max_depth non-negative");
    if ((int64_t)p->width * p->height > (int64_t)1 << 28) return fail(RT_ERR_INVALID_ARG, "image too large");
    if (p->light_strategy < RT_LIGHTS_ALL || p->light_strategy > RT_LIGHTS_UNIFORM)
        return fail(RT_ERR_INVALID_ARG, "unknown light strategy");
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
    rc.light_pick = p->light_strategy;
    return rc;
}

// Renders into a device film (3*W*H, planar). Caller holds sc->mu.
int wf_render_one(RtScene* sc, const RtRenderParams* p, const RtCameraDesc& cam, float* d_film, RtStats* st);

int render_to_device(RtScene* sc, const RtRenderParams* p, const RtCameraDesc& cam, float* d_film, RtStats* st) {
    auto t0 = std::chrono::steady_clock::now();
    int rc_ = validate_params(sc, p);
    if (rc_ != RT_OK) return rc_;
    CUDA_TRY(cudaSetDevice(sc->device));
    if (p->kernel == RT_KERNEL_WAVEFRONT && !p->count_work) return wf_render_one(sc, p, cam, d_film, st);
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
            st->shadow_node_visits = w[5];
            st->shadow_prim_tests = w[6];
            st->shadow_other_tests = w[7];
        }
        st->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return RT_OK;
}


// ---------------------------------------------------------------------------
// Wavefront host driver
// ---------------------------------------------------------------------------
struct HostReq {
    RtScene* scene;
    rt::RenderConst rc;
    int x0, y0, ww, wh, spp, spp0;
    int W, H;
    float* d_film;
};

struct WfWorkspace {
    void* mem = nullptr;
    size_t bytes = 0;
    unsigned long long* pinned = nullptr;   // two read-back slots of {next, live | overflow}
    cudaEvent_t polled[2] = {nullptr, nullptr};   // each slot's read-back has landed
    // The last instantiated iteration graph and the kernel arguments and launch
    // shapes it was captured with: a repeated render of the same configuration
    // replays it instead of capturing and instantiating a new one.
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> exec_key;
};
std::mutex g_wf_mu;
WfWorkspace g_wf_ws[16];

struct Carve {
    char* base;
    size_t off = 0;
    template <typename T>
    T* take(size_t n) {
        off = (off + 255) & ~(size_t)255;
        T* p = reinterpret_cast<T*>(base + off);
        off += n * sizeof(T);
        return p;
    }
};

// Autotuned (wavefront size, block size, sort) per scene set, kept for the
// process lifetime; filled by rt_autotune or the defaults below.
struct WfConfig {
    int slots = 1 << 22;
    int block = 256;
    int sort = 1;
    int profile = 0;   // per-kernel events instead of the graph
    int layout = 2;    // BVH records of extend/occlude: 2 or 4 wide
    int fetch = 1;     // 1 one ray per thread, 2 persistent warps with dynamic fetch (two-wide only)
    int tblock = 0;    // block of extend/occlude (0: block)
    int groups = 0;    // 1 slot order, 2 block-local regrouping, 3 sorted bounce rays, 4 and shadow rays; 0 default_groups
    int iter_limit = 0;     // test only: > 0 caps the iterations below the host's bound
    int shadow_limit = 0;   // test only: > 0 caps the shadow queue's records
};

// The test-only limits of a render request (0: none).
void apply_test_limits(WfConfig& cfg, const RtRenderParams* p) {
    cfg.iter_limit = std::max(0, p->iteration_limit);
    cfg.shadow_limit = std::max(0, p->shadow_queue_limit);
}

// Untuned ray order: bounce and shadow rays sorted, except with a
// participating medium. There nearly every slot is a bounce ray scattered in
// mid-air and the scene is small, so the sorts' keys and ranks in shade cost
// more than the coherence wins back (measured, bounce rays sorted: icosphere
// field +12%, Cornell box +12%, mixed batch +10%, the medium scene -3%; shadow
// rays sorted as well: a further +3%, +1% and -3%).
int default_groups(const std::vector<RtScene*>& scenes) {
    for (const RtScene* sc : scenes)
        if (sc->host.has_medium) return 1;
    return 4;
}

// mode: rt::WF_RENDER renders the requests into their films; rt::WF_RECORD
// and rt::WF_REPLAY are the two passes of the wavefront adjoint over the same
// requests, with adj holding their buffers (rt_adjoint).
int wf_render(const std::vector<HostReq>& reqs, const WfConfig& cfg, RtStats* st, int mode = rt::WF_RENDER,
              const rt::WfAdjoint* adj = nullptr) {
    auto t0 = std::chrono::steady_clock::now();
    if (reqs.empty()) return RT_OK;
    if (mode != rt::WF_RENDER && !adj) return fail(RT_ERR_INVALID_ARG, "adjoint pass without its buffers");
    std::lock_guard<std::mutex> lk(g_wf_mu);
    RtScene* s0 = reqs[0].scene;
    int dev = s0->device;
    CUDA_TRY(cudaSetDevice(dev));
    if (dev < 0 || dev >= 16) return fail(RT_ERR_INVALID_ARG, "device index out of range");
    cudaStream_t stream = s0->stream;
    // Distinct scenes of the batch, material key bases, limits.
    std::vector<RtScene*> scenes;
    std::vector<int> req_scene(reqs.size());
    for (size_t r = 0; r < reqs.size(); r++) {
        auto it = std::find(scenes.begin(), scenes.end(), reqs[r].scene);
        if (it == scenes.end()) {
            scenes.push_back(reqs[r].scene);
            req_scene[r] = (int)scenes.size() - 1;
        } else {
            req_scene[r] = (int)(it - scenes.begin());
        }
        if (reqs[r].scene->device != dev) return fail(RT_ERR_INVALID_ARG, "batch scenes live on different devices");
        if (reqs[r].scene->host.max_stack > kStack) return fail(RT_ERR_STACK, "scene stack bound exceeded");
    }
    std::vector<rt::SceneView> views;
    std::vector<int> key_base;
    int nkeys = 0, max_shadow = 1, opaque = 1, dielectrics = 0;
    for (RtScene* sc : scenes) {
        views.push_back(sc->view);
        key_base.push_back(nkeys);
        nkeys += (int)sc->host.materials.size();
        int sh = 0;
        for (const rt::Light& l : sc->host.lights) sh += l.shadow_samples;
        max_shadow = std::max(max_shadow, sh);
        opaque &= sc->opaque;
        dielectrics |= sc->dielectrics;
    }
    int sort = cfg.sort && nkeys < 255;
    int64_t total = 0;
    std::vector<rt::WfRequest> wreq(reqs.size());
    for (size_t r = 0; r < reqs.size(); r++) {
        rt::WfRequest& q = wreq[r];
        q.rc = reqs[r].rc;
        q.rc.opaque = opaque;
        q.rc.dielectrics = dielectrics;
        q.scene = req_scene[r];
        q.x0 = reqs[r].x0;
        q.y0 = reqs[r].y0;
        q.ww = reqs[r].ww;
        q.wh = reqs[r].wh;
        q.spp = reqs[r].spp;
        q.spp0 = reqs[r].spp0;
        q.begin = total;
        q.count = (long long)q.ww * q.wh * q.spp;
        total += q.count;
        if (q.ww >= 65536 || q.wh >= 32768) return fail(RT_ERR_INVALID_ARG, "render window too large");
    }
    int nslots = (int)std::max<int64_t>(1024, std::min<int64_t>(cfg.slots, total));
    nslots = (nslots + 255) / 256 * 256;
    int64_t cap = (int64_t)nslots * max_shadow;
    if (cap >= ((int64_t)1 << 31) || nslots >= (1 << 29)) return fail(RT_ERR_INVALID_ARG, "wavefront too large");
    if (cfg.shadow_limit > 0) cap = std::min<int64_t>(cap, cfg.shadow_limit);
    // Workspace layout.
    size_t need = 0;
    auto add = [&](size_t b) { need = ((need + 255) & ~(size_t)255) + b; };
    add(views.size() * sizeof(rt::SceneView));
    add(wreq.size() * sizeof(rt::WfRequest));
    add(key_base.size() * sizeof(int));
    add(sizeof(rt::WfCtl));
    for (int k = 0; k < 9; k++) add((size_t)nslots * sizeof(float4));
    add((size_t)nslots * sizeof(int));
    add((size_t)nslots * sizeof(int));
    add((size_t)nslots * sizeof(int));
    if (dielectrics) {
        add((size_t)nslots * sizeof(float4));
        add((size_t)nslots * 8 * sizeof(float));
    }
    for (int k = 0; k < 3; k++) add((size_t)cap * sizeof(float4));
    add(sizeof(int));
    for (int k = 0; k < 3; k++) add((size_t)cap * sizeof(int));
    for (int k = 0; k < 4; k++) add((size_t)rt::kRayKeys * sizeof(int));
    for (auto& q : wreq) add((size_t)3 * q.ww * q.wh * sizeof(double));
    add(reqs.size() * sizeof(float*));
    add(reqs.size() * sizeof(int) * 2);
    if (mode == rt::WF_REPLAY) add((size_t)nslots * rt::kAdjState * sizeof(float4));
    need += 1024;
    WfWorkspace& ws = g_wf_ws[dev];
    if (ws.bytes < need) {
        if (ws.exec) cudaGraphExecDestroy(ws.exec);   // captured with pointers into the old workspace
        ws.exec = nullptr;
        ws.exec_key.clear();
        if (ws.mem) cudaFree(ws.mem);
        ws.mem = nullptr;
        ws.bytes = 0;
        if (cudaMalloc(&ws.mem, need) != cudaSuccess) return fail(RT_ERR_OOM, "wavefront workspace allocation failed");
        ws.bytes = need;
    }
    if (!ws.pinned && cudaMallocHost(&ws.pinned, 4 * sizeof(unsigned long long)) != cudaSuccess)
        return fail(RT_ERR_OOM, "pinned read-back allocation failed");
    for (cudaEvent_t& e : ws.polled)
        if (!e && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return fail(RT_ERR_CUDA, "event creation failed");
    Carve cv{static_cast<char*>(ws.mem)};
    rt::WfArgs a;
    std::memset(&a, 0, sizeof(a));   // padding too: the bytes key the cached graph
    auto* d_views = cv.take<rt::SceneView>(views.size());
    auto* d_reqs = cv.take<rt::WfRequest>(wreq.size());
    auto* d_kb = cv.take<int>(key_base.size());
    auto* d_ctl = cv.take<rt::WfCtl>(1);
    a.P.o = cv.take<float4>(nslots);
    a.P.d = cv.take<float4>(nslots);
    a.P.beta = cv.take<float4>(nslots);
    a.P.w = cv.take<float4>(nslots);
    a.P.lp = cv.take<float4>(nslots);
    a.P.la = cv.take<float4>(nslots);
    a.P.pre = cv.take<float4>(nslots);
    a.P.att0 = cv.take<float4>(nslots);
    a.P.hit = cv.take<float4>(nslots);
    a.P.order = cv.take<int>(nslots);
    a.P.keys = cv.take<int>(nslots);
    a.P.rrank = cv.take<int>(nslots);
    if (dielectrics) {
        a.P.ab = cv.take<float4>(nslots);
        a.P.ior = cv.take<float>((size_t)nslots * 8);
    }
    a.S.o = cv.take<float4>(cap);
    a.S.d = cv.take<float4>(cap);
    a.S.c = cv.take<float4>(cap);
    a.S.count = cv.take<int>(1);
    a.S.capacity = (int)cap;
    a.S.key = cv.take<int>(cap);
    a.S.rank = cv.take<int>(cap);
    a.S.order = cv.take<int>(cap);
    a.rhist = cv.take<int>(rt::kRayKeys);
    a.roff = cv.take<int>(rt::kRayKeys);
    a.shist = cv.take<int>(rt::kRayKeys);
    a.soff = cv.take<int>(rt::kRayKeys);
    std::vector<float*> films(reqs.size());
    std::vector<int> fdims(2 * reqs.size());
    for (size_t r = 0; r < reqs.size(); r++) {
        wreq[r].accum = cv.take<double>((size_t)3 * wreq[r].ww * wreq[r].wh);
        films[r] = reqs[r].d_film;
        fdims[r] = reqs[r].W;
        fdims[reqs.size() + r] = reqs[r].H;
    }
    auto* d_films = cv.take<float*>(reqs.size());
    auto* d_fdims = cv.take<int>(2 * reqs.size());
    if (adj) a.J = *adj;
    if (mode == rt::WF_REPLAY) a.J.st = cv.take<float4>((size_t)nslots * rt::kAdjState);
    a.views = d_views;
    a.nviews = (int)views.size();
    a.reqs = d_reqs;
    a.nreq = (int)wreq.size();
    a.nslots = nslots;
    a.opaque = opaque;
    a.sort = sort;
    a.nkeys = nkeys;
    a.key_base = d_kb;
    a.ctl = d_ctl;
    a.err = s0->d_err;
    rt::WfCtl ctl0{};
    ctl0.total = (unsigned long long)total;
    CUDA_TRY(cudaMemcpyAsync(d_views, views.data(), views.size() * sizeof(rt::SceneView), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(d_reqs, wreq.data(), wreq.size() * sizeof(rt::WfRequest), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(d_kb, key_base.data(), key_base.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(d_ctl, &ctl0, sizeof(ctl0), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(d_films, films.data(), films.size() * sizeof(float*), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(d_fdims, fdims.data(), fdims.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemsetAsync(a.P.d, 0, (size_t)nslots * sizeof(float4), stream));
    CUDA_TRY(cudaMemsetAsync(a.S.count, 0, sizeof(int), stream));
    for (int* h : {a.rhist, a.roff, a.shist, a.soff})
        CUDA_TRY(cudaMemsetAsync(h, 0, (size_t)rt::kRayKeys * sizeof(int), stream));
    for (auto& q : wreq) CUDA_TRY(cudaMemsetAsync(q.accum, 0, (size_t)3 * q.ww * q.wh * sizeof(double), stream));
    CUDA_TRY(cudaMemsetAsync(s0->d_err, 0, sizeof(int), stream));
    CUDA_TRY(cudaStreamSynchronize(stream));   // host vectors above go out of scope
    // One iteration: reset, regen, extend, [scan, scatter], shade, occlude.
    int blk = cfg.block;
    int tblk = cfg.tblock > 0 ? cfg.tblock : blk;
    bool l4 = cfg.layout == 4;
    for (const HostReq& q : reqs) l4 = l4 && q.scene->host.max_stack4 <= kStack;
    bool pt = !l4 && cfg.fetch == 2;
    // Opaque shadow rays walk the four-wide records in any order whenever the
    // scenes' four-wide stack bound fits: a shadow ray's answer does not
    // depend on the visit order (per 64-spp icosphere frame: occlude 49.4 ms
    // against 51.8 ms on the two-wide records, extend unchanged).
    bool l4_occ = l4;
    if (opaque && !pt) {
        l4_occ = true;
        for (const HostReq& q : reqs) l4_occ = l4_occ && q.scene->host.max_stack4 <= kStack;
    }
    a.any4 = l4_occ && opaque;
    int groups = cfg.groups > 0 ? cfg.groups : default_groups(scenes);
    // shade is compiled with the volumetric branch and the transmission lobe
    // only when a scene of the batch needs them
    bool medium = false;
    for (const RtScene* sc : scenes) medium = medium || sc->host.has_medium;
    const bool transmit = !a.opaque;
    a.regroup = groups == 2;
    a.raysort = groups >= 3 && !pt;
    a.shadowsort = groups == 4 && !pt && mode != rt::WF_REPLAY;   // the replay queues no shadow rays
    // 8x8x8 origin cells x 8x8 direction bins: the measured best of the
    // layouts that fit 15 bits (coarser cells or octant-only directions cost
    // extend 4-13% on the icosphere field)
    a.rkey_bits = 3;
    a.rdir_bits = 6;
    // Shadow records toward one light share their directions, so their key
    // spends the bits on the origin: 16x16x16 cells x direction octant
    // (per 64-spp icosphere frame against the bounce-ray layout: occlude
    // -2.4%, frame -0.6 to -1.8%; 4x4x4 cells x 16x16 directions lost 0.5%,
    // 16x16x16 cells without direction bits 1.8%)
    a.skey_bits = 4;
    a.sdir_bits = 3;
    unsigned gpt_e = 1, gpt_o = 1;
    if (pt) {
        int sms = 148, nb_e = 1, nb_o = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb_e, rt::k_wf_extend_pt<kStack>, tblk, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb_o, rt::k_wf_occlude_pt<kStack>, tblk, 0);
        gpt_e = (unsigned)std::max(1, nb_e * sms);
        gpt_o = (unsigned)std::max(1, nb_o * sms);
    }
    const int adj_blk = 128;
    unsigned gadj = (unsigned)((nslots + adj_blk - 1) / adj_blk);
    size_t adj_shmem = 0;
    if (mode == rt::WF_REPLAY)
        adj_shmem = (size_t)(a.J.use_local ? a.J.nact : (a.J.use_shared ? a.J.nparams : 0)) * sizeof(float);
    unsigned gs = (unsigned)((nslots + blk - 1) / blk);
    unsigned gst = (unsigned)((nslots + tblk - 1) / tblk);
    unsigned gsh = (unsigned)((cap + tblk - 1) / tblk);
    unsigned g256 = (unsigned)((nslots + 255) / 256);
    unsigned gsh256 = (unsigned)((cap + 255) / 256);
    // ev (profiling only): boundaries between the kernel groups of one iteration.
    auto launch_iter = [&](cudaEvent_t* ev) {
        if (ev) cudaEventRecord(ev[0], stream);
        rt::k_wf_reset<<<1, 256, 0, stream>>>(a);
        if (mode == rt::WF_RECORD) rt::k_wf_regen<rt::WF_RECORD><<<g256, 256, 0, stream>>>(a);
        else if (mode == rt::WF_REPLAY) rt::k_wf_regen<rt::WF_REPLAY><<<g256, 256, 0, stream>>>(a);
        else rt::k_wf_regen<rt::WF_RENDER><<<g256, 256, 0, stream>>>(a);
        if (ev) cudaEventRecord(ev[1], stream);
        if (l4) rt::k_wf_extend<kStack, true><<<gst, tblk, 0, stream>>>(a);
        else if (pt) rt::k_wf_extend_pt<kStack><<<gpt_e, tblk, 0, stream>>>(a);
        else rt::k_wf_extend<kStack, false><<<gst, tblk, 0, stream>>>(a);
        if (ev) cudaEventRecord(ev[2], stream);
        if (sort) {
            rt::k_wf_scan<<<1, 256, 0, stream>>>(a);
            rt::k_wf_scatter<<<g256, 256, 0, stream>>>(a);
        }
        if (ev) cudaEventRecord(ev[3], stream);
        if (mode == rt::WF_REPLAY) {   // the adjoint vertex, shadow rays inline: no occlude
            if (medium && transmit) rt::k_wf_adjoint<kStack, true, true><<<gadj, adj_blk, adj_shmem, stream>>>(a);
            else if (medium) rt::k_wf_adjoint<kStack, true, false><<<gadj, adj_blk, adj_shmem, stream>>>(a);
            else if (transmit) rt::k_wf_adjoint<kStack, false, true><<<gadj, adj_blk, adj_shmem, stream>>>(a);
            else rt::k_wf_adjoint<kStack, false, false><<<gadj, adj_blk, adj_shmem, stream>>>(a);
            if (ev) cudaEventRecord(ev[4], stream);
            if (a.raysort) rt::k_wf_rscan<<<1, 1024, 0, stream>>>(a.rhist, a.roff, &d_ctl->nbounce);
            if (ev) {
                cudaEventRecord(ev[5], stream);
                cudaEventRecord(ev[6], stream);
            }
            return;
        }
        if (medium && transmit) rt::k_wf_shade<true, true><<<gs, blk, 0, stream>>>(a);
        else if (medium) rt::k_wf_shade<true, false><<<gs, blk, 0, stream>>>(a);
        else if (transmit) rt::k_wf_shade<false, true><<<gs, blk, 0, stream>>>(a);
        else rt::k_wf_shade<false, false><<<gs, blk, 0, stream>>>(a);
        if (ev) cudaEventRecord(ev[4], stream);   // the ray sorts' scans and scatter count as sorting
        if (a.raysort) rt::k_wf_rscan<<<1, 1024, 0, stream>>>(a.rhist, a.roff, &d_ctl->nbounce);
        if (a.shadowsort) {
            rt::k_wf_rscan<<<1, 1024, 0, stream>>>(a.shist, a.soff, &d_ctl->nshadow);
            rt::k_wf_sscatter<<<gsh256, 256, 0, stream>>>(a);
        }
        if (ev) cudaEventRecord(ev[5], stream);
        if (l4_occ && a.opaque) rt::k_wf_occlude<kStack, true, true><<<gsh, tblk, 0, stream>>>(a);
        else if (l4) rt::k_wf_occlude<kStack, true, false><<<gsh, tblk, 0, stream>>>(a);
        else if (pt && a.opaque) rt::k_wf_occlude_pt<kStack><<<gpt_o, tblk, 0, stream>>>(a);
        else if (a.opaque) rt::k_wf_occlude<kStack, false, true><<<gsh, tblk, 0, stream>>>(a);
        else rt::k_wf_occlude<kStack, false, false><<<gsh, tblk, 0, stream>>>(a);
        if (ev) cudaEventRecord(ev[6], stream);
    };
    constexpr int kEv = 7;   // profiling events per iteration
    const int batch = 4;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaEvent_t> pev;
    if (cfg.profile) {
        pev.resize(batch * kEv);
        for (auto& e : pev)
            if (cudaEventCreate(&e) != cudaSuccess) return fail(RT_ERR_CUDA, "event creation failed");
    } else {
        // The graph is a function of the kernels' arguments and launch shapes
        // alone (everything else it reads lives in the workspace), so those
        // bytes key the cached one.
        const unsigned shape[] = {(unsigned)blk, (unsigned)tblk, (unsigned)l4, (unsigned)l4_occ, (unsigned)pt,
                                  (unsigned)medium, (unsigned)transmit, gpt_e, gpt_o, gs, gst, gsh, g256, gsh256,
                                  (unsigned)mode, gadj, (unsigned)adj_shmem};
        std::vector<unsigned char> key(sizeof(a) + sizeof(shape));
        std::memcpy(key.data(), &a, sizeof(a));
        std::memcpy(key.data() + sizeof(a), shape, sizeof(shape));
        if (ws.exec && ws.exec_key == key) {
            exec = ws.exec;
        } else {
            if (ws.exec) cudaGraphExecDestroy(ws.exec);
            ws.exec = nullptr;
            ws.exec_key.clear();
            cudaGraph_t graph = nullptr;
            CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            launch_iter(nullptr);
            cudaError_t ce = cudaStreamEndCapture(stream, &graph);
            if (ce != cudaSuccess) return fail(RT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
            ce = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);   // the executable graph does not need it
            if (ce != cudaSuccess) return fail(RT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
            ws.exec = exec;
            ws.exec_key = std::move(key);
        }
    }
    int per_iter = (mode == rt::WF_REPLAY ? 4 : 5) + (sort ? 2 : 0) + (a.raysort ? 1 : 0) + (a.shadowsort ? 2 : 0);
    int max_depth = 1;
    for (auto& q : wreq) max_depth = std::max(max_depth, q.rc.max_depth);
    int64_t limit = (total / nslots + 2) * (int64_t)(max_depth + 2) + 64;
    if (cfg.iter_limit > 0) limit = std::min<int64_t>(limit, cfg.iter_limit);
    int64_t iters = 0;
    double t_regen = 0, t_extend = 0, t_sort = 0, t_shade = 0, t_occlude = 0;
    int rc = RT_OK;
    // The poll is pipelined: batch k+1 is queued before the host waits for
    // batch k's read-back, so the device does not idle while the host turns
    // around. Replays after the wavefront has drained find no work and write
    // nothing (the polled batches already ran up to batch-1 of them).
    // Profiling waits for each batch itself, so its events are read before the
    // next batch records them again.
    int cur = 0, waiting = -1;
    CUDA_TRY(cudaEventRecord(s0->ev0, stream));
    for (;;) {
        for (int k = 0; k < batch; k++) {
            if (cfg.profile) {
                launch_iter(&pev[k * kEv]);
            } else if (cudaGraphLaunch(exec, stream) != cudaSuccess) {
                rc = fail(RT_ERR_CUDA, "graph launch failed");
                break;
            }
        }
        if (rc != RT_OK) break;
        iters += batch;
        unsigned long long* slot = ws.pinned + 2 * cur;
        cudaMemcpyAsync(slot, &d_ctl->next, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(slot + 1, &d_ctl->live, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream);
        cudaEventRecord(ws.polled[cur], stream);
        int check = cur;
        if (!cfg.profile) {
            check = waiting;
            waiting = cur;
            cur ^= 1;
            if (check < 0) continue;   // first batch: queue the second before waiting
        }
        if (cudaEventSynchronize(ws.polled[check]) != cudaSuccess) {
            rc = fail(RT_ERR_CUDA, std::string("wavefront iteration failed: ") + cudaGetErrorString(cudaGetLastError()));
            break;
        }
        if (cfg.profile) {
            for (int k = 0; k < batch; k++) {
                float m[kEv - 1];
                for (int e = 0; e < kEv - 1; e++)
                    cudaEventElapsedTime(&m[e], pev[k * kEv + e], pev[k * kEv + e + 1]);
                t_regen += m[0];
                t_extend += m[1];
                t_sort += m[2] + m[4];   // the material sort, then the ray sorts' scans and scatter
                t_shade += m[3];
                t_occlude += m[5];
            }
        }
        unsigned long long next = ws.pinned[2 * check];
        int live = reinterpret_cast<int*>(ws.pinned + 2 * check + 1)[0];
        int overflow = reinterpret_cast<int*>(ws.pinned + 2 * check + 1)[1];
        if (overflow) {
            rc = fail(RT_ERR_BOUNDS, "shadow queue overflow");
            break;
        }
        if (next >= (unsigned long long)total && live == 0) break;
        if (iters > limit) {
            rc = fail(RT_ERR_TIMEOUT, "wavefront did not drain within its iteration bound");
            break;
        }
    }
    if (rc == RT_OK) {
        dim3 g(std::max<unsigned>(1, std::min<unsigned>(4096, (unsigned)((wreq[0].ww * (int64_t)wreq[0].wh + 255) / 256))),
               (unsigned)wreq.size());
        if (mode == rt::WF_RENDER)
            rt::k_wf_finalize<<<g, 256, 0, stream>>>(d_reqs, (int)wreq.size(), d_films, d_fdims, d_fdims + reqs.size());
        CUDA_TRY(cudaEventRecord(s0->ev1, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        rc = check_err(s0);
    }
    // On an error exit up to two batches of replays may still be queued; they
    // write the shared workspace and the films, so let them finish before the
    // graph goes away and the next call reuses the workspace.
    if (rc != RT_OK) cudaStreamSynchronize(stream);
    if (rc == RT_ERR_CUDA && ws.exec) {   // a failed launch: do not replay that graph again
        cudaGraphExecDestroy(ws.exec);
        ws.exec = nullptr;
        ws.exec_key.clear();
    }
    for (auto e : pev) cudaEventDestroy(e);
    if (rc != RT_OK) return rc;
    if (st) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, s0->ev0, s0->ev1);
        st->kernel_ms = ms;
        st->samples = (uint64_t)total;
        st->kernel_launches = (int32_t)(iters * per_iter + (mode == rt::WF_RENDER ? 1 : 0));
        st->iterations = (int32_t)iters;
        st->regen_ms = t_regen;
        st->extend_ms = t_extend;
        st->sort_ms = t_sort;
        st->shade_ms = t_shade;
        st->occlude_ms = t_occlude;
        st->rr_min_bounces = wreq[0].rc.rr_min_bounces;
        st->rr_min_survival = wreq[0].rc.rr_min_survival;
        st->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return RT_OK;
}

WfConfig g_wf_default;

// The wavefront configuration of one scene's request: the scene's tuned
// values, overridden by the request's own.
int wf_config(const RtScene* sc, const RtRenderParams* p, WfConfig& out) {
    WfConfig cfg = g_wf_default;
    if (sc->tuned) {
        cfg.slots = sc->tuned_slots;
        cfg.block = sc->tuned_block;
        cfg.sort = sc->tuned_sort;
        cfg.layout = sc->tuned_layout;
        cfg.fetch = sc->tuned_fetch;
        cfg.tblock = sc->tuned_tblock;
        cfg.groups = sc->tuned_groups;
    }
    if (p->wavefront_size > 0) cfg.slots = p->wavefront_size;
    if (p->block_size > 0) cfg.block = p->block_size;
    if (p->sort_materials >= 0) cfg.sort = p->sort_materials;
    if (p->node_layout == 2 || p->node_layout == 4) cfg.layout = p->node_layout;
    if (p->ray_fetch == 1 || p->ray_fetch == 2) cfg.fetch = p->ray_fetch;
    if (p->trace_block_size > 0) cfg.tblock = p->trace_block_size;
    if (p->ray_groups >= 1 && p->ray_groups <= 4) cfg.groups = p->ray_groups;
    cfg.profile = p->profile_kernels != 0;
    apply_test_limits(cfg, p);
    if (cfg.block != 64 && cfg.block != 128 && cfg.block != 256)
        return fail(RT_ERR_INVALID_ARG, "block_size must be 64, 128 or 256");
    if (cfg.tblock != 0 && cfg.tblock != 64 && cfg.tblock != 128 && cfg.tblock != 256)
        return fail(RT_ERR_INVALID_ARG, "trace_block_size must be 64, 128 or 256");
    out = cfg;
    return RT_OK;
}

int wf_render_one(RtScene* sc, const RtRenderParams* p, const RtCameraDesc& cam, float* d_film, RtStats* st) {
    HostReq q;
    q.scene = sc;
    q.rc = make_rc(sc, p, cam);
    q.x0 = p->pixel_x0;
    q.y0 = p->pixel_y0;
    q.ww = p->window_w > 0 ? p->window_w : p->width;
    q.wh = p->window_h > 0 ? p->window_h : p->height;
    q.spp = p->spp;
    q.spp0 = p->spp_offset;
    q.W = p->width;
    q.H = p->height;
    q.d_film = d_film;
    WfConfig cfg;
    int rc = wf_config(sc, p, cfg);
    if (rc != RT_OK) return rc;
    if (p->window_w > 0 || p->window_h > 0)
        CUDA_TRY(cudaMemsetAsync(d_film, 0, (size_t)3 * p->width * p->height * sizeof(float), sc->stream));
    return wf_render({q}, cfg, st);
}

}  // namespace

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

int rt_abi_version(void) { return RT3D_ABI_VERSION; }

int rt_checked_build(void) {
#ifdef RT_CHECKED
    return 1;
#else
    return 0;
#endif
}

const char* rt_last_error(void) { return g_err.c_str(); }

int rt_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return fail(RT_ERR_NO_DEVICE, "no CUDA device");
    return n;
}

int rt_scene_create(const RtWorldDesc* world, RtScene** out) { return rt_scene_create_ex(world, nullptr, out); }

int rt_scene_create_ex(const RtWorldDesc* world, const RtSceneOptions* options, RtScene** out) {
    if (!world || !out) return fail(RT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    RtSceneOptions opt{};
    if (options) opt = *options;
    if (opt.bvh_build < RT_BVH_AUTO || opt.bvh_build > RT_BVH_DEVICE)
        return fail(RT_ERR_INVALID_ARG, "bvh_build must be RT_BVH_AUTO, RT_BVH_HOST or RT_BVH_DEVICE");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(RT_ERR_NO_DEVICE, "no CUDA device");
    rt::BuildOptions bo;
    if (opt.bvh_build != RT_BVH_HOST) {
        bo.device_builder = rt::device_build_meshes;
        bo.device_min_tris = opt.bvh_build == RT_BVH_AUTO ? RT_BVH_AUTO_MIN_TRIS : 0;
    }
    auto* sc = new RtScene();
    std::string err;
    int rc = rt::build_world(world, sc->host, err, bo);
    if (rc == RT_OK) {
        sc->w = *world;
        sc->w_materials.assign(world->materials, world->materials + world->num_materials);
        sc->w_entities.assign(world->entities, world->entities + world->num_entities);
        if (world->num_tris > 0 && world->tri_verts)
            sc->w_tris.assign(world->tri_verts, world->tri_verts + world->num_tris * 9);
        if (world->num_tris > 0 && world->tri_normals)
            sc->w_normals.assign(world->tri_normals, world->tri_normals + world->num_tris * 9);
        if (world->num_tris > 0 && world->tri_uvs)
            sc->w_uvs.assign(world->tri_uvs, world->tri_uvs + world->num_tris * 6);
        if (world->num_lights > 0 && world->lights)
            sc->w_lights.assign(world->lights, world->lights + world->num_lights);
        sc->w.materials = sc->w_materials.data();
        sc->w.entities = sc->w_entities.data();
        sc->w.tri_verts = sc->w_tris.empty() ? nullptr : sc->w_tris.data();
        sc->w.tri_normals = sc->w_normals.empty() ? nullptr : sc->w_normals.data();
        sc->w.tri_uvs = sc->w_uvs.empty() ? nullptr : sc->w_uvs.data();
        sc->w.lights = sc->w_lights.empty() ? nullptr : sc->w_lights.data();
    }
    if (rc != RT_OK) {
        delete sc;
        return fail(rc, err);
    }
    cudaGetDevice(&sc->device);
    const rt::HostScene& h = sc->host;
    rt::SceneView& v = sc->view;
    int r = RT_OK;
    r = r ? r : upload(sc, h.cnodes, &v.cnodes);
    r = r ? r : upload(sc, h.cnodes4, &v.cnodes4);
    r = r ? r : upload(sc, h.mesh_root4, &v.mesh_root4);
    r = r ? r : upload(sc, h.top_items, &v.top_items);
    r = r ? r : upload(sc, h.tris, &v.tris);
    r = r ? r : upload(sc, h.tri_entity, &v.tri_entity);
    r = r ? r : upload(sc, h.tri_local, &v.tri_local);
    r = r ? r : upload(sc, h.entities, &v.entities);
    r = r ? r : upload(sc, h.ent_box, &v.ent_box);
    r = r ? r : upload(sc, h.quads, &v.quads);
    r = r ? r : upload(sc, h.spheres, &v.spheres);
    r = r ? r : upload(sc, h.materials, &v.materials);
    r = r ? r : upload(sc, h.lights, &v.lights);
    r = r ? r : upload(sc, h.light_tris, &v.light_tris);
    r = r ? r : upload(sc, h.smooth, &v.smooth);
    r = r ? r : upload(sc, h.tri_smooth, &v.tri_smooth, true);
    r = r ? r : upload(sc, h.emitter_light, &v.emitter_light);
    r = r ? r : upload(sc, h.pick_cdf, &v.pick_cdf);
    r = r ? r : upload(sc, h.pick_pdf, &v.pick_pdf);
    r = r ? r : upload(sc, h.lut_e, &v.lut_e);
    r = r ? r : upload(sc, h.lut_eavg, &v.lut_eavg);
    if (r != RT_OK) {
        rt_scene_destroy(sc);
        return r;
    }
    v.num_lights = (int)h.lights.size();
    v.top_is_bvh = h.top_is_bvh;
    v.top_root = h.top_root_code;
    v.top_root4 = h.top_root4;
    v.num_top_items = (int)h.top_items.size();
    v.n_cnodes = (int)(h.cnodes.size() / 4);
    v.n_cnodes4 = (int)(h.cnodes4.size() / 8);
    v.n_tris = (int)(h.tris.size() / 3);
    v.n_entities = (int)h.entities.size();
    v.n_quads = (int)h.quads.size();
    v.n_spheres = (int)h.spheres.size();
    v.n_materials = (int)h.materials.size();
    v.n_light_tris = (int)h.light_tris.size();
    v.n_smooth = (int)h.smooth.size();
    v.has_medium = h.has_medium;
    v.sigma_a = h.sigma_a;
    v.sigma_s = h.sigma_s;
    v.sigma_t = h.sigma_t;
    v.hg_g = h.hg_g;
    v.sky = h.sky;
    v.sky_on = h.sky_on;
    v.env_light = h.env_light;
    ray_sort_box(h, v);
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
    if (sc->film) cudaFree(sc->film);
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
    info->bvh_on_device = h.bvh_on_device;
    info->device_bytes = (int64_t)sc->bytes;
    info->bvh_build_ms = h.bvh_build_ms;
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
        info->bvh_build_ms = h.bvh_build_ms;
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

int rt_render_capture(RtScene* sc, const RtRenderParams* p, float* out, const RtCapture* cap, RtStats* st) {
    if (!sc || !p || !out || !cap) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (p->window_w > 0 || p->window_h > 0 || p->pixel_x0 != 0 || p->pixel_y0 != 0)
        return fail(RT_ERR_INVALID_ARG, "a capturing render covers the whole frame");
    if (p->count_work) return fail(RT_ERR_INVALID_ARG, "count_work is not available with capture");
    std::lock_guard<std::mutex> lk(sc->mu);
    auto t0 = std::chrono::steady_clock::now();
    int rc_ = validate_params(sc, p);
    if (rc_ != RT_OK) return rc_;
    CUDA_TRY(cudaSetDevice(sc->device));
    rt::RenderConst rc = make_rc(sc, p, sc->host.camera);
    int ww = p->width, wh = p->height;
    int64_t npix = (int64_t)ww * wh;
    int64_t target = 148LL * 2048 * 2;
    int nchunks = (int)std::min<int64_t>(p->spp, std::max<int64_t>(1, (target + npix - 1) / npix));
    int per_chunk = (p->spp + nchunks - 1) / nchunks;
    nchunks = (p->spp + per_chunk - 1) / per_chunk;
    size_t partial_bytes = (size_t)nchunks * kCapSums * npix * sizeof(float);
    size_t out_bytes = (size_t)23 * npix * sizeof(float);
    rc_ = ensure_scratch(sc, partial_bytes + out_bytes);
    if (rc_ != RT_OK) return rc_;
    float* partial = static_cast<float*>(sc->scratch);
    float* res = reinterpret_cast<float*>(static_cast<char*>(sc->scratch) + partial_bytes);
    CUDA_TRY(cudaMemsetAsync(sc->d_err, 0, sizeof(int), sc->stream));
    dim3 grid((ww + 15) / 16, (wh + 7) / 8, nchunks);
    CUDA_TRY(cudaEventRecord(sc->ev0, sc->stream));
    k_render_capture<kStack><<<grid, kBlock, 0, sc->stream>>>(sc->view, rc, ww, wh, p->spp_offset, per_chunk, p->spp,
                                                              partial, sc->d_err);
    k_resolve_capture<<<(unsigned)((npix + 255) / 256), 256, 0, sc->stream>>>(partial, nchunks, ww, wh, p->spp, res);
    CUDA_TRY(cudaEventRecord(sc->ev1, sc->stream));
    CUDA_TRY(cudaGetLastError());
    // the planes the caller asked for, in the result's plane order
    float* const dst[9] = {out, cap->beauty_a, cap->beauty_b, cap->albedo_a, cap->albedo_b,
                           cap->normal_a, cap->normal_b, cap->depth_a, cap->depth_b};
    const int first[9] = {0, 3, 6, 9, 12, 15, 18, 21, 22};
    for (int k = 0; k < 9; k++) {
        if (!dst[k]) continue;
        size_t nb = (size_t)(k < 7 ? 3 : 1) * npix * sizeof(float);
        CUDA_TRY(cudaMemcpyAsync(dst[k], res + (size_t)first[k] * npix, nb, cudaMemcpyDeviceToHost, sc->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(sc->stream));
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
        st->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return RT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free megakernel render.
//
// Some hosts cannot allocate device memory while they render: a host that
// reserves its whole device-memory budget at start-up and must not grow it,
// or one that renders from a latency-critical thread where cudaMalloc and
// cudaFree (which synchronise the device) are not allowed. For them the
// megakernel's scratch — the per-chunk partial sums and the error word — lives
// in this one fixed array instead of memory allocated per call. The array is
// 32 MiB (kNoAllocFloats floats): the error word in its first 256 bytes, the
// partial sums after it. Every GPU that loads the library holds it until the
// process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocFloats = size_t(8) << 20;   // 32 MiB
constexpr size_t kNoAllocHeader = 64;                // floats before the partial sums (256 B)
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

std::mutex g_noalloc_mu;
float* g_noalloc_ptr[64] = {};

// The device address of g_noalloc_scratch on the current device, looked up
// once per device (the host-side name is only a stand-in for it).
int noalloc_scratch(int device, float** out) {
    if (device < 0 || device >= 64) return fail(RT_ERR_INVALID_ARG, "device index out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(RT_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[device] = static_cast<float*>(ptr);
    }
    *out = g_noalloc_ptr[device];
    return RT_OK;
}

}  // namespace

extern "C" {

int rt_render_device_noalloc(RtScene* sc, const RtRenderParams* p, float* d_film, RtStats* st) {
    if (!sc || !p || !d_film) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (p->count_work) return fail(RT_ERR_INVALID_ARG, "count_work is not available without allocation");
    if (p->kernel != RT_KERNEL_MEGAKERNEL)
        return fail(RT_ERR_INVALID_ARG, "the allocation-free render runs the megakernel only (kernel must be "
                                        "RT_KERNEL_MEGAKERNEL)");
    std::lock_guard<std::mutex> lk(sc->mu);
    auto t0 = std::chrono::steady_clock::now();
    int rc_ = validate_params(sc, p);
    if (rc_ != RT_OK) return rc_;
    CUDA_TRY(cudaSetDevice(sc->device));
    float* scratch = nullptr;
    rc_ = noalloc_scratch(sc->device, &scratch);
    if (rc_ != RT_OK) return rc_;
    int ww = p->window_w > 0 ? p->window_w : p->width;
    int wh = p->window_h > 0 ? p->window_h : p->height;
    int64_t npix = (int64_t)ww * wh;
    const int64_t cap = (int64_t)(kNoAllocFloats - kNoAllocHeader);
    if (3 * npix > cap)
        return fail(RT_ERR_INVALID_ARG, "render window of " + std::to_string(npix) +
                                            " pixels exceeds the allocation-free maximum of " +
                                            std::to_string(cap / 3) + " pixels");
    // The same chunking as rt_render_device, reduced until the partial sums fit.
    int64_t target = 148LL * 2048 * 2;
    int nchunks = (int)std::min<int64_t>(p->spp, std::max<int64_t>(1, (target + npix - 1) / npix));
    nchunks = (int)std::min<int64_t>(nchunks, cap / (3 * npix));
    int per_chunk = (p->spp + nchunks - 1) / nchunks;
    nchunks = (p->spp + per_chunk - 1) / per_chunk;
    rt::RenderConst rc = make_rc(sc, p, sc->host.camera);
    int* err = reinterpret_cast<int*>(scratch);
    auto* work = reinterpret_cast<unsigned long long*>(scratch + 16);
    float* partial = scratch + kNoAllocHeader;
    // The array keeps the previous call's contents: only the error word must
    // start at zero (every partial sum is overwritten by the kernel).
    CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), sc->stream));
    if (p->window_w > 0 || p->window_h > 0)
        CUDA_TRY(cudaMemsetAsync(d_film, 0, (size_t)3 * p->width * p->height * sizeof(float), sc->stream));
    dim3 grid((ww + 15) / 16, (wh + 7) / 8, nchunks);
    CUDA_TRY(cudaEventRecord(sc->ev0, sc->stream));
    k_render_mega<kStack, false><<<grid, kBlock, 0, sc->stream>>>(sc->view, rc, p->pixel_x0, p->pixel_y0, ww, wh,
                                                                  p->spp_offset, per_chunk, p->spp, partial, work,
                                                                  err);
    k_resolve<<<(unsigned)((npix + 255) / 256), 256, 0, sc->stream>>>(partial, nchunks, ww, wh, p->width, p->height,
                                                                     p->pixel_x0, p->pixel_y0, p->spp, d_film);
    CUDA_TRY(cudaEventRecord(sc->ev1, sc->stream));
    CUDA_TRY(cudaGetLastError());
    int e = 0;
    CUDA_TRY(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, sc->stream));
    CUDA_TRY(cudaStreamSynchronize(sc->stream));
    if (e == RT_ERR_STACK) return fail(RT_ERR_STACK, "traversal stack bound exceeded");
    if (e != 0) return fail(RT_ERR_BOUNDS, "device error " + std::to_string(e));
    rc_ = checked_flag(sc->stream);
    if (rc_ != RT_OK) return rc_;
    if (st) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, sc->ev0, sc->ev1);
        st->kernel_ms = ms;
        st->samples = (uint64_t)npix * (uint64_t)p->spp;
        st->kernel_launches = 2;
        st->rr_min_bounces = rc.rr_min_bounces;
        st->rr_min_survival = rc.rr_min_survival;
        st->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return RT_OK;
}

int rt_render(RtScene* sc, const RtRenderParams* p, float* out, RtStats* st) {
    if (!sc || !out || !p) return fail(RT_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(sc->mu);
    auto t0 = std::chrono::steady_clock::now();
    size_t film_bytes = (size_t)3 * p->width * p->height * sizeof(float);
    if (p->width <= 0 || p->height <= 0) return fail(RT_ERR_INVALID_ARG, "bad image size");
    CUDA_TRY(cudaSetDevice(sc->device));
    // The device film is kept by the scene and grown when a larger image asks
    // for it, so repeated renders allocate nothing (cudaFree would also
    // synchronise the whole device on every call).
    if (sc->film_bytes < film_bytes) {
        if (sc->film) cudaFree(sc->film);
        sc->film = nullptr;
        sc->film_bytes = 0;
        if (cudaMalloc(&sc->film, film_bytes) != cudaSuccess) {
            sc->film = nullptr;
            return fail(RT_ERR_OOM, "film allocation failed");
        }
        sc->film_bytes = film_bytes;
    }
    int rc = render_to_device(sc, p, sc->host.camera, sc->film, st);
    if (rc == RT_OK) {
        if (cudaMemcpyAsync(out, sc->film, film_bytes, cudaMemcpyDeviceToHost, sc->stream) != cudaSuccess ||
            cudaStreamSynchronize(sc->stream) != cudaSuccess)
            rc = fail(RT_ERR_CUDA, "film copy failed");
    }
    if (st && rc == RT_OK)
        st->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int rt_render_batch(RtScene* const* scenes, int32_t num_scenes, const RtRequest* reqs, int32_t n,
                    const RtRenderParams* common, float* const* outs, RtStats* st) {
    if (!scenes || !reqs || !outs || !common || n <= 0 || num_scenes <= 0)
        return fail(RT_ERR_INVALID_ARG, "null argument or empty batch");
    auto t0 = std::chrono::steady_clock::now();
    // Every distinct scene of the batch stays locked for the whole call, as a
    // single-scene call locks its scene: the batch uses their streams, error
    // words, events and parameters. Locks are taken in address order, so two
    // batches over overlapping scenes cannot deadlock.
    std::vector<RtScene*> locked;
    for (int i = 0; i < n; i++) {
        if (reqs[i].scene < 0 || reqs[i].scene >= num_scenes || !scenes[reqs[i].scene])
            return fail(RT_ERR_INVALID_ARG, "request " + std::to_string(i) + ": bad scene");
        locked.push_back(scenes[reqs[i].scene]);
    }
    std::sort(locked.begin(), locked.end(), std::less<RtScene*>());
    locked.erase(std::unique(locked.begin(), locked.end()), locked.end());
    std::vector<std::unique_lock<std::mutex>> guards;
    guards.reserve(locked.size());
    for (RtScene* sc : locked) guards.emplace_back(sc->mu);
    std::vector<HostReq> hq((size_t)n);
    std::vector<float*> d_films((size_t)n, nullptr);
    int rc = RT_OK;
    for (int i = 0; i < n && rc == RT_OK; i++) {
        const RtRequest& q = reqs[i];
        if (q.scene < 0 || q.scene >= num_scenes || !scenes[q.scene] || !outs[i]) {
            rc = fail(RT_ERR_INVALID_ARG, "request " + std::to_string(i) + ": bad scene or output");
            break;
        }
        RtScene* sc = scenes[q.scene];
        RtRenderParams p = *common;
        p.width = q.width;
        p.height = q.height;
        p.spp = q.spp;
        p.max_depth = q.max_depth;
        p.pixel_x0 = p.pixel_y0 = p.window_w = p.window_h = 0;
        p.spp_offset = 0;
        rc = validate_params(sc, &p);
        if (rc != RT_OK) break;
        if (cudaSetDevice(sc->device) != cudaSuccess ||
            cudaMalloc(&d_films[i], (size_t)3 * q.width * q.height * sizeof(float)) != cudaSuccess) {
            rc = fail(RT_ERR_OOM, "film allocation failed");
            break;
        }
        HostReq& h = hq[i];
        h.scene = sc;
        h.rc = make_rc(sc, &p, q.camera);
        h.x0 = h.y0 = 0;
        h.ww = q.width;
        h.wh = q.height;
        h.spp = q.spp;
        h.spp0 = 0;
        h.W = q.width;
        h.H = q.height;
        h.d_film = d_films[i];
    }
    if (rc == RT_OK) {
        WfConfig cfg = g_wf_default;
        RtScene* s0 = scenes[reqs[0].scene];
        if (s0->tuned) {
            cfg.slots = s0->tuned_slots;
            cfg.block = s0->tuned_block;
            cfg.sort = s0->tuned_sort;
            cfg.layout = s0->tuned_layout;
            cfg.fetch = s0->tuned_fetch;
            cfg.tblock = s0->tuned_tblock;
            cfg.groups = s0->tuned_groups;
        }
        if (common->wavefront_size > 0) cfg.slots = common->wavefront_size;
        if (common->block_size > 0) cfg.block = common->block_size;
        if (common->sort_materials >= 0) cfg.sort = common->sort_materials;
        if (common->node_layout == 2 || common->node_layout == 4) cfg.layout = common->node_layout;
        if (common->ray_fetch == 1 || common->ray_fetch == 2) cfg.fetch = common->ray_fetch;
        if (common->trace_block_size > 0) cfg.tblock = common->trace_block_size;
        if (common->ray_groups >= 1 && common->ray_groups <= 4) cfg.groups = common->ray_groups;
        cfg.profile = common->profile_kernels != 0;
        apply_test_limits(cfg, common);
        rc = wf_render(hq, cfg, st);
    }
    for (int i = 0; i < n; i++) {
        if (rc == RT_OK &&
            cudaMemcpy(outs[i], d_films[i], (size_t)3 * reqs[i].width * reqs[i].height * sizeof(float),
                       cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(RT_ERR_CUDA, "film copy failed");
        if (d_films[i]) cudaFree(d_films[i]);
    }
    if (st && rc == RT_OK)
        st->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int rt_autotune(RtScene* sc, const RtRenderParams* params, RtRenderParams* best) {
    if (!sc || !params) return fail(RT_ERR_INVALID_ARG, "null argument");
    int rc = validate_params(sc, params);
    if (rc != RT_OK) return rc;
    std::lock_guard<std::mutex> lk(sc->mu);
    CUDA_TRY(cudaSetDevice(sc->device));
    // A bounded slice of the render: the full window at the spp that gives
    // ~16 M samples (at least 4x the largest wavefront), capped at params->spp.
    int ww = params->window_w > 0 ? params->window_w : params->width;
    int wh = params->window_h > 0 ? params->window_h : params->height;
    int64_t npix = (int64_t)ww * wh;
    int spp = (int)std::max<int64_t>(1, std::min<int64_t>(params->spp, ((int64_t)1 << 24) / npix + 1));
    float* d_film = nullptr;
    if (cudaMalloc(&d_film, (size_t)3 * params->width * params->height * sizeof(float)) != cudaSuccess)
        return fail(RT_ERR_OOM, "film allocation failed");
    const int sizes[3] = {1 << 18, 1 << 20, 1 << 22};
    const int blocks[3] = {64, 128, 256};
    const int layouts[2] = {2, 4};
    int nl = sc->host.max_stack4 <= kStack ? 2 : 1;
    double best_ms = 1e30;
    WfConfig pick;
    for (int si = 0; si < 3 && rc == RT_OK; si++)
        for (int bi = 0; bi < 3 && rc == RT_OK; bi++)
            for (int so = 0; so < 2 && rc == RT_OK; so++)
                for (int li = 0; li < nl && rc == RT_OK; li++) {
                    RtRenderParams p = *params;
                    p.kernel = RT_KERNEL_WAVEFRONT;
                    p.spp = spp;
                    p.count_work = 0;
                    p.wavefront_size = sizes[si];
                    p.block_size = blocks[bi];
                    p.sort_materials = so;
                    p.node_layout = layouts[li];
                    p.ray_fetch = 1;
                    p.trace_block_size = blocks[bi];
                    p.ray_groups = 1;
                    RtStats s1{};
                    rc = render_to_device(sc, &p, sc->host.camera, d_film, &s1);
                    if (rc == RT_OK && s1.kernel_ms < best_ms) {
                        best_ms = s1.kernel_ms;
                        pick.slots = sizes[si];
                        pick.block = blocks[bi];
                        pick.sort = so;
                        pick.layout = layouts[li];
                    }
                }
    pick.tblock = pick.block;
    pick.groups = 1;   // the passes above ran slot order
    // then, on the winner, the block of extend/occlude alone and the
    // persistent dynamic-fetch kernels
    for (int bi = 0; bi < 3 && rc == RT_OK; bi++) {
        if (blocks[bi] == pick.block) continue;
        RtRenderParams p = *params;
        p.kernel = RT_KERNEL_WAVEFRONT;
        p.spp = spp;
        p.count_work = 0;
        p.wavefront_size = pick.slots;
        p.block_size = pick.block;
        p.sort_materials = pick.sort;
        p.node_layout = pick.layout;
        p.ray_fetch = 1;
        p.trace_block_size = blocks[bi];
        p.ray_groups = 1;
        RtStats s1{};
        rc = render_to_device(sc, &p, sc->host.camera, d_film, &s1);
        if (rc == RT_OK && s1.kernel_ms < best_ms) {
            best_ms = s1.kernel_ms;
            pick.tblock = blocks[bi];
        }
    }
    for (int g = 2; g <= 4 && rc == RT_OK; g++) {   // block-local regrouping, then the ray sorts
        RtRenderParams p = *params;
        p.kernel = RT_KERNEL_WAVEFRONT;
        p.spp = spp;
        p.count_work = 0;
        p.wavefront_size = pick.slots;
        p.block_size = pick.block;
        p.sort_materials = pick.sort;
        p.node_layout = pick.layout;
        p.ray_fetch = 1;
        p.trace_block_size = pick.tblock;
        p.ray_groups = g;
        RtStats s1{};
        rc = render_to_device(sc, &p, sc->host.camera, d_film, &s1);
        if (rc == RT_OK && s1.kernel_ms < best_ms) {
            best_ms = s1.kernel_ms;
            pick.groups = g;
        }
    }
    if (rc == RT_OK && pick.layout == 2) {
        RtRenderParams p = *params;
        p.kernel = RT_KERNEL_WAVEFRONT;
        p.spp = spp;
        p.count_work = 0;
        p.wavefront_size = pick.slots;
        p.block_size = pick.block;
        p.sort_materials = pick.sort;
        p.node_layout = 2;
        p.ray_fetch = 2;
        p.trace_block_size = pick.tblock;
        p.ray_groups = pick.groups;
        RtStats s1{};
        rc = render_to_device(sc, &p, sc->host.camera, d_film, &s1);
        if (rc == RT_OK && s1.kernel_ms < best_ms) {
            best_ms = s1.kernel_ms;
            pick.fetch = 2;
        }
    }
    cudaFree(d_film);
    if (rc != RT_OK) return rc;
    sc->tuned = 1;
    sc->tuned_slots = pick.slots;
    sc->tuned_block = pick.block;
    sc->tuned_sort = pick.sort;
    sc->tuned_layout = pick.layout;
    sc->tuned_fetch = pick.fetch;
    sc->tuned_tblock = pick.tblock;
    sc->tuned_groups = pick.groups;
    if (best) {
        *best = *params;
        best->kernel = RT_KERNEL_WAVEFRONT;
        best->wavefront_size = pick.slots;
        best->block_size = pick.block;
        best->sort_materials = pick.sort;
        best->node_layout = pick.layout;
        best->ray_fetch = pick.fetch;
        best->trace_block_size = pick.tblock;
        best->ray_groups = pick.groups;
    }
    return RT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Differentiable parameter vector and the path-replay adjoint.
// ---------------------------------------------------------------------------
namespace {

constexpr int kPerMat = RT_ADJ_PARAMS_PER_MATERIAL;
static_assert(kPerMat == rt::kAdjPerMat, "slot layout");

int param_count(const RtScene* sc) { return (int)sc->w_materials.size() * kPerMat + RT_ADJ_GLOBAL_PARAMS; }

void get_params(const RtScene* sc, float* out) {
    int nm = (int)sc->w_materials.size();
    std::fill(out, out + param_count(sc), 0.0f);
    for (int i = 0; i < nm; i++) {
        const RtMaterialDesc& d = sc->w_materials[i];
        const rt::Material& m = sc->host.materials[i];
        float* p = out + i * kPerMat;
        if (d.type == RT_MAT_EMISSIVE) {
            p[RT_ADJ_RADIANCE + 0] = m.emission.x;
            p[RT_ADJ_RADIANCE + 1] = m.emission.y;
            p[RT_ADJ_RADIANCE + 2] = m.emission.z;
            continue;
        }
        for (int c = 0; c < 3; c++) p[RT_ADJ_BASE_COLOR + c] = d.base_color[c];
        p[RT_ADJ_ROUGHNESS] = d.roughness;
        p[RT_ADJ_METALLIC] = d.metallic;
        p[RT_ADJ_SPECULAR] = d.specular;
        p[RT_ADJ_SPECULAR_TINT] = d.specular_tint;
        p[RT_ADJ_SHEEN] = d.sheen;
        p[RT_ADJ_SHEEN_TINT] = d.sheen_tint;
        p[RT_ADJ_CLEARCOAT] = d.clearcoat;
        p[RT_ADJ_SPEC_TRANS] = d.spec_trans;
        p[RT_ADJ_ANISOTROPIC] = d.anisotropic;
        p[RT_ADJ_ABSORPTION + 0] = m.trans_sigma.x;
        p[RT_ADJ_ABSORPTION + 1] = m.trans_sigma.y;
        p[RT_ADJ_ABSORPTION + 2] = m.trans_sigma.z;
    }
    float* g = out + nm * kPerMat;
    for (int c = 0; c < 3; c++) {
        g[RT_ADJ_MEDIUM_SIGMA_A + c] = sc->w.medium.sigma_a[c];
        g[RT_ADJ_MEDIUM_SIGMA_S + c] = sc->w.medium.sigma_s[c];
    }
}

// Writes the vector into the stored world description. A slot equal to what
// get_params reports leaves its description field untouched, so that
// set(get()) is an exact no-op.
void put_params(RtScene* sc, const float* in) {
    int nm = (int)sc->w_materials.size();
    for (int i = 0; i < nm; i++) {
        RtMaterialDesc& d = sc->w_materials[i];
        const rt::Material& m = sc->host.materials[i];
        const float* p = in + i * kPerMat;
        if (d.type == RT_MAT_EMISSIVE) {   // radiance = colour * intensity; intensity kept
            float cur[3] = {m.emission.x, m.emission.y, m.emission.z};
            if (p[0] == cur[0] && p[1] == cur[1] && p[2] == cur[2]) continue;
            if (!(d.intensity > 0.0f)) {
                d.intensity = 1.0f;
                for (int c = 0; c < 3; c++) d.base_color[c] = p[c];
            } else {
                for (int c = 0; c < 3; c++)
                    if (p[c] != cur[c]) d.base_color[c] = p[c] / d.intensity;
            }
            continue;
        }
        for (int c = 0; c < 3; c++) d.base_color[c] = p[RT_ADJ_BASE_COLOR + c];
        d.roughness = p[RT_ADJ_ROUGHNESS];
        d.metallic = p[RT_ADJ_METALLIC];
        d.specular = p[RT_ADJ_SPECULAR];
        d.specular_tint = p[RT_ADJ_SPECULAR_TINT];
        d.sheen = p[RT_ADJ_SHEEN];
        d.sheen_tint = p[RT_ADJ_SHEEN_TINT];
        d.clearcoat = p[RT_ADJ_CLEARCOAT];
        d.spec_trans = p[RT_ADJ_SPEC_TRANS];
        d.anisotropic = p[RT_ADJ_ANISOTROPIC];
        const float* sg = p + RT_ADJ_ABSORPTION;
        if (sg[0] == m.trans_sigma.x && sg[1] == m.trans_sigma.y && sg[2] == m.trans_sigma.z) continue;
        // transmission_color = exp(-sigma * depth) (ResolveTransmission, DisneyBsdf.cs:1039-1048)
        if (!(d.has_transmission_color && d.transmission_depth > 0.0f)) {
            d.has_transmission_color = 1;
            d.transmission_depth = 1.0f;
        }
        for (int c = 0; c < 3; c++)
            d.transmission_color[c] = std::exp(-std::fmax(sg[c], 0.0f) * d.transmission_depth);
    }
    const float* g = in + nm * kPerMat;
    for (int c = 0; c < 3; c++) {
        sc->w.medium.sigma_a[c] = g[RT_ADJ_MEDIUM_SIGMA_A + c];
        sc->w.medium.sigma_s[c] = g[RT_ADJ_MEDIUM_SIGMA_S + c];
    }
}

// The wavefront adjoint (params->kernel RT_KERNEL_WAVEFRONT): the samples in
// runs of whole spp slices of at most kAdjRecord samples, each run rendered
// once with its end states recorded (WF_RECORD) and then replayed with the
// gradient hooks (WF_REPLAY). base carries the parameter, mask and gradient
// buffers; ms and launches add up the passes.
constexpr long long kAdjRecord = 1LL << 24;   // 64 B per recorded sample: 1 GiB

int wf_adjoint(RtScene* sc, const RtRenderParams* p, const rt::WfAdjoint& base, double& ms, long long& launches) {
    WfConfig cfg;
    int rc = wf_config(sc, p, cfg);
    if (rc != RT_OK) return rc;
    HostReq q;
    q.scene = sc;
    q.rc = make_rc(sc, p, sc->host.camera);
    q.x0 = p->pixel_x0;
    q.y0 = p->pixel_y0;
    q.ww = p->window_w > 0 ? p->window_w : p->width;
    q.wh = p->window_h > 0 ? p->window_h : p->height;
    q.W = p->width;
    q.H = p->height;
    q.d_film = nullptr;
    long long npix = (long long)q.ww * q.wh;
    int per = (int)std::max<long long>(1, std::min<long long>(p->spp, kAdjRecord / std::max<long long>(npix, 1)));
    rt::WfAdjoint J = base;
    J.nrec = npix * per;
    void* mem = nullptr;
    if (cudaMalloc(&mem, (size_t)J.nrec * 4 * sizeof(float4)) != cudaSuccess)
        return fail(RT_ERR_OOM, "adjoint sample record");
    J.rec = static_cast<float4*>(mem);
    for (int s0 = 0; s0 < p->spp && rc == RT_OK; s0 += per) {
        q.spp = std::min(per, p->spp - s0);
        q.spp0 = p->spp_offset + s0;
        for (int mode : {rt::WF_RECORD, rt::WF_REPLAY}) {
            RtStats one{};
            rc = wf_render({q}, cfg, &one, mode, &J);
            if (rc != RT_OK) break;
            ms += one.kernel_ms;
            launches += one.kernel_launches;
        }
    }
    cudaFree(mem);
    return rc;
}

}  // namespace

extern "C" {

int rt_scene_get_params(const RtScene* sc, float* params, int32_t count) {
    if (!sc || !params) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (count != param_count(sc))
        return fail(RT_ERR_INVALID_ARG, "parameter vector needs " + std::to_string(param_count(sc)) + " floats");
    get_params(sc, params);
    return RT_OK;
}

int rt_scene_set_params(RtScene* sc, const float* params, int32_t count) {
    if (!sc || !params) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (count != param_count(sc))
        return fail(RT_ERR_INVALID_ARG, "parameter vector needs " + std::to_string(param_count(sc)) + " floats");
    for (int32_t i = 0; i < count; i++)
        if (!std::isfinite(params[i])) return fail(RT_ERR_INVALID_ARG, "non-finite parameter " + std::to_string(i));
    std::lock_guard<std::mutex> lk(sc->mu);
    std::vector<RtMaterialDesc> keep_m = sc->w_materials;
    RtMediumDesc keep_med = sc->w.medium;
    put_params(sc, params);
    rt::HostScene h;
    std::string err;
    int rc = rt::build_world(&sc->w, h, err);
    if (rc != RT_OK || h.materials.size() != sc->host.materials.size() || h.lights.size() != sc->host.lights.size()) {
        sc->w_materials = keep_m;
        sc->w.medium = keep_med;
        return fail(rc != RT_OK ? rc : RT_ERR_INVALID_ARG, rc != RT_OK ? err : "parameter change altered the lights");
    }
    CUDA_TRY(cudaSetDevice(sc->device));
    CUDA_TRY(cudaStreamSynchronize(sc->stream));
    rt::SceneView& v = sc->view;
    CUDA_TRY(cudaMemcpy(const_cast<rt::Material*>(v.materials), h.materials.data(),
                        h.materials.size() * sizeof(rt::Material), cudaMemcpyHostToDevice));
    if (!h.lights.empty())
        CUDA_TRY(cudaMemcpy(const_cast<rt::Light*>(v.lights), h.lights.data(), h.lights.size() * sizeof(rt::Light),
                            cudaMemcpyHostToDevice));
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
    sc->host = std::move(h);
    return RT_OK;
}

int rt_adjoint(RtScene* sc, const RtRenderParams* p, const float* dimg, const uint8_t* mask, float* grad,
               int32_t count, RtStats* st) {
    if (!sc || !p || !dimg || !grad) return fail(RT_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(sc->mu);
    auto t0 = std::chrono::steady_clock::now();
    int rc_ = validate_params(sc, p);
    if (rc_ != RT_OK) return rc_;
    if (p->count_work) return fail(RT_ERR_INVALID_ARG, "count_work is not available in the adjoint");
    int np = param_count(sc);
    if (count != np) return fail(RT_ERR_INVALID_ARG, "gradient vector needs " + std::to_string(np) + " floats");
    CUDA_TRY(cudaSetDevice(sc->device));
    rt::RenderConst rcon = make_rc(sc, p, sc->host.camera);
    int ww = p->window_w > 0 ? p->window_w : p->width;
    int wh = p->window_h > 0 ? p->window_h : p->height;
    size_t film = (size_t)3 * p->width * p->height;
    std::vector<float> hp((size_t)np);
    get_params(sc, hp.data());
    int nm = (int)sc->w_materials.size();
    std::vector<unsigned> hm((size_t)nm, 0u);
    unsigned gm = 0u;
    for (int i = 0; i < np; i++) {
        if (mask && !mask[i]) continue;
        if (i < nm * kPerMat) hm[(size_t)(i / kPerMat)] |= 1u << (i % kPerMat);
        else gm |= 1u << (i - nm * kPerMat);
    }
    std::vector<int> act;   // the selected slots, for the wavefront replay's gather
    for (int i = 0; i < np; i++) {
        bool on = i < nm * kPerMat ? ((hm[(size_t)(i / kPerMat)] >> (i % kPerMat)) & 1u) : ((gm >> (i - nm * kPerMat)) & 1u);
        if (on) act.push_back(i);
    }
    size_t bytes = (size_t)np * sizeof(double) + (size_t)np * sizeof(float) + film * sizeof(float) +
                   (size_t)nm * sizeof(unsigned) + (size_t)(act.size() + 1) * sizeof(int) + 256;
    void* mem = nullptr;
    if (cudaMalloc(&mem, bytes) != cudaSuccess) return fail(RT_ERR_OOM, "adjoint buffers");
    char* base = static_cast<char*>(mem);
    double* d_grad = reinterpret_cast<double*>(base);
    float* d_params = reinterpret_cast<float*>(base + (size_t)np * sizeof(double));
    float* d_img = d_params + np;
    unsigned* d_mask = reinterpret_cast<unsigned*>(d_img + film);
    int* d_act = reinterpret_cast<int*>(d_mask + nm);
    int rc = RT_OK;
    auto step = [&](cudaError_t e, const char* what) {
        if (rc == RT_OK && e != cudaSuccess) rc = fail(RT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    step(cudaMemcpyAsync(d_img, dimg, film * sizeof(float), cudaMemcpyHostToDevice, sc->stream), "dL/dimage copy");
    step(cudaMemcpyAsync(d_params, hp.data(), (size_t)np * sizeof(float), cudaMemcpyHostToDevice, sc->stream),
         "parameter copy");
    step(cudaMemcpyAsync(d_mask, hm.data(), (size_t)nm * sizeof(unsigned), cudaMemcpyHostToDevice, sc->stream),
         "mask copy");
    if (!act.empty())
        step(cudaMemcpyAsync(d_act, act.data(), act.size() * sizeof(int), cudaMemcpyHostToDevice, sc->stream),
             "slot list copy");
    step(cudaMemsetAsync(d_grad, 0, (size_t)np * sizeof(double), sc->stream), "gradient clear");
    step(cudaMemsetAsync(sc->d_err, 0, sizeof(int), sc->stream), "error clear");
    AdjArgs a;
    a.x0 = p->pixel_x0;
    a.y0 = p->pixel_y0;
    a.ww = ww;
    a.wh = wh;
    a.W = p->width;
    a.H = p->height;
    a.spp = p->spp;
    a.spp0 = p->spp_offset;
    a.dimg = d_img;
    a.params = d_params;
    a.mmask = d_mask;
    a.gmask = gm;
    a.grad = d_grad;
    a.nparams = np;
    a.medium_base = nm * kPerMat;
    size_t shmem = (size_t)np * sizeof(float);
    a.use_shared = shmem <= 48 * 1024;
    if (!a.use_shared) shmem = 0;
    a.use_local = RT_ADJ_LOCAL_ACC && np <= rt::kAdjLocal;
    a.any4 = rcon.opaque && sc->host.max_stack4 <= kStack;
    long long total = (long long)ww * wh * p->spp;
    long long blocks = std::min<long long>((total + kBlock - 1) / kBlock, 148LL * 16);
    double wf_ms = 0.0;
    long long launches = 1;
    const bool wavefront = p->kernel == RT_KERNEL_WAVEFRONT;
    if (rc == RT_OK && wavefront) {
        rt::WfAdjoint J{};
        J.dimg = d_img;
        J.W = p->width;
        J.H = p->height;
        J.inv_spp = 1.0f / (float)p->spp;
        J.params = d_params;
        J.mmask = d_mask;
        J.gmask = gm;
        J.nparams = np;
        J.medium_base = nm * kPerMat;
        J.act = d_act;
        J.nact = (int)act.size();
        J.use_local = RT_ADJ_LOCAL_ACC && np <= rt::kAdjLocal;
        J.use_shared = (size_t)np * sizeof(float) <= 48 * 1024;
        J.grad = d_grad;
        launches = 0;
        if (!act.empty()) rc = wf_adjoint(sc, p, J, wf_ms, launches);
    } else if (rc == RT_OK) {
        step(cudaEventRecord(sc->ev0, sc->stream), "event");
        k_adjoint<kStack><<<(unsigned)std::max<long long>(blocks, 1), kBlock, shmem, sc->stream>>>(sc->view, rcon, a,
                                                                                                     sc->d_err);
        step(cudaGetLastError(), "k_adjoint launch");
        step(cudaEventRecord(sc->ev1, sc->stream), "event");
    }
    std::vector<double> hg((size_t)np, 0.0);
    if (rc == RT_OK) {
        step(cudaMemcpyAsync(hg.data(), d_grad, (size_t)np * sizeof(double), cudaMemcpyDeviceToHost, sc->stream),
             "gradient copy");
        step(cudaStreamSynchronize(sc->stream), "adjoint");
    }
    if (rc == RT_OK) rc = check_err(sc);
    float ms = 0.0f;
    if (rc == RT_OK && !wavefront) cudaEventElapsedTime(&ms, sc->ev0, sc->ev1);
    if (wavefront) ms = (float)wf_ms;
    cudaFree(mem);
    if (rc != RT_OK) return rc;
    for (int i = 0; i < np; i++) grad[i] = (float)hg[(size_t)i];
    if (st) {
        *st = RtStats{};
        st->kernel_ms = ms;
        st->samples = (uint64_t)total;
        st->kernel_launches = (int32_t)launches;
        st->rr_min_bounces = rcon.rr_min_bounces;
        st->rr_min_survival = rcon.rr_min_survival;
        st->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return RT_OK;
}

int rt_trace_closest(RtScene* sc, const float* rays, int64_t n, float tmin, float tmax, int32_t* hits,
                     int32_t node_layout) {
    if (!sc || !rays || !hits || n < 0) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (node_layout != 2 && node_layout != 4) return fail(RT_ERR_INVALID_ARG, "node_layout must be 2 or 4");
    if (n == 0) return RT_OK;
    std::lock_guard<std::mutex> lk(sc->mu);
    CUDA_TRY(cudaSetDevice(sc->device));
    if ((node_layout == 4 ? sc->host.max_stack4 : sc->host.max_stack) > kStack)
        return fail(RT_ERR_STACK, "scene stack bound exceeded");
    size_t rb = (size_t)n * 8 * sizeof(float), hb = (size_t)n * 6 * sizeof(int);
    int rc = ensure_scratch(sc, rb + hb);
    if (rc != RT_OK) return rc;
    float* d_r = static_cast<float*>(sc->scratch);
    int* d_h = reinterpret_cast<int*>(static_cast<char*>(sc->scratch) + rb);
    CUDA_TRY(cudaMemsetAsync(sc->d_err, 0, sizeof(int), sc->stream));
    CUDA_TRY(cudaMemcpyAsync(d_r, rays, rb, cudaMemcpyHostToDevice, sc->stream));
    unsigned g = (unsigned)((n + 127) / 128);
    if (node_layout == 4)
        k_trace_closest<kStack, true><<<g, 128, 0, sc->stream>>>(sc->view, d_r, n, tmin, tmax, d_h, sc->d_err);
    else
        k_trace_closest<kStack, false><<<g, 128, 0, sc->stream>>>(sc->view, d_r, n, tmin, tmax, d_h, sc->d_err);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(hits, d_h, hb, cudaMemcpyDeviceToHost, sc->stream));
    return check_err(sc);
}

int rt_trace_any(RtScene* sc, const float* rays, int64_t n, float* out, int32_t node_layout) {
    if (!sc || !rays || !out || n < 0) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (node_layout != 2 && node_layout != 4) return fail(RT_ERR_INVALID_ARG, "node_layout must be 2 or 4");
    if (n == 0) return RT_OK;
    std::lock_guard<std::mutex> lk(sc->mu);
    CUDA_TRY(cudaSetDevice(sc->device));
    if ((node_layout == 4 ? sc->host.max_stack4 : sc->host.max_stack) > kStack)
        return fail(RT_ERR_STACK, "scene stack bound exceeded");
    size_t rb = (size_t)n * 8 * sizeof(float), ob = (size_t)n * 3 * sizeof(float);
    int rc = ensure_scratch(sc, rb + ob);
    if (rc != RT_OK) return rc;
    float* d_r = static_cast<float*>(sc->scratch);
    float* d_o = reinterpret_cast<float*>(static_cast<char*>(sc->scratch) + rb);
    CUDA_TRY(cudaMemsetAsync(sc->d_err, 0, sizeof(int), sc->stream));
    CUDA_TRY(cudaMemcpyAsync(d_r, rays, rb, cudaMemcpyHostToDevice, sc->stream));
    unsigned g = (unsigned)((n + 127) / 128);
    if (node_layout == 4)
        k_trace_any<kStack, true><<<g, 128, 0, sc->stream>>>(sc->view, sc->opaque, d_r, n, d_o, sc->d_err);
    else
        k_trace_any<kStack, false><<<g, 128, 0, sc->stream>>>(sc->view, sc->opaque, d_r, n, d_o, sc->d_err);
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

int rt_medium_batch(RtScene* sc, const RtMediumQuery* q, int64_t n, RtMediumResult* out) {
    if (!sc || !q || !out || n < 0) return fail(RT_ERR_INVALID_ARG, "null argument");
    if (!sc->host.has_medium) return fail(RT_ERR_INVALID_ARG, "the scene has no participating medium");
    if (n == 0) return RT_OK;
    std::lock_guard<std::mutex> lk(sc->mu);
    CUDA_TRY(cudaSetDevice(sc->device));
    size_t qb = (size_t)n * sizeof(RtMediumQuery), ob = (size_t)n * sizeof(RtMediumResult);
    size_t qb_al = (qb + 255) & ~(size_t)255;
    int rc = ensure_scratch(sc, qb_al + ob);
    if (rc != RT_OK) return rc;
    auto* d_q = static_cast<RtMediumQuery*>(sc->scratch);
    auto* d_o = reinterpret_cast<RtMediumResult*>(static_cast<char*>(sc->scratch) + qb_al);
    CUDA_TRY(cudaMemcpyAsync(d_q, q, qb, cudaMemcpyHostToDevice, sc->stream));
    k_medium<<<(unsigned)((n + 127) / 128), 128, 0, sc->stream>>>(sc->view, d_q, n, d_o);
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

int rt_tonemap(const float* hdr, int32_t width, int32_t height, float exposure_ev, float* rgb) {
    if (!hdr || !rgb || width <= 0 || height <= 0) return fail(RT_ERR_INVALID_ARG, "bad tonemap arguments");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(RT_ERR_NO_DEVICE, "no CUDA device");
    size_t n = (size_t)width * height, b = n * 3 * sizeof(float);
    float* d = nullptr;
    if (cudaMalloc(&d, 2 * b) != cudaSuccess) return fail(RT_ERR_OOM, "allocation failed");
    int rc = RT_OK;
    if (cudaMemcpy(d, hdr, b, cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = fail(RT_ERR_CUDA, "copy failed");
    } else {
        k_tonemap<<<(unsigned)((n + 255) / 256), 256>>>(d, (int)n, powf(2.0f, exposure_ev), d + n * 3);
        if (cudaGetLastError() != cudaSuccess || cudaMemcpy(rgb, d + n * 3, b, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(RT_ERR_CUDA, "tonemap failed");
    }
    cudaFree(d);
    return rc;
}

}  // extern "C"

namespace {

// L2 read bandwidth: every thread streams float4s through L2 only (.cg), a
// grid-stride pass over a buffer small enough to stay L2-resident, several
// times. The sum is written so the loads cannot be dropped.
__global__ void __launch_bounds__(256) k_l2_probe(const float4* buf, int64_t n4, int passes, float* sink) {
    float acc = 0.0f;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int p = 0; p < passes; p++)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
            float4 v = __ldcg(buf + i);
            acc += (v.x + v.y) + (v.z + v.w);
        }
    if (acc == 1.2345678f) sink[0] = acc;   // never true for the zeroed buffer; keeps the loads live
}

}  // namespace

extern "C" {

int rt_probe_l2_bandwidth(int32_t device, int64_t bytes, int32_t passes, double* gbs) {
    if (!gbs || bytes < (1 << 20) || passes < 1) return fail(RT_ERR_INVALID_ARG, "bytes >= 1 MiB and passes >= 1");
    CUDA_TRY(cudaSetDevice(device));
    int64_t n4 = bytes / 16;
    void* mem = nullptr;
    if (cudaMalloc(&mem, (size_t)n4 * 16 + 256) != cudaSuccess) return fail(RT_ERR_OOM, "probe buffer");
    float4* buf = static_cast<float4*>(mem);
    float* sink = reinterpret_cast<float*>(static_cast<char*>(mem) + (size_t)n4 * 16);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = RT_OK;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaMemset(mem, 0, (size_t)n4 * 16 + 256) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess) {
        rc = fail(RT_ERR_CUDA, "probe set-up");
    } else {
        unsigned grid = (unsigned)sms * 8;
        k_l2_probe<<<grid, 256>>>(buf, n4, 1, sink);   // warm: bring the buffer into L2
        cudaEventRecord(e0);
        k_l2_probe<<<grid, 256>>>(buf, n4, passes, sink);
        cudaEventRecord(e1);
        float ms = 0.0f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
            cudaGetLastError() != cudaSuccess)
            rc = fail(RT_ERR_CUDA, "probe run");
        else
            *gbs = (double)n4 * 16.0 * passes / (ms * 1e-3) / 1e9;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(mem);
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
