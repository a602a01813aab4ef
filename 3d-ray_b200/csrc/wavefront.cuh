// Persistent, request-batched wavefront form of the bounce loop.
//
// A fixed pool of path slots (the wavefront) is advanced one vertex per
// iteration by four small kernels instead of one large one:
//   regen   : resolve finished samples into their request's film, then refill
//             the slot with the next (request, sample, pixel) work item from a
//             global counter (warp-aggregated atomics): camera ray generation.
//   extend  : closest hit of every live path's current ray.
//   shade   : one TraceRay vertex (medium, emission, NEE, BSDF sample, RR).
//             Shadow rays go to a queue instead of being traced inline.
//   occlude : any-hit (or the transparent walk) of the queued shadow rays;
//             visible contributions are added to their path's accumulator.
// The iteration is captured once in a CUDA graph and replayed until every
// request's samples are done. Optional material sorting (a counting sort of
// live slots by material id) feeds shade coherent warps.
//
// Many requests of uneven resolution, spp and depth share the pool: a work id
// maps to (request, sample, pixel) with a binary search over the requests'
// prefix offsets, samples outermost so a warp shares a sample index.
//
// The same loop runs the path-replay adjoint (rt_adjoint) in two passes over
// a range of samples: WF_RECORD renders them with the forward kernels and
// regen stores each finished sample's end state (lp, la, pre, att0) by work id
// instead of adding it to a film; WF_REPLAY traces the same samples again,
// regen seeds each new path with the adjoints of its recorded resolve, and
// k_wf_adjoint (wf_adjoint.cuh) replaces shade and occlude: it runs the vertex
// with the replay's gradient hooks and its shadow rays inline.
#pragma once

#include "adjoint.cuh"
#include "integrator.cuh"

namespace rt {

enum : int {
    PF_ALIVE = 1,       // a ray is in flight
    PF_DONE = 2,        // finished: the sample waits for resolve
    PF_PREV_DELTA = 4,
    PF_FIRST = 8,
    PF_CLAMP = 16,
};

struct WfRequest {
    RenderConst rc;
    int scene;
    int x0, y0, ww, wh;   // render window inside the W x H image
    int spp, spp0;
    long long begin;      // first global work id of this request
    long long count;      // ww * wh * spp
    double* accum;        // 3 * ww * wh: sums of clamped samples (planar, pixels in strip_pixel order).
                          // Double: a float sum of 65 536 samples of one pixel drifts by ~1e-3 of its
                          // value through the rounding of every addition.
};

// SoA path state (144 B per slot + 16 B hit).
struct WfPaths {
    float4* o;      // o.xyz, prev_pdf
    float4* d;      // d.xyz, flags
    float4* beta;   // beta.xyz, depth
    float4* w;      // w.xyz, rng dim
    float4* lp;     // lp.xyz, sample index
    float4* la;     // la.xyz, pixel (lx | ly << 16, window-local)
    float4* pre;    // pre.xyz, request
    float4* att0;   // att0.xyz, la mask (3 bits)
    float4* ab;     // cur_abs.xyz, ior count   (dielectric scenes)
    float* ior;     // 8 per slot                (dielectric scenes)
    float4* hit;    // t, u, v, kind << 30 | slot
    int* order;     // slot order for shade (material-sorted or identity); for extend under the ray sort
    int* keys;      // material key per slot (sorting); after shade, the ray sort's key
    int* rrank;     // ray sort: the slot's rank among the rays of its key
};

struct WfShadow {
    float4* o;    // o.xyz, tmax
    float4* d;    // d.xyz, slot << 1 | to_la
    float4* c;    // contribution.xyz, scene
    int* count;
    int capacity;
    int* key;     // shadow sort: the record's ray_key
    int* rank;    // shadow sort: its rank among the records of its key
    int* order;   // shadow sort: records in key order, for occlude
};

struct WfCtl {
    unsigned long long next;    // next global work id
    unsigned long long total;   // total work ids
    int live;                   // slots alive or done after the last regen
    int overflow;               // shadow queue overflow (never expected: sized by the host)
    // (the host reads next, then live and overflow as one 8-byte copy: keep them adjacent)
    unsigned ext_next;          // persistent extend: next slot to fetch
    unsigned occ_next;          // persistent occlude: next shadow record to fetch
    unsigned long long iter_first;   // ray sort: the first work id of this iteration
    int nbounce;                // ray sort: bounce rays shade continued (order[0 .. nbounce))
    int nshadow;                // shadow sort: records counted by key (the queue's count)
    int hist[256];              // material histogram (sorting)
};

// Buckets of the bounce-ray sort.
constexpr int kRayKeys = 1 << 15;

enum : int { WF_RENDER = 0, WF_RECORD = 1, WF_REPLAY = 2 };
// float4s of a replayed slot's adjoint state: 5 for the resolve adjoints, the
// interior material, the film gradient and the clamped value, then 5 for the
// throughput's log derivatives (dlb) while a medium slot is differentiated
constexpr int kAdjState = 10;

// The adjoint passes' buffers and parameters (zero in WF_RENDER).
struct WfAdjoint {
    float4* rec;            // per work id, 4 float4: {lp, clamp flag}, la, pre, att0 of the finished sample
    long long nrec;         // work ids the record holds
    float4* st;             // per slot, kAdjState float4: the replay's resolve adjoints, interior material,
                            // film gradient and clamped value
    const float* dimg;      // dLoss/dfilm, 3 planes of W x H
    int W, H;
    float inv_spp;          // 1 / the request's spp: the film is the mean of its samples
    const float* params;    // raw parameter vector, 16 per material, then the medium's 6
    const unsigned* mmask;  // per material: bit k = slot k is differentiated
    unsigned gmask;         // the medium's slots
    int nparams, medium_base;
    const int* act;         // the differentiated slots, nact of them
    int nact;
    int use_local;          // gradients gather in per-thread arrays (nparams <= kAdjLocal)
    int use_shared;         // ... otherwise in shared memory (nparams floats), else global atomics
    double* grad;           // nparams accumulators
};

struct WfArgs {
    const SceneView* views;
    int nviews;
    const WfRequest* reqs;
    int nreq;
    int nslots;
    int opaque;       // every scene of the batch is opaque: any-hit shadows
    int sort;
    int nkeys;        // material keys (sum over scenes) for sorting
    const int* key_base;   // per scene: first key
    int regroup;      // extend/occlude regroup their block's rays by kind (block_group)
    int raysort;      // extend walks bounce rays sorted by ray_key, then camera rays in pixel order
    int rkey_bits;    // ray_key of bounce rays: origin cell bits per axis (0 .. 4)
    int rdir_bits;    // ray_key of bounce rays: direction bits (0, 3: octant, or an even count up to 8)
    int skey_bits;    // the same two for shadow records
    int sdir_bits;
    int* rhist;       // kRayKeys: bounce rays per key (filled by shade)
    int* roff;        // kRayKeys: the keys' first positions in order (the scanned histogram)
    int shadowsort;   // occlude walks the shadow records sorted by ray_key
    int* shist;       // kRayKeys: shadow records per key (filled by shade)
    int* soff;        // kRayKeys: the keys' first positions in S.order
    WfPaths P;
    WfShadow S;
    WfCtl* ctl;
    int* err;
    int any4;         // opaque shadow rays may walk the four-wide records (their stack bound fits)
    WfAdjoint J;
};

RT_D int fbits(float f) { return __float_as_int(f); }
RT_D float ibits(int i) { return __int_as_float(i); }

// Warp-aggregated atomic add of 1 per active lane; returns this lane's slot.
RT_D unsigned long long wagg_next(unsigned long long* ctr) {
    unsigned mask = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    int rank = __popc(mask & ((1u << lane) - 1u));
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(ctr, (unsigned long long)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + (unsigned long long)rank;
}
RT_D int wagg_next_int(int* ctr) {
    unsigned mask = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    int rank = __popc(mask & ((1u << lane) - 1u));
    int base = 0;
    if (lane == leader) base = atomicAdd(ctr, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + rank;
}

RT_D void wf_store(const WfArgs& a, int i, const PathState& ps, int flags, int req, int pix) {
    a.P.o[i] = make_float4(ps.o.x, ps.o.y, ps.o.z, ps.prev_pdf);
    a.P.d[i] = make_float4(ps.d.x, ps.d.y, ps.d.z, ibits(flags));
    a.P.beta[i] = make_float4(ps.beta.x, ps.beta.y, ps.beta.z, ibits(ps.depth));
    a.P.w[i] = make_float4(ps.w.x, ps.w.y, ps.w.z, ibits((int)ps.rng.dim));
    a.P.lp[i] = make_float4(ps.lp.x, ps.lp.y, ps.lp.z, ibits((int)ps.rng.index));
    a.P.la[i] = make_float4(ps.la.x, ps.la.y, ps.la.z, ibits(pix));
    a.P.pre[i] = make_float4(ps.pre.x, ps.pre.y, ps.pre.z, ibits(req));
    int mask = (ps.mask.x != 0.0f ? 1 : 0) | (ps.mask.y != 0.0f ? 2 : 0) | (ps.mask.z != 0.0f ? 4 : 0);
    a.P.att0[i] = make_float4(ps.att0.x, ps.att0.y, ps.att0.z, ibits(mask));
}

RT_D int wf_flags(const PathState& ps, int alive) {
    return (alive ? PF_ALIVE : PF_DONE) | (ps.prev_delta ? PF_PREV_DELTA : 0) | (ps.first ? PF_FIRST : 0) |
           (ps.clamp_mode ? PF_CLAMP : 0);
}

// The window's pixels in 8-pixel-wide column strips, rows inside a strip:
// regen hands out work ids in this order, so the 32 camera rays of a warp
// cover an 8x4 block rather than a 32x1 run, and the accumulation buffer is
// laid out the same way, so that the film atomics of consecutive slots stay
// contiguous. The last strip is narrower when ww % 8 != 0.
constexpr int kStripW = 8;   // 4 and 16 measured the same
RT_D void strip_pixel(int p, int ww, int wh, int& lx, int& ly) {
    int strip = p / (kStripW * wh);
    int in = p - strip * kStripW * wh;
    int sw = min(kStripW, ww - kStripW * strip);
    lx = kStripW * strip + in % sw;
    ly = in / sw;
}
RT_D int strip_index(int lx, int ly, int ww, int wh) {
    int strip = lx / kStripW;
    int sw = min(kStripW, ww - kStripW * strip);
    return strip * kStripW * wh + ly * sw + (lx - kStripW * strip);
}

RT_D uint32_t pixel_seed(int px, int py) { return ((uint32_t)px * 73856093u) ^ ((uint32_t)py * 19349663u); }

// Rebuilds the register path state of slot i (lp/la read after occlude).
RT_D void wf_load(const WfArgs& a, int i, const WfRequest& R, PathState& ps, int& flags, int& pix) {
    float4 o = a.P.o[i], d = a.P.d[i], b = a.P.beta[i], w = a.P.w[i], lp = a.P.lp[i], la = a.P.la[i],
           pre = a.P.pre[i], at = a.P.att0[i];
    flags = fbits(d.w);
    pix = fbits(la.w);
    ps.o = v3(o.x, o.y, o.z);
    ps.prev_pdf = o.w;
    ps.d = v3(d.x, d.y, d.z);
    ps.beta = v3(b.x, b.y, b.z);
    ps.depth = fbits(b.w);
    ps.w = v3(w.x, w.y, w.z);
    ps.lp = v3(lp.x, lp.y, lp.z);
    ps.la = v3(la.x, la.y, la.z);
    ps.pre = v3(pre.x, pre.y, pre.z);
    ps.att0 = v3(at.x, at.y, at.z);
    int mask = fbits(at.w);
    ps.mask = v3((mask & 1) ? 1.0f : 0.0f, (mask & 2) ? 1.0f : 0.0f, (mask & 4) ? 1.0f : 0.0f);
    ps.prev_delta = (flags & PF_PREV_DELTA) != 0;
    ps.first = (flags & PF_FIRST) != 0;
    ps.clamp_mode = (flags & PF_CLAMP) != 0;
    int lx = pix & 0xFFFF, ly = pix >> 16;
    ps.rng = Sampler{pixel_seed(R.x0 + lx, R.y0 + ly), (uint32_t)fbits(lp.w), (uint32_t)fbits(w.w)};
    ps.cur_abs = v3(0.0f);
    ps.iors.n = 0;
    if (R.rc.dielectrics) {
        float4 ab = a.P.ab[i];
        ps.cur_abs = v3(ab.x, ab.y, ab.z);
        ps.iors.n = fbits(ab.w);
        for (int k = 0; k < 8; k++) ps.iors.slot[k] = a.P.ior[(size_t)i * 8 + k];
    }
}

RT_D void wf_store_media(const WfArgs& a, int i, const WfRequest& R, const PathState& ps) {
    if (!R.rc.dielectrics) return;
    a.P.ab[i] = make_float4(ps.cur_abs.x, ps.cur_abs.y, ps.cur_abs.z, ibits(ps.iors.n));
    for (int k = 0; k < 8; k++) a.P.ior[(size_t)i * 8 + k] = ps.iors.slot[k];
}

RT_D int find_request(const WfRequest* reqs, int n, unsigned long long id) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if ((unsigned long long)reqs[mid].begin <= id) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_wf_regen(WfArgs a) {
    // Work ids come from the global counter with one atomic per block (a
    // ballot prefix over the block's free slots), and the live count with one
    // more: a per-warp atomic on one address serialised in L2.
    __shared__ int s_warp[8];   // blockDim 256: per-warp free-slot offsets
    __shared__ unsigned long long s_base;
    __shared__ int s_live;
    const unsigned full = 0xffffffffu;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    bool in = i < a.nslots;
    int flags = in ? fbits(a.P.d[i].w) : 0;
    bool alive = in && (flags & PF_ALIVE);
    bool need = in && !alive;
    if (MODE == WF_RECORD && need && (flags & PF_DONE)) {   // keep the finished sample's end state
        float4 lp = a.P.lp[i], la = a.P.la[i], pre = a.P.pre[i], at = a.P.att0[i];
        const WfRequest& R = a.reqs[RT_IX(fbits(pre.w), a.nreq)];
        int pix = fbits(la.w);
        int lx = pix & 0xFFFF, ly = pix >> 16;
        long long id = R.begin + (long long)(fbits(lp.w) - R.spp0) * ((long long)R.ww * R.wh) +
                       strip_index(lx, ly, R.ww, R.wh);
        if (id >= 0 && id < a.J.nrec) {
            float4* r = a.J.rec + 4 * id;
            r[0] = make_float4(lp.x, lp.y, lp.z, ibits(flags & PF_CLAMP));
            r[1] = la;
            r[2] = pre;
            r[3] = at;
        } else {
            atomicExch(a.err, RT_ERR_BOUNDS);
        }
    }
    if (MODE == WF_RENDER && need && (flags & PF_DONE)) {   // resolve the finished sample into its film
        // path_resolve reads lp, la, pre, att0 and the clamp flag alone: load
        // those four records, not the whole path state
        float4 lp = a.P.lp[i], la = a.P.la[i], pre = a.P.pre[i], at = a.P.att0[i];
        int req = RT_IX(fbits(pre.w), a.nreq);
        const WfRequest& R = a.reqs[req];
        PathState ps;
        ps.lp = v3(lp.x, lp.y, lp.z);
        ps.la = v3(la.x, la.y, la.z);
        ps.pre = v3(pre.x, pre.y, pre.z);
        ps.att0 = v3(at.x, at.y, at.z);
        ps.clamp_mode = (flags & PF_CLAMP) != 0;
        int pix = fbits(la.w);
        V3 L = path_resolve(ps, R.rc);
        int lx = pix & 0xFFFF, ly = pix >> 16;
        size_t plane = (size_t)R.ww * R.wh, k = (size_t)RT_IX(strip_index(lx, ly, R.ww, R.wh), plane);
        atomicAdd(R.accum + k, (double)L.x);
        atomicAdd(R.accum + plane + k, (double)L.y);
        atomicAdd(R.accum + 2 * plane + k, (double)L.z);
    }
    unsigned m = __ballot_sync(full, need);
    if (lane == 0) s_warp[wid] = __popc(m);
    if (threadIdx.x == 0) s_live = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            int c = s_warp[w];
            s_warp[w] = tot;
            tot += c;
        }
        s_base = tot ? atomicAdd(&a.ctl->next, (unsigned long long)tot) : 0ull;
    }
    __syncthreads();
    bool live = alive;
    if (alive && a.raysort) {
        // a bounce ray shade continued: its key's first position plus the rank
        // shade's count gave it
        int pos = a.roff[RT_IX(a.P.keys[i], kRayKeys)] + a.P.rrank[i];
        if (pos < a.ctl->nbounce) a.P.order[pos] = i;
        else atomicExch(a.err, RT_ERR_BOUNDS);
    }
    if (need) {
        unsigned long long id = s_base + (unsigned long long)(s_warp[wid] + __popc(m & ((1u << lane) - 1u)));
        if (id >= a.ctl->total) {
            a.P.d[i].w = ibits(0);
        } else {
            int req = RT_IX(find_request(a.reqs, a.nreq, id), a.nreq);
            const WfRequest& R = a.reqs[req];
            long long local = (long long)(id - (unsigned long long)R.begin);
            long long npix = (long long)R.ww * R.wh;
            int s = (int)(local / npix);
            int p = (int)(local % npix);
            int lx, ly;
            strip_pixel(p, R.ww, R.wh, lx, ly);
            PathState ps;
            path_init(ps, R.rc, R.x0 + lx, R.y0 + ly, (uint32_t)(R.spp0 + s));
            int al = path_alive(ps);
            if (MODE == WF_REPLAY) {   // the adjoints of the recorded resolve; no gradient, no replay
                const WfAdjoint& J = a.J;
                size_t plane = (size_t)J.W * J.H, fi = (size_t)(R.y0 + ly) * J.W + (R.x0 + lx);
                V3 delta = v3(J.dimg[fi], J.dimg[plane + fi], J.dimg[2 * plane + fi]) * J.inv_spp;
                AdjResolve ar{};
                if (id < (unsigned long long)J.nrec && !is_zero(delta)) {
                    const float4* r = J.rec + 4 * id;
                    float4 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3];
                    ar = adjoint_resolve(R.rc, v3(r0.x, r0.y, r0.z), v3(r1.x, r1.y, r1.z), v3(r2.x, r2.y, r2.z),
                                         v3(r3.x, r3.y, r3.z), fbits(r0.w) != 0, delta);
                }
                al = al && !is_zero(ar.g_a);
                float4* q = J.st + kAdjState * (size_t)i;
                q[0] = make_float4(ar.tot_a.x, ar.tot_a.y, ar.tot_a.z, ar.tot_la.x);
                q[1] = make_float4(ar.tot_la.y, ar.tot_la.z, ar.g_a.x, ar.g_a.y);
                q[2] = make_float4(ar.g_a.z, ar.g_la.x, ar.g_la.y, ar.g_la.z);
                q[3] = make_float4(ar.g_att0.x, ar.g_att0.y, ar.g_att0.z, ibits(-1));
                q[4] = make_float4(ar.delta.x, ar.delta.y, ar.delta.z, ar.val);
                if (J.gmask & 0x3Fu)
                    for (int k = 5; k < kAdjState; k++) q[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
            wf_store(a, i, ps, wf_flags(ps, al), req, lx | (ly << 16));
            wf_store_media(a, i, R, ps);
            live = true;
            if (a.raysort) {   // camera rays after the bounce rays, in work-id (pixel) order
                long long pos = (long long)a.ctl->nbounce + (long long)(id - a.ctl->iter_first);
                if (pos < a.nslots) a.P.order[pos] = al ? i : -1;
                else atomicExch(a.err, RT_ERR_BOUNDS);
            }
        }
    }
    int wl = __popc(__ballot_sync(full, live));
    if (lane == 0 && wl) atomicAdd(&s_live, wl);
    __syncthreads();
    if (threadIdx.x == 0 && s_live) atomicAdd(&a.ctl->live, s_live);
}

// Block-local counting partition; blockDim.x is a multiple of 32, at most 256,
// and every thread of the block calls it. Each thread offers one item of class
// cls (cls < 0: none). On return s_idx[0 .. n) holds the block's items ordered
// by class, in thread order within a class, and n is returned.
template <int NC>
RT_D int block_group(int item, int cls, int* s_idx, int (*s_cnt)[8], int* s_tot) {
    static_assert(NC <= 32, "one class per lane of the scanning warp");
    const unsigned full = 0xffffffffu;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned mine = 0;
#pragma unroll
    for (int c = 0; c < NC; c++) {
        unsigned m = __ballot_sync(full, cls == c);
        if (cls == c) mine = m;
        if (lane == 0) s_cnt[c][wid] = __popc(m);
    }
    __syncthreads();
    if (wid == 0) {
        // lane c: the class's count, an exclusive scan over the classes, then
        // the running offsets of its warps (class-major order)
        int sum = 0;
        if (lane < NC)
            for (int w = 0; w < nw; w++) sum += s_cnt[lane][w];
        int incl = sum;
        for (int off = 1; off < 32; off <<= 1) {
            int v = __shfl_up_sync(full, incl, off);
            if (lane >= off) incl += v;
        }
        int run = incl - sum;
        if (lane < NC)
            for (int w = 0; w < nw; w++) {
                int c = s_cnt[lane][w];
                s_cnt[lane][w] = run;
                run += c;
            }
        if (lane == 31) *s_tot = incl;   // lanes past NC add nothing: lane 31 holds the total
    }
    __syncthreads();
    if (cls >= 0) s_idx[s_cnt[cls][wid] + __popc(mine & ((1u << lane) - 1u))] = item;
    __syncthreads();
    return *s_tot;
}

RT_D int octant(float x, float y, float z) { return (x < 0.0f) | ((y < 0.0f) << 1) | ((z < 0.0f) << 2); }

// Spreads the low 4 bits of v to bits 0, 3, 6, 9 (a Morton code's axis).
RT_D unsigned spread3(unsigned v) { return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4) | ((v & 8u) << 6); }

// Sort key of a bounce ray (0 .. kRayKeys): the origin's cell in the scene's
// sort box, cb bits per axis in Morton order, above a direction bin of db
// bits: none, the octant for 3, else a square grid over the octahedral map of
// the direction. Rays that share a key start close together in similar
// directions, so they walk much the same BVH nodes.
RT_D int ray_key(const SceneView& s, V3 o, V3 d, int cb, int db) {
    unsigned cell = 0;
    if (cb > 0) {
        float n = (float)(1 << cb);
        V3 u = (o - s.sort_lo) * s.sort_scale;
        unsigned cx = (unsigned)fminf(fmaxf(u.x * n, 0.0f), n - 1.0f);
        unsigned cy = (unsigned)fminf(fmaxf(u.y * n, 0.0f), n - 1.0f);
        unsigned cz = (unsigned)fminf(fmaxf(u.z * n, 0.0f), n - 1.0f);
        cell = spread3(cx) | (spread3(cy) << 1) | (spread3(cz) << 2);
    }
    unsigned dir = 0;
    if (db == 3) {
        dir = (unsigned)octant(d.x, d.y, d.z);
    } else if (db > 0) {
        // octahedral map of the direction onto [-1, 1]^2
        float l1 = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
        float px = l1 > 0.0f ? d.x / l1 : 0.0f, py = l1 > 0.0f ? d.y / l1 : 0.0f;
        if (d.z < 0.0f) {
            float qx = (1.0f - fabsf(py)) * (px < 0.0f ? -1.0f : 1.0f);
            float qy = (1.0f - fabsf(px)) * (py < 0.0f ? -1.0f : 1.0f);
            px = qx;
            py = qy;
        }
        float g = (float)(1 << (db / 2));
        unsigned gx = (unsigned)fminf(fmaxf((px * 0.5f + 0.5f) * g, 0.0f), g - 1.0f);
        unsigned gy = (unsigned)fminf(fmaxf((py * 0.5f + 0.5f) * g, 0.0f), g - 1.0f);
        dir = gx | (gy << (db / 2));
    }
    return (int)((cell << db) | dir) & (kRayKeys - 1);
}

// Stores slot i's closest hit and, when sorting, its material key.
RT_D void extend_store(const WfArgs& a, int i, int req, const SceneView& s, const Hit& h) {
    int packed = h.kind == HIT_NONE ? 0 : ((h.kind << 30) | h.slot);
    a.P.hit[i] = make_float4(h.t, h.u, h.v, ibits(packed));
    if (a.sort) {   // material key for the counting sort
        int key = a.nkeys;   // misses and emitters sort last
        if (h.kind != HIT_NONE) {
            int ent = h.kind == HIT_TRI ? s.tri_entity[RT_IX(h.slot, s.n_tris)] : h.slot;
            key = RT_IX(a.key_base[a.reqs[req].scene] + s.entities[RT_IX(ent, s.n_entities)].material, a.nkeys);
        }
        a.P.keys[i] = key;
        // one atomic per distinct key in the warp (__match_any_sync groups lanes)
        unsigned grp = __match_any_sync(__activemask(), key);
        if ((int)(threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&a.ctl->hist[key], __popc(grp));
    }
}

// One thread per slot.
// One thread per slot. With regroup, the block first reorders its live slots:
// camera rays, then bounce rays by direction octant. Regen hands a block's free
// slots consecutive pixels, so its camera rays are coherent, but they sit
// between the bounce rays of paths still in flight; regrouped, a warp holds
// one kind of ray and no longer waits on its slowest bounce ray.
// The register budget of 5 blocks of 256 (48 registers) lets 10 blocks of the
// autotuned 128 threads share an SM instead of 9: extend -2.5% per 64-spp
// icosphere frame, for an 8-byte spill.
template <int STACK, bool L4>
__global__ void __launch_bounds__(256, 5) k_wf_extend(WfArgs a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (a.raysort) {
        // order[0 .. nbounce): bounce rays by key; then this iteration's camera rays
        unsigned long long nx = a.ctl->next < a.ctl->total ? a.ctl->next : a.ctl->total;
        long long ncam = (long long)nx - (long long)a.ctl->iter_first;
        long long n = (long long)a.ctl->nbounce + (ncam > 0 ? ncam : 0);
        if ((long long)i >= n || i >= a.nslots) return;
        i = a.P.order[i];
        if (i < 0) return;
        i = RT_IX(i, a.nslots);
    } else if (a.regroup) {
        __shared__ int s_idx[256], s_cnt[9][8], s_tot;
        int cls = -1;
        if (i < a.nslots) {
            float4 d = a.P.d[i];
            int fl = fbits(d.w);
            if (fl & PF_ALIVE) cls = (fl & PF_FIRST) ? 0 : 1 + octant(d.x, d.y, d.z);
        }
        int n = block_group<9>(i, cls, s_idx, s_cnt, &s_tot);
        if ((int)threadIdx.x >= n) return;
        i = s_idx[threadIdx.x];
    } else if (i >= a.nslots) {
        return;
    }
    float4 d = a.P.d[i];
    if (!(fbits(d.w) & PF_ALIVE)) return;
    float4 o = a.P.o[i];
    int req = RT_IX(fbits(a.P.pre[i].w), a.nreq);
    const SceneView& s = a.views[RT_IX(a.reqs[req].scene, a.nviews)];
    Hit h;
    trace<false, STACK, L4>(s, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), kEps, kInf, h, nullptr, a.err);
    extend_store(a, i, req, s, h);
}

// Persistent form with dynamic ray fetch (Aila and Laine 2009): a grid sized
// to fill the GPU once walks rays in rounds (Walker::step). Between rounds,
// once kRefill lanes of a warp have finished (or all of them), the finished
// lanes take the next slots from a global counter, so a few long rays no
// longer keep a warp whose other lanes are done. The rays, their walks and
// their results are those of the one-thread-per-slot kernel.
constexpr int kRefill = 8;

template <int STACK>
__global__ void __launch_bounds__(256) k_wf_extend_pt(WfArgs a) {
    const unsigned full = 0xffffffffu;
    int lane = threadIdx.x & 31;
    Walker<false, STACK> w;
    int slot = -1, req = 0;
    bool exhausted = false;
    for (;;) {
        bool idle = slot < 0 && !exhausted;
        unsigned need = __ballot_sync(full, idle);
        unsigned busy = __ballot_sync(full, slot >= 0);
        if (!need && !busy) break;
        if (need && (__popc(need) >= kRefill || !busy)) {
            int leader = __ffs(need) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(&a.ctl->ext_next, (unsigned)__popc(need));
            base = __shfl_sync(full, base, leader);
            if (idle) {
                unsigned i = base + (unsigned)__popc(need & ((1u << lane) - 1u));
                if (i >= (unsigned)a.nslots) {
                    exhausted = true;
                } else {
                    float4 d = a.P.d[i];
                    if (fbits(d.w) & PF_ALIVE) {
                        float4 o = a.P.o[i];
                        req = RT_IX(fbits(a.P.pre[i].w), a.nreq);
                        slot = (int)i;
                        w.start(a.views[RT_IX(a.reqs[req].scene, a.nviews)], v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), kEps, kInf,
                                nullptr, false, 0);
                    }
                }
            }
            continue;
        }
        if (slot >= 0) {
            const SceneView& s = a.views[RT_IX(a.reqs[req].scene, a.nviews)];
            if (w.step(s, nullptr, a.err)) {
                extend_store(a, slot, req, s, w.best);
                slot = -1;
            }
        }
    }
}

// Exclusive scan of the material histogram (one block) and the scatter of
// live slots into material order.
__global__ void k_wf_scan(WfArgs a) {
    __shared__ int s[257];
    int t = threadIdx.x;
    if (t <= a.nkeys) s[t] = a.ctl->hist[t];
    __syncthreads();
    if (t == 0) {
        int acc = 0;
        for (int k = 0; k <= a.nkeys; k++) {
            int c = s[k];
            s[k] = acc;
            acc += c;
        }
    }
    __syncthreads();
    if (t <= a.nkeys) a.ctl->hist[t] = s[t];
}
__global__ void k_wf_scatter(WfArgs a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nslots) return;
    if (!(fbits(a.P.d[i].w) & PF_ALIVE)) return;
    int key = RT_IX(a.P.keys[i], a.nkeys + 1);
    unsigned grp = __match_any_sync(__activemask(), key);
    int lane = threadIdx.x & 31;
    int leader = __ffs(grp) - 1;
    int rank = __popc(grp & ((1u << lane) - 1u));
    int base = 0;
    if (lane == leader) base = atomicAdd(&a.ctl->hist[key], __popc(grp));
    base = __shfl_sync(grp, base, leader);
    a.P.order[RT_IX(base + rank, a.nslots)] = i;
}

// Shadow sink of the wavefront: queue the ray with its contribution.
// Shadow sink of the wavefront: queue the ray with its contribution.
struct QueueShadows : NoAdjoint {
    const WfArgs* a;
    int slot;
    int scene;
    RT_D void shadow(PathState& ps, V3 o, V3 d, float tmax, V3 c, int to_la) {
        if (!isfinite(c.x) || !isfinite(c.y) || !isfinite(c.z)) {
            ps.add(c, to_la);   // records the per-frame sanitize in the mask
            return;
        }
        int j = wagg_next_int(a->S.count);
        if (j >= a->S.capacity) {
            atomicExch(&a->ctl->overflow, 1);
            return;
        }
        a->S.o[j] = make_float4(o.x, o.y, o.z, tmax);
        a->S.d[j] = make_float4(d.x, d.y, d.z, ibits((slot << 1) | to_la));
        a->S.c[j] = make_float4(c.x, c.y, c.z, ibits(scene));
        if (a->shadowsort) {   // the record's sort key and its rank in the key's count
            int key = ray_key(a->views[scene], o, d, a->skey_bits, a->sdir_bits);
            unsigned grp = __match_any_sync(__activemask(), key);
            int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&a->shist[key], __popc(grp));
            base = __shfl_sync(grp, base, leader);
            a->S.key[j] = key;
            a->S.rank[j] = base + __popc(grp & ((1u << lane) - 1u));
        }
    }
    RT_D void skipped(V3, V3, float) {}
};

// Under the ray sort: the continued ray's sort key and its rank in the key's
// count (one returning atomic per distinct key in the warp).
RT_D void wf_rank_ray(const WfArgs& a, const SceneView& s, const PathState& ps, int i) {
    int key = ray_key(s, ps.o, ps.d, a.rkey_bits, a.rdir_bits);
    unsigned grp = __match_any_sync(__activemask(), key);
    int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&a.rhist[key], __popc(grp));
    base = __shfl_sync(grp, base, leader);
    a.P.keys[i] = key;
    a.P.rrank[i] = base + __popc(grp & ((1u << lane) - 1u));
}

// Hit record of slot i as extend wrote it.
RT_D Hit wf_hit(const WfArgs& a, int i) {
    float4 hh = a.P.hit[i];
    int packed = fbits(hh.w);
    Hit h;
    h.t = hh.x;
    h.u = hh.y;
    h.v = hh.z;
    h.kind = packed == 0 ? HIT_NONE : ((unsigned)packed >> 30);
    h.slot = packed & 0x3FFFFFFF;
    return h;
}

// Minimum resident blocks of 256 for shade (a register budget); a build knob.
#ifndef RT_SHADE_MIN_BLOCKS
#define RT_SHADE_MIN_BLOCKS 2
#endif
template <bool MEDIUM, bool TRANSMIT>
__global__ void __launch_bounds__(256, RT_SHADE_MIN_BLOCKS) k_wf_shade(WfArgs a) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int i;
    if (a.sort) {
        // the scatter left the live slots in material order in order[0 .. live)
        if (t >= a.ctl->hist[a.nkeys]) return;
        i = RT_IX(a.P.order[RT_IX(t, a.nslots)], a.nslots);
    } else {
        if (t >= a.nslots) return;
        i = t;
    }
    float4 d4 = a.P.d[i];
    int flags = fbits(d4.w);
    if (!(flags & PF_ALIVE)) return;
    int req = RT_IX(fbits(a.P.pre[i].w), a.nreq);
    const WfRequest& R = a.reqs[req];
    const SceneView& s = a.views[RT_IX(R.scene, a.nviews)];
    PathState ps;
    int fl, pix;
    wf_load(a, i, R, ps, fl, pix);
    Hit h = wf_hit(a, i);
    QueueShadows sink{{}, &a, i, R.scene};
    bool alive = shade_vertex<MEDIUM, TRANSMIT>(s, R.rc, ps, h, sink);
    wf_store(a, i, ps, wf_flags(ps, alive), req, pix);
    wf_store_media(a, i, R, ps);
    if (a.raysort && alive) wf_rank_ray(a, s, ps, i);
}

// Exclusive scan of a ray-sort key histogram (kRayKeys counts) into off (one
// block of 1024 threads, a run of kRayKeys / 1024 keys each), clearing the
// histogram for the next shade; *total receives the sum.
__global__ void __launch_bounds__(1024) k_wf_rscan(int* hist, int* off, int* total) {
    constexpr int kPer = kRayKeys / 1024;
    static_assert(kPer % 4 == 0, "whole int4 runs per thread");
    __shared__ int s_w[32];
    const unsigned full = 0xffffffffu;
    int t = threadIdx.x, lane = t & 31, w = t >> 5;
    int4* h4 = reinterpret_cast<int4*>(hist) + t * (kPer / 4);
    int4* o4 = reinterpret_cast<int4*>(off) + t * (kPer / 4);
    int4 v[kPer / 4];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kPer / 4; k++) {
        v[k] = h4[k];
        sum += v[k].x + v[k].y + v[k].z + v[k].w;
    }
    int incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        int x = __shfl_up_sync(full, incl, o);
        if (lane >= o) incl += x;
    }
    if (lane == 31) s_w[w] = incl;
    __syncthreads();
    if (w == 0) {
        int x = s_w[lane];
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(full, x, o);
            if (lane >= o) x += y;
        }
        s_w[lane] = x;
    }
    __syncthreads();
    int base = (w ? s_w[w - 1] : 0) + incl - sum;
#pragma unroll
    for (int k = 0; k < kPer / 4; k++) {
        int4 r;
        r.x = base;
        r.y = r.x + v[k].x;
        r.z = r.y + v[k].y;
        r.w = r.z + v[k].z;
        base = r.w + v[k].w;
        o4[k] = r;
        h4[k] = make_int4(0, 0, 0, 0);
    }
    if (t == 1023) *total = base;
}

// Shadow sort: each queued record goes to its key's offset plus its rank.
__global__ void k_wf_sscatter(WfArgs a) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    int n = min(*a.S.count, a.S.capacity);
    if (j >= n) return;
    int pos = a.soff[RT_IX(a.S.key[j], kRayKeys)] + a.S.rank[j];
    if (pos < n) a.S.order[pos] = j;
    else atomicExch(a.err, RT_ERR_BOUNDS);
}

// Persistent any-hit for opaque batches (the walk is one any-hit traversal):
// the dynamic-fetch scheme of k_wf_extend_pt over the shadow queue.
template <int STACK>
__global__ void __launch_bounds__(256) k_wf_occlude_pt(WfArgs a) {
    const unsigned full = 0xffffffffu;
    int lane = threadIdx.x & 31;
    int n = min(*a.S.count, a.S.capacity);
    Walker<true, STACK> w;
    int rec = -1;
    bool exhausted = false;
    for (;;) {
        bool idle = rec < 0 && !exhausted;
        unsigned need = __ballot_sync(full, idle);
        unsigned busy = __ballot_sync(full, rec >= 0);
        if (!need && !busy) break;
        if (need && (__popc(need) >= kRefill || !busy)) {
            int leader = __ffs(need) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(&a.ctl->occ_next, (unsigned)__popc(need));
            base = __shfl_sync(full, base, leader);
            if (idle) {
                unsigned j = base + (unsigned)__popc(need & ((1u << lane) - 1u));
                if (j >= (unsigned)n) {
                    exhausted = true;
                } else {
                    float4 o = a.S.o[j], d = a.S.d[j], c = a.S.c[j];
                    rec = (int)j;
                    w.start(a.views[RT_IX(fbits(c.w), a.nviews)], v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), kEps, o.w, nullptr, false, 0);
                }
            }
            continue;
        }
        if (rec >= 0) {
            float4 c = a.S.c[rec];
            if (w.step(a.views[RT_IX(fbits(c.w), a.nviews)], nullptr, a.err)) {
                if (w.best.kind == HIT_NONE) {   // visible: transmittance 1
                    int packed = fbits(a.S.d[rec].w);
                    int slot = RT_IX(packed >> 1, a.nslots);
                    float4* dst = (packed & 1) ? (a.P.la + slot) : (a.P.lp + slot);
                    float* f = reinterpret_cast<float*>(dst);
                    atomicAdd(f, c.x);
                    atomicAdd(f + 1, c.y);
                    atomicAdd(f + 2, c.z);
                }
                rec = -1;
            }
        }
    }
}

// OPAQUE: a batch with no transmissive material, whose shadow rays are any-hit
// walks. That variant has a register budget of 5 blocks of 256 (48 registers):
// 10 blocks of the autotuned 128 threads per SM instead of 8, occlude -7.8%
// per 64-spp icosphere frame. The transparent variant keeps the full budget
// its longer walk needs.
template <int STACK, bool L4, bool OPAQUE>
__global__ void __launch_bounds__(256, OPAQUE ? 5 : 1) k_wf_occlude(WfArgs a) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    int n = min(*a.S.count, a.S.capacity);
    if (a.shadowsort) {
        if (j >= n) return;
        j = RT_IX(a.S.order[j], n);
    } else if (a.regroup) {
        // shadow rays by direction octant (blocks wholly past the queue leave at once)
        if ((int)(blockIdx.x * blockDim.x) >= n) return;
        __shared__ int s_idx[256], s_cnt[8][8], s_tot;
        int cls = -1;
        if (j < n) {
            float4 d = a.S.d[j];
            cls = octant(d.x, d.y, d.z);
        }
        int m = block_group<8>(j, cls, s_idx, s_cnt, &s_tot);
        if ((int)threadIdx.x >= m) return;
        j = s_idx[threadIdx.x];
    } else if (j >= n) {
        return;
    }
    float4 o = a.S.o[j], d = a.S.d[j], c = a.S.c[j];
    const SceneView& s = a.views[RT_IX(fbits(c.w), a.nviews)];
    V3 tr = shadow_transmittance<STACK, L4>(s, OPAQUE ? 1 : a.opaque, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), kEps,
                                            o.w, nullptr, a.err);
    if (near_zero(tr)) return;
    int packed = fbits(d.w);
    int slot = RT_IX(packed >> 1, a.nslots);
    V3 v = v3(c.x, c.y, c.z) * tr;
    float4* dst = (packed & 1) ? (a.P.la + slot) : (a.P.lp + slot);
    float* f = reinterpret_cast<float*>(dst);
    atomicAdd(f, v.x);
    atomicAdd(f + 1, v.y);
    atomicAdd(f + 2, v.z);
}

// Per-iteration reset of the counters the next iteration accumulates.
__global__ void k_wf_reset(WfArgs a) {
    int t = threadIdx.x;
    if (t == 0) {
        *a.S.count = 0;
        a.ctl->live = 0;
        a.ctl->ext_next = 0;
        a.ctl->occ_next = 0;
        a.ctl->iter_first = a.ctl->next;
    }
    if (a.sort)
        for (int k = t; k <= a.nkeys; k += blockDim.x) a.ctl->hist[k] = 0;
}

// Mean of the accumulated sums into the films (Renderer.cs:711).
__global__ void k_wf_finalize(const WfRequest* reqs, int nreq, float* const* films, const int* film_w,
                              const int* film_h) {
    int r = blockIdx.y;
    if (r >= nreq) return;
    const WfRequest& R = reqs[r];
    long long plane = (long long)R.ww * R.wh;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        int lx, ly;
        strip_pixel((int)i, R.ww, R.wh, lx, ly);   // the accumulation buffer is in strip order
        size_t fp = (size_t)film_w[r] * film_h[r];
        size_t fi = (size_t)(R.y0 + ly) * film_w[r] + (R.x0 + lx);
        for (int c = 0; c < 3; c++) films[r][c * fp + fi] = (float)(R.accum[c * plane + i] / (double)R.spp);
    }
}

}  // namespace rt
