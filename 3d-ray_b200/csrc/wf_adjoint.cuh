// The replay pass of the path-replay adjoint on the wavefront (WF_REPLAY).
//
// One launch advances every live replayed path by one vertex, in material
// order like k_wf_shade: it runs shade_vertex with the AdjointReplay sink, so
// the vertex's terms and factors turn into parameter gradients exactly as in
// k_adjoint, and the vertex's shadow rays are traced inline (their absorption
// lengths and transmittances feed the NEE gradients of the same vertex). The
// adjoints of the sample's resolve come from the slot's adjoint state, which
// regen filled from the primal record; the interior-absorption material is the
// only part of it a vertex changes.
//
// Gradients gather per thread (per-thread arrays when the parameter vector
// fits kAdjLocal, else shared memory), are summed over the warp and the block,
// and reach the global double accumulators with one atomic per selected slot
// per block.
#pragma once

#include "adjoint.cuh"
#include "wavefront.cuh"

namespace rt {

template <int STACK, bool MEDIUM, bool TRANSMIT>
__global__ void __launch_bounds__(128) k_wf_adjoint(WfArgs a) {
    extern __shared__ float s_acc[];
    const WfAdjoint& J = a.J;
    const int nacc = J.use_local ? J.nact : (J.use_shared ? J.nparams : 0);
    for (int k = threadIdx.x; k < nacc; k += blockDim.x) s_acc[k] = 0.0f;
    float loc[kAdjLocal];
    if (J.use_local)
        for (int k = 0; k < J.nact; k++) loc[J.act[k]] = 0.0f;
    __syncthreads();
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int i = -1;
    if (a.sort) {   // the scatter left the live slots in material order in order[0 .. live)
        if (t < a.ctl->hist[a.nkeys]) i = RT_IX(a.P.order[RT_IX(t, a.nslots)], a.nslots);
    } else if (t < a.nslots) {
        i = t;
    }
    int flags = i >= 0 ? fbits(a.P.d[i].w) : 0;
    if (flags & PF_ALIVE) {
        int req = RT_IX(fbits(a.P.pre[i].w), a.nreq);
        const WfRequest& R = a.reqs[req];
        const SceneView& s = a.views[RT_IX(R.scene, a.nviews)];
        PathState ps;
        int fl, pix;
        wf_load(a, i, R, ps, fl, pix);
        Hit h = wf_hit(a, i);
        AdjointReplay<STACK> adj;
        adj.s = &s;
        adj.params = J.params;
        adj.mmask = J.mmask;
        adj.gmask = J.gmask;
        adj.loc = J.use_local ? loc : nullptr;
        adj.acc = (!J.use_local && J.use_shared) ? s_acc : nullptr;
        adj.gacc = J.grad;
        adj.medium_base = J.medium_base;
        adj.opaque = R.rc.opaque;
        adj.any4 = a.any4;
        adj.err = a.err;
        adj.sh_added = 0;
        adj.sh_n = 0;
        float4* q = J.st + kAdjState * (size_t)i;
        float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4];
        adj.tot_a = v3(q0.x, q0.y, q0.z);
        adj.tot_la = v3(q0.w, q1.x, q1.y);
        adj.g_a = v3(q1.z, q1.w, q2.x);
        adj.g_la = v3(q2.y, q2.z, q2.w);
        adj.g_att0 = v3(q3.x, q3.y, q3.z);
        adj.abs_mat = fbits(q3.w);
        adj.delta = v3(q4.x, q4.y, q4.z);
        adj.val = q4.w;
        adj.max_rad = R.rc.max_rad;
        adj.ind_max = R.rc.ind_max;
        const bool track = MEDIUM && (J.gmask & 0x3Fu);
        if (track) {   // the throughput's log derivatives, 18 floats in q[5 .. 9]
            const float* f = reinterpret_cast<const float*>(q + 5);
            for (int c = 0; c < 3; c++)
                for (int k = 0; k < 6; k++) adj.dlb[c][k] = f[c * 6 + k];
        }
        bool alive = shade_vertex<MEDIUM, TRANSMIT>(s, R.rc, ps, h, adj);
        if (track && alive) {
            float* f = reinterpret_cast<float*>(q + 5);
            for (int c = 0; c < 3; c++)
                for (int k = 0; k < 6; k++) f[c * 6 + k] = adj.dlb[c][k];
        }
        wf_store(a, i, ps, wf_flags(ps, alive), req, pix);
        wf_store_media(a, i, R, ps);
        if (adj.abs_mat != fbits(q3.w)) q[3] = make_float4(q3.x, q3.y, q3.z, ibits(adj.abs_mat));
        if (a.raysort && alive) wf_rank_ray(a, s, ps, i);
    }
    if (J.use_local) {   // warp sums of the per-thread accumulators, then the block's
        const unsigned full = 0xffffffffu;
        int lane = threadIdx.x & 31;
        for (int k = 0; k < J.nact; k++) {
            float v = loc[J.act[k]];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(full, v, o);
            if (lane == 0 && v != 0.0f) atomicAdd(s_acc + k, v);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nacc; k += blockDim.x) {
        float v = s_acc[k];
        if (v != 0.0f) atomicAdd(J.grad + (J.use_local ? J.act[k] : k), (double)v);
    }
}

}  // namespace rt
