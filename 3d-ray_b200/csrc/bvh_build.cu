// Device binned-SAH build of mesh BVHs: node for node, and item for item in
// leaf order, the trees the host build (and BvhNode's constructor,
// Acceleration/BvhNode.cs:91-364) makes for the same triangles.
//
// All meshes of a world are built together. Positions 0..N-1 hold the
// triangles of mesh 0, then mesh 1, ...; a node owns a contiguous range of
// positions, as in the host's in-place recursion.
//
// Large nodes (more than kSmall triangles) are split level by level, all
// nodes of a level at once:
//   k_bounds   node box and centroid bounds per node (warp-segmented min/max,
//              then atomics; min/max are exact in any order);
//   k_bins     16 bins per axis per node (count and box);
//   k_split    one thread per node evaluates the planes with sah_eval_axis,
//              the host's own code, so the choice and the costs are the same
//              floats;
//   k_flags    each triangle's side; an exclusive scan ranks the left ones;
//   k_ptr_*    the right items' order. The host partition swaps each left
//              item with the first right one, so right items rotate like a
//              queue. Writing T[p] for what position p holds once the swap at
//              p is done, a left item with left-rank r gives T[p] = T[start + r]
//              and a right item is its own source, so every final right
//              position resolves its source by following p -> start + r(p);
//              pointer jumping does that in log2(span) rounds;
//   k_scatter  writes both children's ranges.
// Nodes of at most kSmall triangles are built whole by one thread each with
// sah_split, the host's own partition, in place. Levels give BFS node ids;
// subtree sizes (bottom-up) then give every node its pre-order index, which
// is the host's node order.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "sah.h"
#include "world.h"

namespace rt {
namespace {

constexpr int kSmall = 32;        // nodes of at most this many triangles: one thread builds the subtree
constexpr int kAccA = 12;         // per node: box min xyz, box max xyz, centroid min xyz, centroid max xyz
constexpr int kBinsAll = 3 * kSahBins;

// Order-preserving map of floats to ints, so atomicMin/atomicMax on the ints
// give the float min/max (the boxes hold no NaN and no -0: tri_box never
// produces a -0, and non-finite vertices are rejected).
__device__ __forceinline__ int f2o(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

struct BuildCtl {
    int next_act;     // large nodes of the next level
    int small;        // small subtree roots so far
    int max_span;     // largest span of the next level's large nodes
    int bad_vertex;   // a vertex coordinate is not finite
};

struct SplitInfo {
    int start, end, mid;
    int mode;         // 0 partition, 1 keep the order (median split)
    int axis, bin;
    float c0, scale;
};

struct Buffers {
    int n = 0, meshes = 0;
    float4* blo = nullptr;       // per triangle (batch id = its position before the build)
    float4* bhi = nullptr;
    float4* cen = nullptr;
    int* idx[2] = {nullptr, nullptr};
    int* seg[2] = {nullptr, nullptr};
    int* ptr[2] = {nullptr, nullptr};
    int* flag = nullptr;
    int* rank = nullptr;
    int* order = nullptr;        // final leaf order (written when a node becomes small)
    int* acc_a = nullptr;        // [S][12]
    int* acc_c = nullptr;        // [S][48]
    int* acc_b = nullptr;        // [S][48][6]
    SplitInfo* split = nullptr;  // [S]
    int* seg_next = nullptr;     // [2S]: a child's large-node index in the next level, or -1
    // nodes (BFS ids)
    int* n_start = nullptr;
    int* n_end = nullptr;
    int* n_mesh = nullptr;
    int* n_level = nullptr;
    int* n_child = nullptr;      // first child's id (the second is +1); -1 for a small root
    int* n_axis = nullptr;
    float4* n_lo = nullptr;
    float4* n_hi = nullptr;
    int* n_size = nullptr;
    int* n_pre = nullptr;
    int* act = nullptr;          // large nodes, level after level
    int* small = nullptr;        // small subtree roots
    NodeF* tmp = nullptr;        // small subtrees in pre-order, at 2 * start
    NodeF* out = nullptr;        // every mesh's nodes, mesh after mesh
    int* mesh_pos = nullptr;     // per mesh: first position
    int* mesh_depth = nullptr;
    int* mesh_base = nullptr;    // per mesh: first output node
    BuildCtl* ctl = nullptr;
    char* scan_tmp = nullptr;
    size_t scan_bytes = 0;
};

// --- triangle boxes -----------------------------------------------------------
__global__ void k_boxes(int n, const float* __restrict__ verts, float4* blo, float4* bhi, float4* cen,
                        BuildCtl* ctl) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* p = verts + (size_t)t * 9;
    float v[9];
    bool ok = true;
    for (int k = 0; k < 9; k++) {
        v[k] = p[k];
        ok = ok && isfinite(v[k]);
    }
    if (!ok) atomicExch(&ctl->bad_vertex, 1);
    Box b = tri_box(v3(v[0], v[1], v[2]), v3(v[3], v[4], v[5]), v3(v[6], v[7], v[8]));
    V3 c = box_centroid(b);
    blo[t] = make_float4(b.mn.x, b.mn.y, b.mn.z, 0.0f);
    bhi[t] = make_float4(b.mx.x, b.mx.y, b.mx.z, 0.0f);
    cen[t] = make_float4(c.x, c.y, c.z, 0.0f);
}

// Roots: one per mesh. Large roots start level 0; small roots go to the
// small list. Positions of large meshes get their root's large-node index.
__global__ void k_roots(int meshes, const int* mesh_pos, int n, Buffers B) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= meshes) return;
    int s = mesh_pos[m], e = m + 1 < meshes ? mesh_pos[m + 1] : n;
    B.n_start[m] = s;
    B.n_end[m] = e;
    B.n_mesh[m] = m;
    B.n_level[m] = 0;
    B.n_pre[m] = 0;
    B.n_child[m] = -1;
    if (e - s > kSmall) {
        int j = atomicAdd(&B.ctl->next_act, 1);
        B.act[j] = m;
        atomicMax(&B.ctl->max_span, e - s);
    } else {
        B.small[atomicAdd(&B.ctl->small, 1)] = m;
    }
}

__global__ void k_init_positions(int n, Buffers B) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    B.idx[0][p] = p;
    B.order[p] = p;
    B.seg[0][p] = -1;
}

// Block j marks the positions of large root j.
__global__ void k_root_positions(Buffers B) {
    int j = blockIdx.x;
    int m = B.act[j];
    for (int p = B.n_start[m] + threadIdx.x; p < B.n_end[m]; p += blockDim.x) B.seg[0][p] = j;
}

__global__ void k_acc_init(int64_t S, int* acc_a, int* acc_c, int* acc_b) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int hi = f2o(kInf), lo = f2o(-kInf);
    if (i < S * kAccA) {
        int k = (int)(i % kAccA);
        acc_a[i] = (k < 3 || (k >= 6 && k < 9)) ? hi : lo;
    }
    if (i < S * kBinsAll) acc_c[i] = 0;
    if (i < S * kBinsAll * 6) acc_b[i] = (i % 6) < 3 ? hi : lo;
}

// Node box and centroid bounds of every large node of the level.
__global__ void __launch_bounds__(256) k_bounds(int n, const int* __restrict__ seg, const int* __restrict__ idx,
                                                const float4* __restrict__ blo, const float4* __restrict__ bhi,
                                                const float4* __restrict__ cen, int* acc_a) {
    const unsigned full = 0xffffffffu;
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    int lane = threadIdx.x & 31;
    int s = p < n ? seg[p] : -1;
    int key = s >= 0 ? s : -2 - lane;
    int v[kAccA];
    if (s >= 0) {
        int t = idx[p];
        float4 a = blo[t], b = bhi[t], c = cen[t];
        v[0] = f2o(a.x); v[1] = f2o(a.y); v[2] = f2o(a.z);
        v[3] = f2o(b.x); v[4] = f2o(b.y); v[5] = f2o(b.z);
        v[6] = f2o(c.x); v[7] = f2o(c.y); v[8] = f2o(c.z);
        v[9] = v[6]; v[10] = v[7]; v[11] = v[8];
    } else {
        for (int k = 0; k < kAccA; k++) v[k] = 0;
    }
    // a node's positions are contiguous, so its lanes form one run: reduce
    // each run into its first lane
    for (int o = 1; o < 32; o <<= 1) {
        int ko = __shfl_down_sync(full, key, o);
        bool take = lane + o < 32 && ko == key;
        for (int k = 0; k < kAccA; k++) {
            int x = __shfl_down_sync(full, v[k], o);
            bool is_min = k < 3 || (k >= 6 && k < 9);
            if (take) v[k] = is_min ? min(v[k], x) : max(v[k], x);
        }
    }
    int kp = __shfl_up_sync(full, key, 1);
    if (s >= 0 && (lane == 0 || kp != key)) {
        int* a = acc_a + (size_t)s * kAccA;
        for (int k = 0; k < kAccA; k++) {
            bool is_min = k < 3 || (k >= 6 && k < 9);
            if (is_min) atomicMin(a + k, v[k]);
            else atomicMax(a + k, v[k]);
        }
    }
}

// The three axes' bins of every large node (axes with a zero centroid extent
// are skipped, as in the host build).
__global__ void __launch_bounds__(256) k_bins(int n, const int* __restrict__ seg, const int* __restrict__ idx,
                                              const float4* __restrict__ blo, const float4* __restrict__ bhi,
                                              const float4* __restrict__ cen, const int* __restrict__ acc_a,
                                              int* acc_c, int* acc_b) {
    const unsigned full = 0xffffffffu;
    __shared__ int stage[8][32][6];
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int s = p < n ? seg[p] : -1;
    float c[3] = {0.0f, 0.0f, 0.0f};
    if (s >= 0) {
        int t = idx[p];
        float4 a = blo[t], b = bhi[t], cc = cen[t];
        stage[w][lane][0] = f2o(a.x); stage[w][lane][1] = f2o(a.y); stage[w][lane][2] = f2o(a.z);
        stage[w][lane][3] = f2o(b.x); stage[w][lane][4] = f2o(b.y); stage[w][lane][5] = f2o(b.z);
        c[0] = cc.x; c[1] = cc.y; c[2] = cc.z;
    }
    __syncwarp();
    for (int ax = 0; ax < 3; ax++) {
        int key = -1 - lane;
        int k = 0;
        if (s >= 0) {
            const int* a = acc_a + (size_t)s * kAccA;
            float c0 = o2f(a[6 + ax]), c1 = o2f(a[9 + ax]);
            float e = c1 - c0;
            if (e > 0.0f) {
                k = sah_bin(c[ax], c0, (float)kSahBins / e);
                key = s * kSahBins + k;
            }
        }
        unsigned peers = __match_any_sync(full, key);
        if (key >= 0 && lane == __ffs(peers) - 1) {
            int r[6];
            for (int j = 0; j < 6; j++) r[j] = stage[w][lane][j];
            for (unsigned m = peers & (peers - 1); m; m &= m - 1) {
                int q = __ffs(m) - 1;
                for (int j = 0; j < 3; j++) r[j] = min(r[j], stage[w][q][j]);
                for (int j = 3; j < 6; j++) r[j] = max(r[j], stage[w][q][j]);
            }
            size_t bi = (size_t)s * kBinsAll + ax * kSahBins + k;
            atomicAdd(acc_c + bi, __popc(peers));
            int* bb = acc_b + bi * 6;
            for (int j = 0; j < 3; j++) atomicMin(bb + j, r[j]);
            for (int j = 3; j < 6; j++) atomicMax(bb + j, r[j]);
        }
    }
}

// One thread per large node: the host's plane choice, then the children.
__global__ void k_split(int S, int level, int child_base, int* act_next, Buffers B) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= S) return;
    int node = B.act[a];
    SplitInfo si;
    si.start = B.n_start[node];
    si.end = B.n_end[node];
    int span = si.end - si.start;
    const int* acc = B.acc_a + (size_t)a * kAccA;
    V3 bmn = v3(o2f(acc[0]), o2f(acc[1]), o2f(acc[2]));
    V3 bmx = v3(o2f(acc[3]), o2f(acc[4]), o2f(acc[5]));
    V3 cmin = v3(o2f(acc[6]), o2f(acc[7]), o2f(acc[8]));
    V3 cmax = v3(o2f(acc[9]), o2f(acc[10]), o2f(acc[11]));
    V3 ext = cmax - cmin;
    float max_ext = fmaxf(ext.x, fmaxf(ext.y, ext.z));
    si.mode = 1;
    si.axis = 0;
    si.bin = -1;
    si.mid = si.start + span / 2;
    si.c0 = 0.0f;
    si.scale = 0.0f;
    if (max_ext > 0.0f) {
        int best_axis = -1, best_bin = -1;
        float best_cost = kInf;
        int cnt[kSahBins];
        Box bb[kSahBins];
        for (int ax = 0; ax < 3; ax++) {
            if (axis_of(ext, ax) <= 0.0f) continue;
            const int* c = B.acc_c + (size_t)a * kBinsAll + ax * kSahBins;
            const int* b = B.acc_b + ((size_t)a * kBinsAll + ax * kSahBins) * 6;
            for (int i = 0; i < kSahBins; i++) {
                cnt[i] = c[i];
                bb[i].mn = v3(o2f(b[6 * i]), o2f(b[6 * i + 1]), o2f(b[6 * i + 2]));
                bb[i].mx = v3(o2f(b[6 * i + 3]), o2f(b[6 * i + 4]), o2f(b[6 * i + 5]));
            }
            sah_eval_axis(ax, cnt, bb, best_cost, best_axis, best_bin);
        }
        if (best_axis >= 0) {
            const int* c = B.acc_c + (size_t)a * kBinsAll + best_axis * kSahBins;
            int nl = 0;
            for (int i = 0; i <= best_bin; i++) nl += c[i];
            si.axis = best_axis;
            if (nl > 0 && nl < span) {
                si.mode = 0;
                si.bin = best_bin;
                si.mid = si.start + nl;
                si.c0 = axis_of(cmin, best_axis);
                si.scale = (float)kSahBins / axis_of(ext, best_axis);
            }
        }
    }
    B.split[a] = si;
    B.n_axis[node] = si.axis;
    B.n_lo[node] = make_float4(bmn.x, bmn.y, bmn.z, 0.0f);
    B.n_hi[node] = make_float4(bmx.x, bmx.y, bmx.z, 0.0f);
    int c0 = child_base + 2 * a;
    B.n_child[node] = c0;
    int mesh = B.n_mesh[node];
    for (int side = 0; side < 2; side++) {
        int c = c0 + side;
        int cs = side ? si.mid : si.start, ce = side ? si.end : si.mid;
        B.n_start[c] = cs;
        B.n_end[c] = ce;
        B.n_mesh[c] = mesh;
        B.n_level[c] = level + 1;
        B.n_child[c] = -1;
        if (ce - cs > kSmall) {
            int j = atomicAdd(&B.ctl->next_act, 1);
            act_next[j] = c;
            B.seg_next[2 * a + side] = j;
            atomicMax(&B.ctl->max_span, ce - cs);
        } else {
            B.seg_next[2 * a + side] = -1;
            B.small[atomicAdd(&B.ctl->small, 1)] = c;
        }
    }
}

__global__ void k_flags(int n, const int* __restrict__ seg, const int* __restrict__ idx,
                        const float4* __restrict__ cen, const SplitInfo* __restrict__ split, int* flag) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int s = seg[p];
    int f = 0;
    if (s >= 0) {
        SplitInfo si = split[s];
        if (si.mode == 0) {
            float4 c = cen[idx[p]];
            float x = si.axis == 0 ? c.x : (si.axis == 1 ? c.y : c.z);
            f = sah_bin(x, si.c0, si.scale) <= si.bin;
        }
    }
    flag[p] = f;
}

__global__ void k_ptr_init(int n, const int* __restrict__ seg, const SplitInfo* __restrict__ split,
                           const int* __restrict__ flag, const int* __restrict__ rank, int* ptr) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int s = seg[p];
    if (s < 0) return;
    int st = split[s].start;
    ptr[p] = flag[p] ? st + (rank[p] - rank[st]) : p;
}

__global__ void k_ptr_jump(int n, const int* __restrict__ seg, const int* __restrict__ in, int* out) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || seg[p] < 0) return;
    out[p] = in[in[p]];
}

__device__ __forceinline__ void put(const Buffers& B, int* seg_out, int* idx_out, int s, int side, int dest, int v) {
    int cs = B.seg_next[2 * s + side];
    seg_out[dest] = cs;
    if (cs >= 0) idx_out[dest] = v;
    else B.order[dest] = v;
}

__global__ void k_scatter(int n, Buffers B, const int* __restrict__ seg, const int* __restrict__ idx,
                          const int* __restrict__ ptr, int* seg_out, int* idx_out) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int s = seg[p];
    if (s < 0) {
        seg_out[p] = -1;
        return;
    }
    SplitInfo si = B.split[s];
    if (si.mode == 1) {
        put(B, seg_out, idx_out, s, p >= si.mid, p, idx[p]);
        return;
    }
    if (B.flag[p]) put(B, seg_out, idx_out, s, 0, si.start + (B.rank[p] - B.rank[si.start]), idx[p]);
    if (p >= si.mid) put(B, seg_out, idx_out, s, 1, p, idx[ptr[p]]);
}

// One thread per small root: the host recursion on [start, end) of the leaf
// order, in place, nodes in pre-order into tmp[2 * start ...].
__global__ void k_small(int count, Buffers B) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    int node = B.small[k];
    int start = B.n_start[node], end = B.n_end[node];
    int mesh = B.n_mesh[node];
    int base = B.mesh_pos[mesh];
    NodeF* out = B.tmp + 2 * (size_t)start;
    const float4* blo = B.blo;
    const float4* bhi = B.bhi;
    auto box_of = [blo, bhi](int t) {
        float4 a = blo[t], b = bhi[t];
        return Box{v3(a.x, a.y, a.z), v3(b.x, b.y, b.z)};
    };
    struct Item {
        int s, e, depth, parent;   // parent: the node whose right child this is, or -1
    };
    Item stack[2 * kSmall + 2];
    int sp = 0;
    stack[sp++] = Item{start, end, 0, -1};
    int cnt = 0, max_depth = 0;
    while (sp > 0) {
        Item it = stack[--sp];
        int me = cnt++;
        if (it.parent >= 0) {
            int b;
            memcpy(&b, &out[it.parent].hi[3], 4);
            b |= me;
            memcpy(&out[it.parent].hi[3], &b, 4);
        }
        Box box = box_of(B.order[it.s]);
        for (int i = it.s + 1; i < it.e; i++) box = surround(box, box_of(B.order[i]));
        NodeF& nd = out[me];
        nd.lo[0] = box.mn.x; nd.lo[1] = box.mn.y; nd.lo[2] = box.mn.z;
        nd.hi[0] = box.mx.x; nd.hi[1] = box.mx.y; nd.hi[2] = box.mx.z;
        int span = it.e - it.s;
        if (span <= kSahMaxLeaf) {
            int a = ~(it.s - base), b = span | (LEAF_TRIS << 16);
            memcpy(&nd.lo[3], &a, 4);
            memcpy(&nd.hi[3], &b, 4);
            max_depth = max(max_depth, it.depth);
            continue;
        }
        int axis, mid;
        if (!sah_split(it.s, it.e, B.order, box_of, axis, mid)) {
            axis = 0;
            mid = it.s + span / 2;
        }
        int a = me + 1, b = axis << 30;   // the right child's index is or-ed in when it is emitted
        memcpy(&nd.lo[3], &a, 4);
        memcpy(&nd.hi[3], &b, 4);
        stack[sp++] = Item{mid, it.e, it.depth + 1, me};
        stack[sp++] = Item{it.s, mid, it.depth + 1, -1};
    }
    B.n_size[node] = cnt;
    B.n_lo[node] = make_float4(out[0].lo[0], out[0].lo[1], out[0].lo[2], 0.0f);
    B.n_hi[node] = make_float4(out[0].hi[0], out[0].hi[1], out[0].hi[2], 0.0f);
    atomicMax(&B.mesh_depth[mesh], B.n_level[node] + max_depth);
}

__global__ void k_sizes(int count, const int* act, Buffers B) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    int node = act[j], c = B.n_child[node];
    B.n_size[node] = 1 + B.n_size[c] + B.n_size[c + 1];
}

__global__ void k_preorder(int count, const int* act, Buffers B) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    int node = act[j], c = B.n_child[node];
    int pre = B.n_pre[node];
    B.n_pre[c] = pre + 1;
    B.n_pre[c + 1] = pre + 1 + B.n_size[c];
}

__global__ void k_emit_large(int count, Buffers B) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    int node = B.act[j], c = B.n_child[node];
    NodeF nd;
    float4 lo = B.n_lo[node], hi = B.n_hi[node];
    nd.lo[0] = lo.x; nd.lo[1] = lo.y; nd.lo[2] = lo.z;
    nd.hi[0] = hi.x; nd.hi[1] = hi.y; nd.hi[2] = hi.z;
    int a = B.n_pre[c], b = B.n_pre[c + 1] | (B.n_axis[node] << 30);
    memcpy(&nd.lo[3], &a, 4);
    memcpy(&nd.hi[3], &b, 4);
    B.out[B.mesh_base[B.n_mesh[node]] + B.n_pre[node]] = nd;
}

__global__ void k_emit_small(int count, Buffers B) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    int node = B.small[k];
    int pre = B.n_pre[node], size = B.n_size[node];
    const NodeF* src = B.tmp + 2 * (size_t)B.n_start[node];
    NodeF* dst = B.out + B.mesh_base[B.n_mesh[node]] + pre;
    for (int i = 0; i < size; i++) {
        NodeF nd = src[i];
        int a, b;
        memcpy(&a, &nd.lo[3], 4);
        if (a >= 0) {
            memcpy(&b, &nd.hi[3], 4);
            a += pre;
            b = (b & ~0x3FFFFFFF) | ((b & 0x3FFFFFFF) + pre);
            memcpy(&nd.lo[3], &a, 4);
            memcpy(&nd.hi[3], &b, 4);
        }
        dst[i] = nd;
    }
}

// RT3D_BVH_TIMING=1 prints the build's phases (host wall time) to stderr.
struct PhaseLog {
    bool on = getenv("RT3D_BVH_TIMING") != nullptr;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    void mark(const char* what) {
        if (!on) return;
        auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "bvh_build %-10s %8.3f ms\n", what, std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

inline unsigned blocks(int64_t n, int t) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

// The build's scratch comes from a private stream-ordered pool per device.
// The pool keeps up to kPoolKeep bytes reserved after a build (about 380 B
// per triangle are needed), so a later build in the process skips the
// allocation and frees never synchronise the device.
constexpr uint64_t kPoolKeep = 1ull << 30;

cudaError_t build_pool(int dev, cudaMemPool_t* out) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p;
    cudaError_t e = cudaMemPoolCreate(&p, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = kPoolKeep;
    e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
        cudaMemPoolDestroy(p);
        return e;
    }
    pools[dev] = p;
    *out = p;
    return cudaSuccess;
}

struct Pool {   // device allocations of one build, stream-ordered, freed together
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    std::vector<void*> ptrs;
    template <class T>
    cudaError_t get(T** p, size_t count) {
        void* v = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&v, std::max<size_t>(count, 1) * sizeof(T), pool, stream);
        if (e == cudaSuccess) ptrs.push_back(v);
        *p = (T*)v;
        return e;
    }
    void release() {
        for (void* v : ptrs) cudaFreeAsync(v, stream);
        ptrs.clear();
    }
    ~Pool() { release(); }
};

}  // namespace

// MeshBvhBuilder on the current device (see world.h).
int device_build_meshes(const float* tri_verts, const int64_t* first, const int64_t* count, int meshes,
                        MeshBvh* out, std::string& err) {
#define BV_TRY(x)                                                          \
    do {                                                                   \
        cudaError_t e_ = (x);                                              \
        if (e_ != cudaSuccess) {                                           \
            err = std::string("device BVH build: ") + cudaGetErrorString(e_); \
            return RT_ERR_CUDA;                                            \
        }                                                                  \
    } while (0)
    int64_t total = 0;
    for (int m = 0; m < meshes; m++) {
        if (count[m] <= kSahMaxLeaf) {
            err = "device BVH build: a mesh of at most 4 triangles is a flat list";
            return RT_ERR_INVALID_ARG;
        }
        total += count[m];
    }
    if (meshes <= 0 || total >= (int64_t)1 << 28) {
        err = "device BVH build: batch size out of range";
        return RT_ERR_INVALID_ARG;
    }
    const int n = (int)total;
    PhaseLog log;
    int dev = 0;
    BV_TRY(cudaGetDevice(&dev));
    cudaStream_t st = nullptr;
    BV_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {   // declared before the pool: destroyed after its frees are queued
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard{st};
    Pool pool;
    pool.stream = st;
    BV_TRY(build_pool(dev, &pool.pool));
    Buffers B;
    B.n = n;
    B.meshes = meshes;
    const int64_t node_cap = 2 * (int64_t)n + meshes;
    const int64_t seg_cap = n / (kSmall + 1) + meshes + 1;
    float* d_verts = nullptr;
    BV_TRY(pool.get(&d_verts, (size_t)n * 9));
    BV_TRY(pool.get(&B.blo, n));
    BV_TRY(pool.get(&B.bhi, n));
    BV_TRY(pool.get(&B.cen, n));
    for (int k = 0; k < 2; k++) {
        BV_TRY(pool.get(&B.idx[k], n));
        BV_TRY(pool.get(&B.seg[k], n));
        BV_TRY(pool.get(&B.ptr[k], n));
    }
    BV_TRY(pool.get(&B.flag, n));
    BV_TRY(pool.get(&B.rank, n));
    BV_TRY(pool.get(&B.order, n));
    BV_TRY(pool.get(&B.acc_a, (size_t)seg_cap * kAccA));
    BV_TRY(pool.get(&B.acc_c, (size_t)seg_cap * kBinsAll));
    BV_TRY(pool.get(&B.acc_b, (size_t)seg_cap * kBinsAll * 6));
    BV_TRY(pool.get(&B.split, seg_cap));
    BV_TRY(pool.get(&B.seg_next, 2 * seg_cap));
    BV_TRY(pool.get(&B.n_start, node_cap));
    BV_TRY(pool.get(&B.n_end, node_cap));
    BV_TRY(pool.get(&B.n_mesh, node_cap));
    BV_TRY(pool.get(&B.n_level, node_cap));
    BV_TRY(pool.get(&B.n_child, node_cap));
    BV_TRY(pool.get(&B.n_axis, node_cap));
    BV_TRY(pool.get(&B.n_lo, node_cap));
    BV_TRY(pool.get(&B.n_hi, node_cap));
    BV_TRY(pool.get(&B.n_size, node_cap));
    BV_TRY(pool.get(&B.n_pre, node_cap));
    BV_TRY(pool.get(&B.act, n + meshes));
    BV_TRY(pool.get(&B.small, n + meshes));
    BV_TRY(pool.get(&B.tmp, 2 * (size_t)n));
    BV_TRY(pool.get(&B.mesh_pos, meshes));
    BV_TRY(pool.get(&B.mesh_depth, meshes));
    BV_TRY(pool.get(&B.mesh_base, meshes));
    BV_TRY(pool.get(&B.ctl, 1));
    BV_TRY(cub::DeviceScan::ExclusiveSum(nullptr, B.scan_bytes, B.flag, B.rank, n));
    BV_TRY(pool.get(&B.scan_tmp, B.scan_bytes));
    log.mark("alloc");

    std::vector<int> mesh_pos(meshes);
    {
        int64_t pos = 0;
        for (int m = 0; m < meshes; m++) {
            mesh_pos[m] = (int)pos;
            BV_TRY(cudaMemcpyAsync(d_verts + pos * 9, tri_verts + first[m] * 9, (size_t)count[m] * 9 * sizeof(float),
                                   cudaMemcpyHostToDevice, st));
            pos += count[m];
        }
    }
    BV_TRY(cudaMemcpyAsync(B.mesh_pos, mesh_pos.data(), meshes * sizeof(int), cudaMemcpyHostToDevice, st));
    BV_TRY(cudaMemsetAsync(B.mesh_depth, 0, meshes * sizeof(int), st));
    BV_TRY(cudaMemsetAsync(B.ctl, 0, sizeof(BuildCtl), st));
    k_boxes<<<blocks(n, 256), 256, 0, st>>>(n, d_verts, B.blo, B.bhi, B.cen, B.ctl);
    k_roots<<<blocks(meshes, 128), 128, 0, st>>>(meshes, B.mesh_pos, n, B);
    BuildCtl ctl{};
    BV_TRY(cudaMemcpyAsync(&ctl, B.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaStreamSynchronize(st));
    if (ctl.bad_vertex) {
        err = "device BVH build: a vertex coordinate is not finite";
        return RT_ERR_UNSUPPORTED;
    }
    log.mark("upload");
    k_init_positions<<<blocks(n, 256), 256, 0, st>>>(n, B);
    if (ctl.next_act > 0) k_root_positions<<<ctl.next_act, 256, 0, st>>>(B);
    BV_TRY(cudaGetLastError());

    // --- large nodes, level by level
    std::vector<int> lvl_off{0};   // large nodes of level L: act[lvl_off[L] .. lvl_off[L + 1])
    int S = ctl.next_act, max_span = ctl.max_span;
    int small_count = ctl.small;
    int nodes = meshes;            // BFS ids handed out so far
    int cur = 0;
    int level = 0;
    while (S > 0) {
        lvl_off.push_back(lvl_off.back() + S);
        int* act_cur = B.act + lvl_off[level];
        int* act_next = B.act + lvl_off[level + 1];
        Buffers L = B;
        L.act = act_cur;
        BuildCtl zero{0, small_count, 0, 0};
        BV_TRY(cudaMemcpyAsync(B.ctl, &zero, sizeof(zero), cudaMemcpyHostToDevice, st));
        k_acc_init<<<blocks((int64_t)S * kBinsAll * 6, 256), 256, 0, st>>>(S, B.acc_a, B.acc_c, B.acc_b);
        k_bounds<<<blocks(n, 256), 256, 0, st>>>(n, B.seg[cur], B.idx[cur], B.blo, B.bhi, B.cen, B.acc_a);
        k_bins<<<blocks(n, 256), 256, 0, st>>>(n, B.seg[cur], B.idx[cur], B.blo, B.bhi, B.cen, B.acc_a, B.acc_c,
                                               B.acc_b);
        k_split<<<blocks(S, 128), 128, 0, st>>>(S, level, nodes, act_next, L);
        k_flags<<<blocks(n, 256), 256, 0, st>>>(n, B.seg[cur], B.idx[cur], B.cen, B.split, B.flag);
        BV_TRY(cub::DeviceScan::ExclusiveSum(B.scan_tmp, B.scan_bytes, B.flag, B.rank, n, st));
        k_ptr_init<<<blocks(n, 256), 256, 0, st>>>(n, B.seg[cur], B.split, B.flag, B.rank, B.ptr[0]);
        int rounds = 1;
        while ((1 << (rounds - 1)) < max_span) rounds++;   // 2^(rounds-1) >= the longest chain
        int pc = 0;
        for (int r = 0; r < rounds; r++) {
            k_ptr_jump<<<blocks(n, 256), 256, 0, st>>>(n, B.seg[cur], B.ptr[pc], B.ptr[pc ^ 1]);
            pc ^= 1;
        }
        k_scatter<<<blocks(n, 256), 256, 0, st>>>(n, B, B.seg[cur], B.idx[cur], B.ptr[pc], B.seg[cur ^ 1],
                                                  B.idx[cur ^ 1]);
        BV_TRY(cudaGetLastError());
        BV_TRY(cudaMemcpyAsync(&ctl, B.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st));
        BV_TRY(cudaStreamSynchronize(st));
        nodes += 2 * S;
        S = ctl.next_act;
        max_span = ctl.max_span;
        small_count = ctl.small;
        cur ^= 1;
        level++;
        if ((int64_t)nodes + 2 * (int64_t)S > node_cap) {
            err = "device BVH build: node capacity exceeded";
            return RT_ERR_BOUNDS;
        }
    }
    const int levels = level;
    const int n_large = lvl_off.back();
    log.mark("levels");

    // --- small subtrees, subtree sizes, pre-order indices
    k_small<<<blocks(small_count, 128), 128, 0, st>>>(small_count, B);
    for (int l = levels - 1; l >= 0; l--) {
        int c = lvl_off[l + 1] - lvl_off[l];
        k_sizes<<<blocks(c, 256), 256, 0, st>>>(c, B.act + lvl_off[l], B);
    }
    for (int l = 0; l < levels; l++) {
        int c = lvl_off[l + 1] - lvl_off[l];
        k_preorder<<<blocks(c, 256), 256, 0, st>>>(c, B.act + lvl_off[l], B);
    }
    BV_TRY(cudaGetLastError());
    std::vector<int> root_size(meshes), mesh_depth(meshes);
    std::vector<float4> root_lo(meshes), root_hi(meshes);
    BV_TRY(cudaMemcpyAsync(root_size.data(), B.n_size, meshes * sizeof(int), cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaMemcpyAsync(root_lo.data(), B.n_lo, meshes * sizeof(float4), cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaMemcpyAsync(root_hi.data(), B.n_hi, meshes * sizeof(float4), cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaMemcpyAsync(mesh_depth.data(), B.mesh_depth, meshes * sizeof(int), cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaStreamSynchronize(st));
    log.mark("small");
    std::vector<int> mesh_base(meshes);
    int64_t total_nodes = 0;
    for (int m = 0; m < meshes; m++) {
        mesh_base[m] = (int)total_nodes;
        total_nodes += root_size[m];
    }
    BV_TRY(pool.get(&B.out, (size_t)total_nodes));
    BV_TRY(cudaMemcpyAsync(B.mesh_base, mesh_base.data(), meshes * sizeof(int), cudaMemcpyHostToDevice, st));
    k_emit_large<<<blocks(n_large, 256), 256, 0, st>>>(n_large, B);
    k_emit_small<<<blocks(small_count, 128), 128, 0, st>>>(small_count, B);
    BV_TRY(cudaGetLastError());
    std::vector<NodeF> all((size_t)total_nodes);
    std::vector<int> order(n);
    BV_TRY(cudaMemcpyAsync(all.data(), B.out, (size_t)total_nodes * sizeof(NodeF), cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaMemcpyAsync(order.data(), B.order, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
    BV_TRY(cudaStreamSynchronize(st));
    log.mark("download");
    for (int m = 0; m < meshes; m++) {
        MeshBvh& mb = out[m];
        mb.nodes.assign(all.begin() + mesh_base[m], all.begin() + mesh_base[m] + root_size[m]);
        mb.order.resize((size_t)count[m]);
        for (int64_t i = 0; i < count[m]; i++) mb.order[i] = order[mesh_pos[m] + i] - mesh_pos[m];
        mb.box_mn = v3(root_lo[m].x, root_lo[m].y, root_lo[m].z);
        mb.box_mx = v3(root_hi[m].x, root_hi[m].y, root_hi[m].z);
        mb.max_depth = mesh_depth[m];
    }
    log.mark("unpack");
    pool.release();
    BV_TRY(cudaStreamSynchronize(st));
    log.mark("free");
    return RT_OK;
#undef BV_TRY
}

}  // namespace rt
