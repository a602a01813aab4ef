// Binned-SAH split of BvhNode's constructor (Acceleration/BvhNode.cs:218-363),
// shared by the host build (world.cpp) and the device build (bvh_build.cu) so
// that both evaluate the same float expressions in the same order: 16 bins
// per axis over the centroid bounds, traversal cost 0.5, the first strictly
// cheaper (axis, bin) wins, then an in-place partition in which left items
// keep their order and each left item swaps with the first right one.
#pragma once

#include "vec.cuh"

namespace rt {

constexpr int kSahBins = 16;     // BvhNode.cs:60
constexpr int kSahMaxLeaf = 4;   // BvhNode.cs:53

struct Box {
    V3 mn, mx;
};
RT_HD Box surround(const Box& a, const Box& b) { return {vmin(a.mn, b.mn), vmax(a.mx, b.mx)}; }
RT_HD Box empty_box() { return {v3(kInf), v3(-kInf)}; }   // AABB.Empty (Core/AABB.cs:77)
RT_HD float surface_area(const Box& b) {                   // AABB.SurfaceArea (Core/AABB.cs:70-75)
    V3 d = b.mx - b.mn;
    if (d.x < 0.0f || d.y < 0.0f || d.z < 0.0f) return 0.0f;
    return 2.0f * (d.x * d.y + d.x * d.z + d.y * d.z);
}
RT_HD Box tri_box(V3 a, V3 b, V3 c) {   // Triangle.BoundingBox (Geometry/Triangle.cs:144-149)
    return {vmin(vmin(a, b), c) - v3(kEps), vmax(vmax(a, b), c) + v3(kEps)};
}
RT_HD V3 box_centroid(const Box& b) { return (b.mn + b.mx) * 0.5f; }

// Bin of a centroid coordinate c on an axis whose centroid bounds start at c0,
// with scale = kSahBins / extent.
RT_HD int sah_bin(float c, float c0, float scale) {
    int k = (int)((c - c0) * scale);
    return k < 0 ? 0 : (k >= kSahBins ? kSahBins - 1 : k);
}

// Evaluates the 15 split planes of one axis from its bins and keeps the
// cheapest so far (strictly cheaper replaces, so ties keep the earlier axis
// and bin).
RT_HD void sah_eval_axis(int ax, const int* cnt, const Box* bb, float& best_cost, int& best_axis, int& best_bin) {
    int pre_c[kSahBins], suf_c[kSahBins];
    Box pre_b[kSahBins], suf_b[kSahBins];
    int cum = 0;
    Box cb = empty_box();
    for (int i = 0; i < kSahBins; i++) {
        cum += cnt[i];
        cb = surround(cb, bb[i]);
        pre_c[i] = cum;
        pre_b[i] = cb;
    }
    cum = 0;
    cb = empty_box();
    for (int i = kSahBins - 1; i >= 0; i--) {
        cum += cnt[i];
        cb = surround(cb, bb[i]);
        suf_c[i] = cum;
        suf_b[i] = cb;
    }
    float parent = surface_area(pre_b[kSahBins - 1]);
    if (parent <= 0.0f) return;
    for (int i = 0; i < kSahBins - 1; i++) {
        int nl = pre_c[i], nr = suf_c[i + 1];
        if (nl == 0 || nr == 0) continue;
        float cost = 0.5f + (nl * surface_area(pre_b[i]) + nr * surface_area(suf_b[i + 1])) / parent;
        if (cost < best_cost) {
            best_cost = cost;
            best_axis = ax;
            best_bin = i;
        }
    }
}

// TryFindSAHSplit on the items idx[start, end): returns false (no split: the
// caller splits at the median, axis 0) when the centroids coincide or no
// plane separates them; otherwise partitions idx in place and sets the axis
// and the first right position `mid` (the median when a side is empty).
// box_of(item) returns the item's box.
template <class BoxOf>
RT_HD bool sah_split(int start, int end, int* idx, const BoxOf& box_of, int& best_axis, int& mid) {
    int span = end - start;
    V3 cmin = v3(kInf), cmax = v3(-kInf);
    for (int i = start; i < end; i++) {
        V3 c = box_centroid(box_of(idx[i]));
        cmin = vmin(cmin, c);
        cmax = vmax(cmax, c);
    }
    V3 ext = cmax - cmin;
    float max_ext = fmaxf(ext.x, fmaxf(ext.y, ext.z));
    best_axis = -1;
    mid = start;
    if (max_ext <= 0.0f) return false;
    int best_bin = -1;
    float best_cost = kInf;
    int cnt[kSahBins];
    Box bb[kSahBins];
    for (int ax = 0; ax < 3; ax++) {
        float e = axis_of(ext, ax);
        if (e <= 0.0f) continue;
        float c0 = axis_of(cmin, ax);
        float scale = (float)kSahBins / e;
        for (int i = 0; i < kSahBins; i++) {
            cnt[i] = 0;
            bb[i] = empty_box();
        }
        for (int i = start; i < end; i++) {
            Box b = box_of(idx[i]);
            int k = sah_bin(axis_of(box_centroid(b), ax), c0, scale);
            cnt[k]++;
            bb[k] = surround(bb[k], b);
        }
        sah_eval_axis(ax, cnt, bb, best_cost, best_axis, best_bin);
    }
    if (best_axis < 0) return false;
    float c0 = axis_of(cmin, best_axis);
    float scale = (float)kSahBins / axis_of(ext, best_axis);
    int wp = start;
    for (int i = start; i < end; i++) {
        if (sah_bin(axis_of(box_centroid(box_of(idx[i])), best_axis), c0, scale) <= best_bin) {
            int t = idx[i];
            idx[i] = idx[wp];
            idx[wp] = t;
            wp++;
        }
    }
    mid = wp;
    if (mid == start || mid == end) mid = start + span / 2;
    return true;
}

}  // namespace rt
