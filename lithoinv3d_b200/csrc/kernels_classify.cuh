// Point classification and the constraint penalty.
//
// LithologyModel::classifyPoint (modules/litho-model/src/litho/
// lithology_model.cpp:288-363): below the model's bottom depth -> -1; else
// the label grid, when one is set and the point's voxel holds a group id
// >= 0; else a ray along +x from the point (offset by 1.234567e-6 in y and
// 2.345678e-6 in z) is intersected with every triangle of each group mesh
// in group order (Moller-Trumbore), and the first group crossed an odd
// number of times is the answer (-1 if none).  The intersection test is
// restated with every operation rounded explicitly in the reference's
// order, so the GPU answer equals the reference's bit for bit, including
// points that graze an edge.
//
// ConstraintHandler (modules/litho-inversion/src/inversion/
// constraint_handler.cpp:16-66): violation of a constraint = |z_bottom -
// z_top| when its interval midpoint is not classified as its group, penalty
// = weight x sum of squared violations in constraint order.
#pragma once
#include "kernels_fp64.cuh"

namespace litho_b200 {

struct LabelGridDev {
    int nx = 0, ny = 0, nz = 0;
    double x0 = 0, y0 = 0, z0 = 0, dx = 1, dy = 1, dz = 1;
    const int32_t* labels = nullptr;  // [nz][ny][nx], nullptr: no grid
};

// One ray-triangle test of classifyPoint (lithology_model.cpp:328-353) with
// rayDir = (1, 0, 0): true when the ray from o crosses triangle (p0, p1, p2)
// at t > 1e-12.
__device__ __forceinline__ bool ray_x_hits(double ox, double oy, double oz, const double* p0, const double* p1,
                                           const double* p2) {
    const double e1x = __dsub_rn(p1[0], p0[0]), e1y = __dsub_rn(p1[1], p0[1]), e1z = __dsub_rn(p1[2], p0[2]);
    const double e2x = __dsub_rn(p2[0], p0[0]), e2y = __dsub_rn(p2[1], p0[1]), e2z = __dsub_rn(p2[2], p0[2]);
    // h = rayDir x e2, component by component as the cross product forms it
    const double hx = __dsub_rn(__dmul_rn(0.0, e2z), __dmul_rn(0.0, e2y));
    const double hy = __dsub_rn(__dmul_rn(0.0, e2x), __dmul_rn(1.0, e2z));
    const double hz = __dsub_rn(__dmul_rn(1.0, e2y), __dmul_rn(0.0, e2x));
    const double a = __dadd_rn(__dadd_rn(__dmul_rn(e1x, hx), __dmul_rn(e1y, hy)), __dmul_rn(e1z, hz));
    if (fabs(a) < 1e-30) return false;
    const double f = __ddiv_rn(1.0, a);
    const double sx = __dsub_rn(ox, p0[0]), sy = __dsub_rn(oy, p0[1]), sz = __dsub_rn(oz, p0[2]);
    const double u = __dmul_rn(f, __dadd_rn(__dadd_rn(__dmul_rn(sx, hx), __dmul_rn(sy, hy)), __dmul_rn(sz, hz)));
    if (u < 0.0 || u > 1.0) return false;
    // q = s x e1
    const double qx = __dsub_rn(__dmul_rn(sy, e1z), __dmul_rn(sz, e1y));
    const double qy = __dsub_rn(__dmul_rn(sz, e1x), __dmul_rn(sx, e1z));
    const double qz = __dsub_rn(__dmul_rn(sx, e1y), __dmul_rn(sy, e1x));
    const double v = __dmul_rn(f, __dadd_rn(__dadd_rn(__dmul_rn(1.0, qx), __dmul_rn(0.0, qy)), __dmul_rn(0.0, qz)));
    if (v < 0.0 || __dadd_rn(u, v) > 1.0) return false;
    const double t = __dmul_rn(f, __dadd_rn(__dadd_rn(__dmul_rn(e2x, qx), __dmul_rn(e2y, qy)), __dmul_rn(e2z, qz)));
    return t > 1e-12;
}

constexpr int kClassifyThreads = 256;

// One CTA per point (any block size that is a multiple of 32): out[i] =
// classifyPoint(pts[i]) over the current positions.  The parity of each
// group's crossings is the parity of the number of threads that saw an odd
// count (__syncthreads_count), so the answer does not depend on how the
// triangles are split among threads.
__global__ void k_classify_points(int n, const double* __restrict__ pts, int G, const int32_t* __restrict__ grp_off,
                                  const int32_t* __restrict__ tri, const double* __restrict__ pos,
                                  double bottom_depth, LabelGridDev lg, int32_t* __restrict__ out) {
    const int i = blockIdx.x;
    if (i >= n) return;  // block-uniform
    const double px = pts[3 * i], py = pts[3 * i + 1], pz = pts[3 * i + 2];
    if (G <= 0 || pz < bottom_depth) {
        if (threadIdx.x == 0) out[i] = -1;
        return;
    }
    if (lg.labels) {
        const int ix = static_cast<int>(__ddiv_rn(__dsub_rn(px, lg.x0), lg.dx));
        const int iy = static_cast<int>(__ddiv_rn(__dsub_rn(py, lg.y0), lg.dy));
        const int iz = static_cast<int>(__ddiv_rn(__dsub_rn(pz, lg.z0), lg.dz));
        if (ix >= 0 && ix < lg.nx && iy >= 0 && iy < lg.ny && iz >= 0 && iz < lg.nz) {
            const int gid = lg.labels[(iz * lg.ny + iy) * lg.nx + ix];
            if (gid >= 0) {
                if (threadIdx.x == 0) out[i] = gid;
                return;
            }
        }
    }
    const double ox = px, oy = __dadd_rn(py, 1.234567e-6), oz = __dadd_rn(pz, 2.345678e-6);
    int result = -1;
    for (int g = 0; g < G; ++g) {
        int hits = 0;
        for (int t = grp_off[g] + (int)threadIdx.x; t < grp_off[g + 1]; t += blockDim.x) {
            const int32_t* tv = tri + 3 * (size_t)t;
            hits += ray_x_hits(ox, oy, oz, pos + 3 * (size_t)tv[0], pos + 3 * (size_t)tv[1], pos + 3 * (size_t)tv[2]);
        }
        if (__syncthreads_count(hits & 1) & 1) {
            result = g;
            break;  // block-uniform: every thread saw the same count
        }
    }
    if (threadIdx.x == 0) out[i] = result;
}

// The same classification spread over many CTAs per point, for up to 64
// groups: the answer only needs each group's crossing parity, and parities
// combine by XOR, which is exact and order-free.
//   k_classify_prep   per point: the bottom-depth and label-grid answers;
//                     undecided points get kClassPending and a zero mask;
//   k_classify_cross  (point, slice of the triangle list): each thread XORs
//                     bit face_group[t] into its mask for every crossed
//                     triangle t; warps combine and atomicXor into the
//                     point's mask;
//   k_classify_finish per undecided point: the lowest set bit (the first
//                     group in group order crossed an odd number of
//                     times), -1 for an empty mask.
constexpr int kClassPending = -2147483647 - 1;
constexpr int kCrossThreads = 256;

__global__ void k_classify_prep(int n, const double* __restrict__ pts, int G, double bottom_depth, LabelGridDev lg,
                                int32_t* __restrict__ out, unsigned long long* __restrict__ mask) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double px = pts[3 * i], py = pts[3 * i + 1], pz = pts[3 * i + 2];
    mask[i] = 0ull;
    if (G <= 0 || pz < bottom_depth) {
        out[i] = -1;
        return;
    }
    if (lg.labels) {
        const int ix = static_cast<int>(__ddiv_rn(__dsub_rn(px, lg.x0), lg.dx));
        const int iy = static_cast<int>(__ddiv_rn(__dsub_rn(py, lg.y0), lg.dy));
        const int iz = static_cast<int>(__ddiv_rn(__dsub_rn(pz, lg.z0), lg.dz));
        if (ix >= 0 && ix < lg.nx && iy >= 0 && iy < lg.ny && iz >= 0 && iz < lg.nz) {
            const int gid = lg.labels[(iz * lg.ny + iy) * lg.nx + ix];
            if (gid >= 0) {
                out[i] = gid;
                return;
            }
        }
    }
    out[i] = kClassPending;
}

__global__ void __launch_bounds__(kCrossThreads) k_classify_cross(int n, const double* __restrict__ pts, int T,
                                                                  int slice, const int16_t* __restrict__ face_group,
                                                                  const int32_t* __restrict__ tri,
                                                                  const double* __restrict__ pos,
                                                                  const int32_t* __restrict__ out,
                                                                  unsigned long long* __restrict__ mask) {
    const int i = blockIdx.x;
    if (i >= n || out[i] != kClassPending) return;  // block-uniform
    const double ox = pts[3 * i], oy = __dadd_rn(pts[3 * i + 1], 1.234567e-6),
                 oz = __dadd_rn(pts[3 * i + 2], 2.345678e-6);
    const int t0 = blockIdx.y * slice, t1 = min(T, t0 + slice);
    unsigned long long m = 0ull;
    for (int t = t0 + (int)threadIdx.x; t < t1; t += blockDim.x) {
        const int32_t* tv = tri + 3 * (size_t)t;
        if (ray_x_hits(ox, oy, oz, pos + 3 * (size_t)tv[0], pos + 3 * (size_t)tv[1], pos + 3 * (size_t)tv[2]))
            m ^= 1ull << face_group[t];
    }
    for (int off = 16; off > 0; off >>= 1) m ^= __shfl_xor_sync(0xffffffffu, m, off);
    if ((threadIdx.x & 31) == 0 && m) atomicXor(mask + i, m);
}

__global__ void k_classify_finish(int n, const unsigned long long* __restrict__ mask, int32_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || out[i] != kClassPending) return;
    const unsigned long long m = mask[i];
    out[i] = m ? __ffsll((long long)m) - 1 : -1;
}

// ConstraintHandler::evaluate (constraint_handler.cpp:31-42) from the
// classified interval midpoints: out = weight x sum_k v_k^2 in constraint
// order, v_k = 0 when cls[k] == group[k], else |z_bottom - z_top|.  One
// block of kPenaltyThreads: the squares are formed in parallel into shared
// memory a chunk at a time and thread 0 adds them in order (the reference's
// summation order, so the result is bit-identical).
constexpr int kPenaltyThreads = 256;
__global__ void __launch_bounds__(kPenaltyThreads) k_constraint_penalty(int n, const int32_t* __restrict__ cls,
                                                                        const int32_t* __restrict__ group,
                                                                        const double* __restrict__ thick,
                                                                        double weight, double* __restrict__ out) {
    __shared__ double sq[kPenaltyThreads];
    double pen = 0.0;
    for (int k0 = 0; k0 < n; k0 += kPenaltyThreads) {
        const int k = k0 + (int)threadIdx.x;
        double v = 0.0;
        if (k < n && cls[k] != group[k]) v = thick[k];
        sq[threadIdx.x] = __dmul_rn(v, v);
        __syncthreads();
        if (threadIdx.x == 0) {
            const int m = min(kPenaltyThreads, n - k0);
            for (int i = 0; i < m; ++i) pen = __dadd_rn(pen, sq[i]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = __dmul_rn(weight, pen);
}

// Parameter j of the finite-difference sweep of ConstraintHandler::gradient
// (constraint_handler.cpp:44-66): mode 0 p[j] = p0[j] + h, mode 1
// p[j] = (p0[j] + h) - 2h (the reference steps from the + position), mode 2
// p[j] = p0[j].
__global__ void k_constraint_step(double* __restrict__ p, const double* __restrict__ p0, int j, double h, int mode) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double up = __dadd_rn(p0[j], h);
    p[j] = mode == 0 ? up : (mode == 1 ? __dsub_rn(up, __dmul_rn(2.0, h)) : p0[j]);
}

// grad[j] = weight x (fp[j] - fm[j]) / (2h).
__global__ void k_constraint_fd(int np, const double* __restrict__ fp, const double* __restrict__ fm, double h,
                                double weight, double* __restrict__ grad) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < np) grad[j] = __dmul_rn(weight, __ddiv_rn(__dsub_rn(fp[j], fm[j]), __dmul_rn(2.0, h)));
}

// InversionRunner::smoothGradient (modules/litho-inversion/src/inversion/
// runner.cpp:643-706): each DOF-mapped vertex axis of a mesh takes
// (1 - w) x its gradient + w x the mean gradient of its mesh neighbours
// (sorted neighbour order) that carry the same axis; every global DOF then
// takes the value of its last (mesh, local DOF) reference, DOFs without
// references keep their gradient.  Three passes: refs -> per-vertex-axis
// values (k_gsmooth_scatter), the neighbour blend (k_gsmooth_vertex), and the
// gather (k_gsmooth_gather); products and sums rounded explicitly in the
// reference's order.
__global__ void k_gsmooth_scatter(int np, const int32_t* __restrict__ dof_off, const int32_t* __restrict__ ref_vertex,
                                  const uint8_t* __restrict__ ref_axis, const double* __restrict__ g,
                                  double* __restrict__ vg, uint8_t* __restrict__ has) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= np) return;
    for (int r = dof_off[j]; r < dof_off[j + 1]; ++r) {
        const size_t idx = 3 * (size_t)ref_vertex[r] + ref_axis[r];
        vg[idx] = g[j];
        has[idx] = 1;
    }
}

__global__ void k_gsmooth_vertex(int V, const int32_t* __restrict__ nb_off, const int32_t* __restrict__ nb,
                                 const double* __restrict__ vg, const uint8_t* __restrict__ has, double w,
                                 double* __restrict__ sg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * V) return;
    if (!has[i]) return;
    const int v = i / 3, a = i % 3;
    double sum = 0.0;
    int n = 0;
    for (int k = nb_off[v]; k < nb_off[v + 1]; ++k) {
        const size_t ni = 3 * (size_t)nb[k] + a;
        if (has[ni]) {
            sum = __dadd_rn(sum, vg[ni]);
            ++n;
        }
    }
    if (n > 0) {
        const double mean = __ddiv_rn(sum, (double)n);
        sg[i] = __dadd_rn(__dmul_rn(__dsub_rn(1.0, w), vg[i]), __dmul_rn(w, mean));
    } else {
        sg[i] = vg[i];
    }
}

__global__ void k_gsmooth_gather(int np, const int32_t* __restrict__ dof_off, const int32_t* __restrict__ ref_vertex,
                                 const uint8_t* __restrict__ ref_axis, const double* __restrict__ g,
                                 const double* __restrict__ sg, double* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= np) return;
    const int r = dof_off[j + 1] - 1;
    out[j] = r >= dof_off[j] ? sg[3 * (size_t)ref_vertex[r] + ref_axis[r]] : g[j];
}

}  // namespace litho_b200
