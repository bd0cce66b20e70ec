// Mixed-precision (FP32 bulk, FP64 near field) forward and gradient kernels.
//
// Why the split: the facet formula of the reference (sum_i d_perp_i Lambda_i
// - h Omega, faceNagyContribution gravity_forward.cpp:13-42) is a
// cancellation.  Over a closed lithology surface the edge terms are ~100-500
// times larger than their sum, so FP32 rounding of Lambda and of the edge
// coefficients alone costs 1e-6..5e-6 relative in gz.  Two facts fix it:
//  * a facet far from a station tile (centroid distance >= tau x facet size)
//    is integrated directly: gz facet = n_z * integral of 1/r over the facet,
//    evaluated with Radon's 7-point degree-5 rule in FP32 (positive terms, no
//    cancellation);
//  * a facet near the tile uses the analytic formula in FP64, in the facet's
//    local frame (origin at a vertex, x along the longest edge, z along the
//    unit normal).
// The TMI facet term of the reference (magneticFacet magnetic_forward.cpp:
// 312-347) has no such cancellation; far facets evaluate it analytically in
// FP32, with Lambda formed in the orientation that avoids the d + s
// cancellation and taken as log1p of an accurately formed ratio.
#pragma once
#include "kernels_fp64.cuh"

namespace litho_b200 {

// Mixed facet constants, SoA [NMC][T] (FP64; FP32 copies are made in shared
// memory).  The local frame starts at vertex `a` of the facet rotated so that
// a->b is the longest edge; magnetic products follow that rotation.
enum MixedConst {
    MC_AX = 0, MC_AY, MC_AZ,          // local origin
    MC_XX, MC_XY, MC_XZ,              // local x axis
    MC_YX, MC_YY, MC_YZ,              // local y axis
    MC_ZX, MC_ZY, MC_ZZ,              // local z axis (unit normal)
    MC_L0, MC_CX, MC_CY,              // b = (L0, 0, 0), c = (CX, CY, 0)
    MC_E1X, MC_E1Y, MC_L1,            // edge b->c
    MC_E2X, MC_E2Y, MC_L2,            // edge c->a
    MC_SGZ,                           // n_z * G * rho * 1e3 * 1e5 (gz facet scale)
    MC_MF, MC_MT0, MC_MT1, MC_MT2,    // -amp*100/(4 pi) * direction products (TMI facet scales)
    MC_CENX, MC_CENY, MC_CENZ,        // centroid (near/far test)
    MC_SIZE,                          // longest edge
    MC_VALID,                         // 1: facet contributes (twice-area >= 1e-15)
    NMC
};

// Radon's 7-point degree-5 rule on the triangle: barycentric (beta_b, beta_c)
// of each point and its weight (weights sum to 1; multiply by the area).
// Points: centroid; (a1,b1,b1) perms with b1 = (6 - sqrt 15)/21, a1 = 1 - 2 b1,
// weight (155 - sqrt 15)/1200; (a2,b2,b2) perms with b2 = (6 + sqrt 15)/21,
// weight (155 + sqrt 15)/1200; the centroid weighs 9/40.
__constant__ float kRadonBb[7] = {0.3333333333333333f, 0.1012865073234563f, 0.7974269853530873f,
                                  0.1012865073234563f, 0.4701420641051151f, 0.0597158717897698f,
                                  0.4701420641051151f};
__constant__ float kRadonBc[7] = {0.3333333333333333f, 0.1012865073234563f, 0.1012865073234563f,
                                  0.7974269853530873f, 0.4701420641051151f, 0.4701420641051151f,
                                  0.0597158717897698f};
__constant__ float kRadonW[7] = {0.225f, 0.1259391805448271f, 0.1259391805448271f, 0.1259391805448271f,
                                 0.1323941527885062f, 0.1323941527885062f, 0.1323941527885062f};

__global__ void k_face_prep_mixed(int T, const int32_t* __restrict__ tri, const double* __restrict__ pos,
                                  const int16_t* __restrict__ face_group, const GroupConst* __restrict__ groups, d3 fdir,
                                  double* __restrict__ mc) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= T) return;
    d3 v[3];
    for (int k = 0; k < 3; ++k) {
        const double* p = pos + 3 * tri[3 * f + k];
        v[k] = mk3(p[0], p[1], p[2]);
    }
    // reference-order normal and magnetic products (bit-identical to the
    // reference, which matters for facets collapsed to a line)
    d3 n = cross_rn(sub_rn(v[1], v[0]), sub_rn(v[2], v[0]));
    double area2 = norm_rn(n);
    double out[NMC];
    for (int k = 0; k < NMC; ++k) out[k] = 0.0;
    if (!(area2 < kEps)) {
        d3 un = div_rn(n, area2);
        const GroupConst& g = groups[face_group[f]];
        d3 m = mk3(g.mdir[0], g.mdir[1], g.mdir[2]);
        double mf = __dmul_rn(dot_rn(m, un), dot_rn(fdir, un));
        double mt[3], L[3];
        for (int i = 0; i < 3; ++i) {
            d3 e = sub_rn(v[(i + 1) % 3], v[i]);
            L[i] = norm_rn(e);
            d3 eh = (L[i] < kEps) ? mk3(0, 0, 0) : div_rn(e, L[i]);
            d3 perp = cross_rn(un, eh);
            mt[i] = __dmul_rn(dot_rn(m, perp), dot_rn(fdir, perp));
        }
        int k = 0;  // rotate so that edge 0 is the longest
        if (L[1] > L[k]) k = 1;
        if (L[2] > L[k]) k = 2;
        d3 a = v[k], b = v[(k + 1) % 3], c = v[(k + 2) % 3];
        double L0 = L[k];
        d3 xh = (b - a) * (1.0 / L0);
        // On a facet collapsed onto a line the reference's unit normal is
        // rounding noise and not perpendicular to the edges; the frame must
        // stay orthonormal for the local coordinates (and so Lambda, which the
        // reference takes from positions alone) to be right.
        d3 zh = un - xh * dot3(un, xh);
        zh = zh * (1.0 / norm3(zh));
        d3 yh = cross3(zh, xh);
        d3 ca = c - a;
        double cx = dot3(ca, xh), cy = dot3(ca, yh);
        double L1 = L[(k + 1) % 3], L2 = L[(k + 2) % 3];
        out[MC_AX] = a.x; out[MC_AY] = a.y; out[MC_AZ] = a.z;
        out[MC_XX] = xh.x; out[MC_XY] = xh.y; out[MC_XZ] = xh.z;
        out[MC_YX] = yh.x; out[MC_YY] = yh.y; out[MC_YZ] = yh.z;
        out[MC_ZX] = zh.x; out[MC_ZY] = zh.y; out[MC_ZZ] = zh.z;
        out[MC_L0] = L0; out[MC_CX] = cx; out[MC_CY] = cy;
        out[MC_L1] = L1; out[MC_L2] = L2;
        if (!(L1 < kEps)) { out[MC_E1X] = (cx - L0) / L1; out[MC_E1Y] = cy / L1; }
        if (!(L2 < kEps)) { out[MC_E2X] = -cx / L2; out[MC_E2Y] = -cy / L2; }
        out[MC_SGZ] = un.z * g.gscale_fwd;
        out[MC_MF] = -g.mscale * mf;
        out[MC_MT0] = -g.mscale * mt[k];
        out[MC_MT1] = -g.mscale * mt[(k + 1) % 3];
        out[MC_MT2] = -g.mscale * mt[(k + 2) % 3];
        out[MC_CENX] = (v[0].x + v[1].x + v[2].x) / 3.0;
        out[MC_CENY] = (v[0].y + v[1].y + v[2].y) / 3.0;
        out[MC_CENZ] = (v[0].z + v[1].z + v[2].z) / 3.0;
        out[MC_SIZE] = L0;
        out[MC_VALID] = 1.0;
    }
    for (int k = 0; k < NMC; ++k) mc[(size_t)k * T + f] = out[k];
}

// ----------------------------------------------------------- FP32 pieces --
// Lambda in the orientation without the d + s cancellation:
// forward  log((s2+d2)/(s1+d1)) = log1p((L + sigma)/(s1 + d1)),
// reverse  log((d1-s1)/(d2-s2)) = log1p((L - sigma)/(d2 - s2)),
// sigma = d2 - d1 = L (s1 + s2) / (d1 + d2).
__device__ __forceinline__ float lam_f32(float s1, float s2, float d1, float d2, float L) {
    float ss = s1 + s2;
    float sig = L * ss / (d1 + d2);
    float delta, den;
    if (ss >= 0.f) { delta = L + sig; den = s1 + d1; }
    else           { delta = L - sig; den = d2 - s2; }
    return log1pf(delta / den);
}

struct FaceF32 {
    float rx[3], ry[3], rz[3];  // rows of the local frame
    float L0, cx, cy, e1x, e1y, L1, e2x, e2y, L2;
    float gq;                   // n_z * gscale * area (quadrature scale)
    float mf, mt0, mt1, mt2;
    float qx[7], qy[7];         // quadrature points in the local frame
};

// Far pair: gz by quadrature, TMI analytic, both FP32.  (x, y, z): station
// in the facet's local frame.
__device__ __forceinline__ void pair_far_f32(const FaceF32& F, float x, float y, float z, float* gz, float* tmi) {
    float z2 = z * z;
    // gz: n_z * gscale * A * sum_q w_q / r_q
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        float dx = F.qx[q] - x, dy = F.qy[q] - y;
        acc = fmaf(kRadonW[q], rsqrtf(fmaf(dx, dx, fmaf(dy, dy, z2))), acc);
    }
    *gz += F.gq * acc;
    // TMI: MF * Omega + sum_i MT_i Lambda_i
    float rbx = F.L0 - x, rcx = F.cx - x, rcy = F.cy - y;
    float la = sqrtf(fmaf(x, x, fmaf(y, y, z2)));
    float lb = sqrtf(fmaf(rbx, rbx, fmaf(y, y, z2)));
    float lc = sqrtf(fmaf(rcx, rcx, fmaf(rcy, rcy, z2)));
    float dab = fmaf(-x, rbx, fmaf(y, y, z2));
    float dac = fmaf(-x, rcx, fmaf(-y, rcy, z2));
    float dbc = fmaf(rbx, rcx, fmaf(-y, rcy, z2));
    float den = la * lb * lc + dab * lc + dac * lb + dbc * la;
    float om = 2.f * atan2f(-z * (F.L0 * F.cy), den);
    float l0 = lam_f32(-x, rbx, la, lb, F.L0);
    float l1 = lam_f32(fmaf(rbx, F.e1x, -y * F.e1y), fmaf(rcx, F.e1x, rcy * F.e1y), lb, lc, F.L1);
    float l2 = lam_f32(fmaf(rcx, F.e2x, rcy * F.e2y), fmaf(-x, F.e2x, -y * F.e2y), lc, la, F.L2);
    *tmi += F.mf * om + F.mt0 * l0 + F.mt1 * l1 + F.mt2 * l2;
}

// Near pair in FP64, local frame, with the reference's lineIntegralTerm and
// solidAngle branch semantics.  Adds gz and TMI contributions.
__device__ __forceinline__ void pair_near_f64(const double* __restrict__ s, int j, int stride, d3 o, double* gz,
                                              double* tmi) {
#define M(k) s[(k) * stride + j]
    double dx = o.x - M(MC_AX), dy = o.y - M(MC_AY), dz = o.z - M(MC_AZ);
    double x = dx * M(MC_XX) + dy * M(MC_XY) + dz * M(MC_XZ);
    double y = dx * M(MC_YX) + dy * M(MC_YY) + dz * M(MC_YZ);
    double z = dx * M(MC_ZX) + dy * M(MC_ZY) + dz * M(MC_ZZ);
    double L0 = M(MC_L0), cx = M(MC_CX), cy = M(MC_CY);
    double rbx = L0 - x, rcx = cx - x, rcy = cy - y, z2 = z * z;
    double la = sqrt(x * x + y * y + z2), lb = sqrt(rbx * rbx + y * y + z2), lc = sqrt(rcx * rcx + rcy * rcy + z2);
    double h = -z;
    double om = 0.0;
    if (!(la < kEps || lb < kEps || lc < kEps)) {
        double den = la * lb * lc + (-x * rbx + y * y + z2) * lc + (-x * rcx - y * rcy + z2) * lb +
                     (rbx * rcx - y * rcy + z2) * la;
        om = 2.0 * atan2(h * (L0 * cy), den);
    }
    bool live;
    double lam0 = (L0 < kEps) ? 0.0 : lambda_from(-x, rbx, la, lb, &live);
    double e1x = M(MC_E1X), e1y = M(MC_E1Y), e2x = M(MC_E2X), e2y = M(MC_E2Y);
    double lam1 = (M(MC_L1) < kEps) ? 0.0 : lambda_from(rbx * e1x - y * e1y, rcx * e1x + rcy * e1y, lb, lc, &live);
    double lam2 = (M(MC_L2) < kEps) ? 0.0 : lambda_from(rcx * e2x + rcy * e2y, -x * e2x - y * e2y, lc, la, &live);
    // d_perp_i = -(r1 . perp_i), perp_i = z x e_i = (-e_y, e_x, 0)
    double dp0 = y;
    double dp1 = rbx * e1y + y * e1x;
    double dp2 = rcx * e2y - rcy * e2x;
    *gz += M(MC_SGZ) * (dp0 * lam0 + dp1 * lam1 + dp2 * lam2 - h * om);
    *tmi += M(MC_MF) * om + M(MC_MT0) * lam0 + M(MC_MT1) * lam1 + M(MC_MT2) * lam2;
#undef M
}

// Station tiles of 128 (stations pre-ordered along a Morton curve so a tile
// is spatially compact) x facet chunks.  A facet is far for the whole tile
// when its centroid is at least tau x size from the tile's bounding box.
template <bool GZ, bool TMI, int FT>
__global__ void __launch_bounds__(128) k_forward_mixed(int S, const double* __restrict__ sta, int T,
                                                       const double* __restrict__ mc, const int32_t* __restrict__ chunk_begin,
                                                       const int32_t* __restrict__ chunk_end, float tau,
                                                       double* __restrict__ part_gz, double* __restrict__ part_tmi,
                                                       unsigned long long* __restrict__ near_pairs) {
    __shared__ double smd[NMC * FT];
    __shared__ FaceF32 smf[FT];
    __shared__ float bbox[6];
    __shared__ float red[6][4];
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    int chunk = blockIdx.y;
    int fb = chunk_begin[chunk], fe = chunk_end[chunk];
    d3 o = mk3(0, 0, 0);
    bool act = s < S;
    if (act) o = mk3(sta[3 * s], sta[3 * s + 1], sta[3 * s + 2]);
    // tile bounding box (warp shuffles, then across the 4 warps)
    {
        float v[6] = {act ? (float)o.x : 3e38f, act ? (float)o.y : 3e38f, act ? (float)o.z : 3e38f,
                      act ? -(float)o.x : 3e38f, act ? -(float)o.y : 3e38f, act ? -(float)o.z : 3e38f};
        for (int k = 0; k < 6; ++k)
            for (int off = 16; off > 0; off >>= 1) v[k] = fminf(v[k], __shfl_xor_sync(0xffffffffu, v[k], off));
        int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0)
            for (int k = 0; k < 6; ++k) red[k][w] = v[k];
        __syncthreads();
        if (threadIdx.x < 6) {
            float m = red[threadIdx.x][0];
            for (int q = 1; q < (int)(blockDim.x >> 5); ++q) m = fminf(m, red[threadIdx.x][q]);
            bbox[threadIdx.x] = threadIdx.x < 3 ? m : -m;
        }
    }
    double gz = 0.0, tmi = 0.0;
    unsigned long long nearCount = 0;
    for (int f0 = fb; f0 < fe; f0 += FT) {
        int nf = min(FT, fe - f0);
        __syncthreads();
        for (int idx = threadIdx.x; idx < NMC * FT; idx += blockDim.x) {
            int k = idx / FT, j = idx % FT;
            smd[idx] = (j < nf) ? mc[(size_t)k * T + f0 + j] : 0.0;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < nf; j += blockDim.x) {
            FaceF32& F = smf[j];
#define M(k) smd[(k) * FT + j]
            F.rx[0] = (float)M(MC_XX); F.rx[1] = (float)M(MC_XY); F.rx[2] = (float)M(MC_XZ);
            F.ry[0] = (float)M(MC_YX); F.ry[1] = (float)M(MC_YY); F.ry[2] = (float)M(MC_YZ);
            F.rz[0] = (float)M(MC_ZX); F.rz[1] = (float)M(MC_ZY); F.rz[2] = (float)M(MC_ZZ);
            F.L0 = (float)M(MC_L0); F.cx = (float)M(MC_CX); F.cy = (float)M(MC_CY);
            F.e1x = (float)M(MC_E1X); F.e1y = (float)M(MC_E1Y); F.L1 = (float)M(MC_L1);
            F.e2x = (float)M(MC_E2X); F.e2y = (float)M(MC_E2Y); F.L2 = (float)M(MC_L2);
            F.gq = (float)(M(MC_SGZ) * 0.5 * M(MC_L0) * M(MC_CY));
            F.mf = (float)M(MC_MF); F.mt0 = (float)M(MC_MT0); F.mt1 = (float)M(MC_MT1); F.mt2 = (float)M(MC_MT2);
            for (int q = 0; q < 7; ++q) {
                F.qx[q] = kRadonBb[q] * F.L0 + kRadonBc[q] * F.cx;
                F.qy[q] = kRadonBc[q] * F.cy;
            }
#undef M
        }
        __syncthreads();
        if (act) {
            float gacc = 0.f, tacc = 0.f;
            for (int j = 0; j < nf; ++j) {
                if (smd[MC_VALID * FT + j] == 0.0) continue;
                // uniform over the CTA: centroid vs tile bounding box
                float cxw = (float)smd[MC_CENX * FT + j], cyw = (float)smd[MC_CENY * FT + j],
                      czw = (float)smd[MC_CENZ * FT + j];
                float ddx = fmaxf(0.f, fmaxf(bbox[0] - cxw, cxw - bbox[3]));
                float ddy = fmaxf(0.f, fmaxf(bbox[1] - cyw, cyw - bbox[4]));
                float ddz = fmaxf(0.f, fmaxf(bbox[2] - czw, czw - bbox[5]));
                float lim = tau * (float)smd[MC_SIZE * FT + j];
                bool far = ddx * ddx + ddy * ddy + ddz * ddz >= lim * lim;
                if (far) {
                    const FaceF32& F = smf[j];
                    double ddx = o.x - smd[MC_AX * FT + j], ddy = o.y - smd[MC_AY * FT + j],
                           ddz = o.z - smd[MC_AZ * FT + j];
                    float dx = (float)ddx, dy = (float)ddy, dz = (float)ddz;
                    float x = fmaf(dx, F.rx[0], fmaf(dy, F.rx[1], dz * F.rx[2]));
                    float y = fmaf(dx, F.ry[0], fmaf(dy, F.ry[1], dz * F.ry[2]));
                    // the height above the facet plane can be tiny next to |o - a|
                    // (a far top facet seen from 1 m above it): FP64
                    float z = (float)(ddx * smd[MC_ZX * FT + j] + ddy * smd[MC_ZY * FT + j] + ddz * smd[MC_ZZ * FT + j]);
                    float g1 = 0.f, t1 = 0.f;
                    pair_far_f32(F, x, y, z, &g1, &t1);
                    if (GZ) gacc += g1;
                    if (TMI) tacc += t1;
                } else {
                    double g1 = 0.0, t1 = 0.0;
                    pair_near_f64(smd, j, FT, o, &g1, &t1);
                    if (GZ) gz += g1;
                    if (TMI) tmi += t1;
                    ++nearCount;
                }
            }
            gz += gacc;
            tmi += tacc;
        }
    }
    if (act) {
        if (GZ) part_gz[(size_t)chunk * S + s] = gz;
        if (TMI) part_tmi[(size_t)chunk * S + s] = tmi;
        if (near_pairs && nearCount) atomicAdd(near_pairs, nearCount);
    }
}

// ---------------------------------------------------- far-field gradient --
// Facet-per-thread twin of k_gradient_fp64 for the station tiles it skips
// (every facet of the warp far from the tile).  In FP32:
//  * gz: I = A sum_q w_q / r_q, so
//      sum_s G0 dI/dv = (dA/dv) Q0 - A sum_q beta_qv D_q,
//    Q0 = sum_s G0 sum_q w_q / r_q, D_q = sum_s G0 w_q (p_q - o) / r_q^3
//    (G0 = gravity adjoint x group scale; n_z enters at the flush and, for
//    its own derivative, through the shared finalisation);
//  * TMI: the closed-form d Omega / dv and d Lambda / dv of the FP64 kernel.
// FP32 sums run over one station tile (<= 64 stations) and are flushed into
// the FP64 accumulators, then the FP64 finalisation differentiates the facet
// constants once.
__global__ void __launch_bounds__(32) k_gradient_far32(int T, const double* __restrict__ gc, int S,
                                                       const double* __restrict__ sta, const double* __restrict__ gcoef,
                                                       const double* __restrict__ mcoef, int stations_per_chunk,
                                                       const double* __restrict__ tile_box,
                                                       const int16_t* __restrict__ face_group,
                                                       const GroupConst* __restrict__ groups, d3 fdir, double tau,
                                                       double* __restrict__ part) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    int chunk = blockIdx.y;
    int sb = chunk * stations_per_chunk, se = min(S, sb + stations_per_chunk);
    bool active = false;
    double C[NGC];
    if (f < T) {
#pragma unroll
        for (int k = 0; k < NGC; ++k) C[k] = gc[(size_t)k * T + f];
        int flags = static_cast<int>(C[GC_FLAGS]);
        active = (flags & 1) && (flags & 2) && (C[GC_GS] != 0.0 || C[GC_MS] != 0.0);
    } else {
        for (int k = 0; k < NGC; ++k) C[k] = 0.0;
    }
    GradAcc A;
    grad_acc_zero(A);
    // FP32 facet constants
    const float L0 = (float)C[GC_L0], cx = (float)C[GC_CX], cy = (float)C[GC_CY];
    const float e1x = (float)C[GC_E1X], e1y = (float)C[GC_E1Y], L1 = (float)C[GC_L1];
    const float e2x = (float)C[GC_E2X], e2y = (float)C[GC_E2Y], L2 = (float)C[GC_L2];
    const float rx0 = (float)C[GC_XX], rx1 = (float)C[GC_XY], rx2 = (float)C[GC_XZ];
    const float ry0 = (float)C[GC_YX], ry1 = (float)C[GC_YY], ry2 = (float)C[GC_YZ];
    const float mf = (float)C[GC_MF], mt0 = (float)C[GC_MT0], mt1 = (float)C[GC_MT1], mt2 = (float)C[GC_MT2];
    const float A2 = L0 * cy;
    const double gsn = C[GC_GS], ms = C[GC_MS];
    float qx[7], qy[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        qx[q] = kRadonBb[q] * L0 + kRadonBc[q] * cx;
        qy[q] = kRadonBc[q] * cy;
    }
    for (int s0 = sb; s0 < se; s0 += kStationTile) {
        int ns = min(kStationTile, se - s0);
        bool allFar = __all_sync(0xffffffffu, facet_far(C, active, tile_box + 6 * (s0 / kStationTile), tau));
        if (!active || !allFar) continue;
        float q0 = 0.f;
        float dqx[7], dqy[7], dqz[7];
#pragma unroll
        for (int q = 0; q < 7; ++q) dqx[q] = dqy[q] = dqz[q] = 0.f;
        float vax = 0.f, vay = 0.f, vaz = 0.f, vbx = 0.f, vby = 0.f, vbz = 0.f, vcx = 0.f, vcy = 0.f, vcz = 0.f;
        float amf = 0.f, amt0 = 0.f, amt1 = 0.f, amt2 = 0.f;
        for (int j = s0; j < s0 + ns; ++j) {
            float G0 = (float)((gcoef ? gcoef[j] : 0.0) * gsn);
            float Ts = (float)((mcoef ? mcoef[j] : 0.0) * ms);
            if (G0 == 0.f && Ts == 0.f) continue;
            double ddx = sta[3 * j] - C[GC_AX], ddy = sta[3 * j + 1] - C[GC_AY], ddz = sta[3 * j + 2] - C[GC_AZ];
            float dx = (float)ddx, dy = (float)ddy, dz = (float)ddz;
            float x = fmaf(dx, rx0, fmaf(dy, rx1, dz * rx2));
            float y = fmaf(dx, ry0, fmaf(dy, ry1, dz * ry2));
            float z = (float)(ddx * C[GC_ZX] + ddy * C[GC_ZY] + ddz * C[GC_ZZ]);
            float z2 = z * z;
            if (G0 != 0.f) {
                float sw = 0.f;
#pragma unroll
                for (int q = 0; q < 7; ++q) {
                    float px = qx[q] - x, py = qy[q] - y;
                    float rs = rsqrtf(fmaf(px, px, fmaf(py, py, z2)));
                    float w = kRadonW[q] * rs;
                    sw += w;
                    float g3 = G0 * w * rs * rs;
                    dqx[q] = fmaf(g3, px, dqx[q]);
                    dqy[q] = fmaf(g3, py, dqy[q]);
                    dqz[q] = fmaf(g3, -z, dqz[q]);
                }
                q0 = fmaf(G0, sw, q0);
            }
            if (Ts != 0.f) {
                float rbx = L0 - x, rcx = cx - x, rcy = cy - y;
                float la = sqrtf(fmaf(x, x, fmaf(y, y, z2)));
                float lb = sqrtf(fmaf(rbx, rbx, fmaf(y, y, z2)));
                float lc = sqrtf(fmaf(rcx, rcx, fmaf(rcy, rcy, z2)));
                float dab = fmaf(-x, rbx, fmaf(y, y, z2));
                float dac = fmaf(-x, rcx, fmaf(-y, rcy, z2));
                float dbc = fmaf(rbx, rcx, fmaf(-y, rcy, z2));
                float den = la * lb * lc + dab * lc + dac * lb + dbc * la;
                float om = 2.f * atan2f(-z * A2, den);
                float s11 = fmaf(rbx, e1x, -y * e1y), s12 = fmaf(rcx, e1x, rcy * e1y);
                float s21 = fmaf(rcx, e2x, rcy * e2y), s22 = fmaf(-x, e2x, -y * e2y);
                float l0 = lam_f32(-x, rbx, la, lb, L0);
                float l1 = lam_f32(s11, s12, lb, lc, L1);
                float l2 = lam_f32(s21, s22, lc, la, L2);
                float ia = 1.f / la, ib = 1.f / lb, ic = 1.f / lc;
                float kom = Ts * mf;
                // edge (p1 -> p2): W = L / (d1 d2 + r1.r2), q = r1 - s1 e, Z = e x r1,
                // P = W (kom Z - kl q); p1 += (P - kl e)/d1, p2 += (P + kl e)/d2
                auto edge = [&](float r1x, float r1y, float r2x, float r2y, float d1, float d2, float ex, float ey,
                                float L, float s1, float kl, float i1, float i2, float& g1x, float& g1y, float& g1z,
                                float& g2x, float& g2y, float& g2z) {
                    float W = L / fmaf(d1, d2, fmaf(r1x, r2x, fmaf(r1y, r2y, z2)));
                    float qxv = fmaf(-s1, ex, r1x), qyv = fmaf(-s1, ey, r1y), qzv = -z;
                    float Zx = -ey * z, Zy = ex * z, Zz = fmaf(ex, r1y, -ey * r1x);  // e x r1, r1.z = -z
                    float Px = W * fmaf(kom, Zx, -kl * qxv), Py = W * fmaf(kom, Zy, -kl * qyv),
                          Pz = W * fmaf(kom, Zz, -kl * qzv);
                    g1x = fmaf(fmaf(-kl, ex, Px), i1, g1x); g1y = fmaf(fmaf(-kl, ey, Py), i1, g1y); g1z = fmaf(Pz, i1, g1z);
                    g2x = fmaf(fmaf(kl, ex, Px), i2, g2x); g2y = fmaf(fmaf(kl, ey, Py), i2, g2y); g2z = fmaf(Pz, i2, g2z);
                };
                edge(-x, -y, rbx, -y, la, lb, 1.f, 0.f, L0, -x, Ts * mt0, ia, ib, vax, vay, vaz, vbx, vby, vbz);
                edge(rbx, -y, rcx, rcy, lb, lc, e1x, e1y, L1, s11, Ts * mt1, ib, ic, vbx, vby, vbz, vcx, vcy, vcz);
                edge(rcx, rcy, -x, -y, lc, la, e2x, e2y, L2, s21, Ts * mt2, ic, ia, vcx, vcy, vcz, vax, vay, vaz);
                amf = fmaf(Ts, om, amf);
                amt0 = fmaf(Ts, l0, amt0); amt1 = fmaf(Ts, l1, amt1); amt2 = fmaf(Ts, l2, amt2);
            }
        }
        // flush the tile into the FP64 accumulators (local frame)
        const double nz = C[GC_ZZ];
        const double Ar = 0.5 * C[GC_L0] * C[GC_CY];
        double sa[3] = {0, 0, 0}, sbv[3] = {0, 0, 0}, sc[3] = {0, 0, 0};
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            double bb = kRadonBb[q], bc = kRadonBc[q], ba = 1.0 - bb - bc;
            sa[0] += ba * dqx[q]; sa[1] += ba * dqy[q]; sa[2] += ba * dqz[q];
            sbv[0] += bb * dqx[q]; sbv[1] += bb * dqy[q]; sbv[2] += bb * dqz[q];
            sc[0] += bc * dqx[q]; sc[1] += bc * dqy[q]; sc[2] += bc * dqz[q];
        }
        const double cxd = C[GC_CX], cyd = C[GC_CY], L0d = C[GC_L0];
        // dA/da = (-cy, cx - L0, 0)/2, dA/db = (cy, -cx, 0)/2, dA/dc = (0, L0, 0)/2
        A.va = A.va + mk3(nz * (-0.5 * cyd * q0 - Ar * sa[0]) + vax, nz * (0.5 * (cxd - L0d) * q0 - Ar * sa[1]) + vay,
                          nz * (-Ar * sa[2]) + vaz);
        A.vb = A.vb + mk3(nz * (0.5 * cyd * q0 - Ar * sbv[0]) + vbx, nz * (-0.5 * cxd * q0 - Ar * sbv[1]) + vby,
                          nz * (-Ar * sbv[2]) + vbz);
        A.vc = A.vc + mk3(nz * (-Ar * sc[0]) + vcx, nz * (0.5 * L0d * q0 - Ar * sc[1]) + vcy, nz * (-Ar * sc[2]) + vcz);
        A.ai += Ar * q0;
        A.amf += amf;
        A.amt[0] += amt0; A.amt[1] += amt1; A.amt[2] += amt2;
    }
    if (f >= T) return;
    double outv[9];
    if (!active) {
        for (int k = 0; k < 9; ++k) outv[k] = 0.0;
    } else {
        grad_finalize(C, A, groups[face_group[f]], fdir, outv);
    }
    for (int k = 0; k < 9; ++k) part[((size_t)chunk * 9 + k) * T + f] = outv[k];
}

// Per station: sum of chunk partials (facet scales are already applied).
__global__ void k_forward_reduce_mixed(int S, int nchunks, const double* __restrict__ part_gz,
                                       const double* __restrict__ part_tmi, double* __restrict__ gz,
                                       double* __restrict__ tmi) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    double g = 0.0, t = 0.0;
    for (int c = 0; c < nchunks; ++c) {
        if (part_gz) g += part_gz[(size_t)c * S + s];
        if (part_tmi) t += part_tmi[(size_t)c * S + s];
    }
    if (gz) gz[s] = g;
    if (tmi) tmi[s] = t;
}

}  // namespace litho_b200
