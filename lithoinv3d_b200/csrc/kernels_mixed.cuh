// Mixed-precision (FP32 bulk, FP64 near field) forward and gradient kernels.
//
// Why the split: the facet formula of the reference (sum_i d_perp_i Lambda_i
// - h Omega, faceNagyContribution gravity_forward.cpp:13-42) is a
// cancellation.  Over a closed lithology surface the edge terms are ~100-500
// times larger than their sum, so FP32 rounding of Lambda and of the edge
// coefficients alone costs 1e-6..5e-6 relative in gz.  Two facts fix it:
//  * a facet far from a station tile (centroid distance >= tau x facet size)
//    is integrated directly: gz facet = n_z * integral of 1/r over the facet,
//    evaluated by quadrature in FP32 (positive terms, no cancellation):
//    Dunavant's 6-point degree-4 rule in the forward (3 points beyond
//    4 tau), Radon's 7-point degree-5 rule in the gradient;
//  * a facet near the tile uses the analytic formula in FP64, in the facet's
//    local frame (origin at a vertex, x along the longest edge, z along the
//    unit normal).
// The TMI facet term of the reference (magneticFacet magnetic_forward.cpp:
// 312-347) has no such cancellation; far facets evaluate it analytically in
// FP32, with Lambda from the symmetric form 2 atanh(L / (d1 + d2)).
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

// Dunavant's 6-point degree-4 rule (D. A. Dunavant, "High degree efficient
// symmetrical Gaussian quadrature rules for the triangle", IJNME 21, 1985):
// (a, b, b) permutations with a = 0.108103018168070, b = 0.445948490915965,
// weight 0.223381589678011, and a = 0.816847572980459, b = 0.091576213509771,
// weight 0.109951743655322.  Its degree-6 error term, which sets the error at
// the far-field distances, is as small as the 7-point rule's; one point fewer.
__constant__ float kDun6Bb[6] = {0.445948490915965f, 0.108103018168070f, 0.445948490915965f,
                                 0.091576213509771f, 0.816847572980459f, 0.091576213509771f};
__constant__ float kDun6Bc[6] = {0.445948490915965f, 0.445948490915965f, 0.108103018168070f,
                                 0.091576213509771f, 0.091576213509771f, 0.816847572980459f};
__constant__ float kDun6W[6] = {0.223381589678011f, 0.223381589678011f, 0.223381589678011f,
                                0.109951743655322f, 0.109951743655322f, 0.109951743655322f};
// 3-point degree-2 rule: (2/3, 1/6, 1/6) permutations, weights 1/3 (Strang &
// Fix).  Taken beyond 4 tau x size, where its (size / distance)^3 error term
// is below 1e-7 of the station total.
__constant__ float kTri3Bb[3] = {0.1666666666666667f, 0.6666666666666667f, 0.1666666666666667f};
__constant__ float kTri3Bc[3] = {0.1666666666666667f, 0.1666666666666667f, 0.6666666666666667f};

// Radon's rule on the four midpoint sub-triangles (a, ab, ca), (ab, b, bc),
// (ca, bc, c), (ab, bc, ca): 28 points in the parent's barycentric (beta_b,
// beta_c), weights kRadonW[q % 7] / 4.  Its error at distance ratio tau/2
// matches the 7-point rule's at tau (degree-5 error ~ (size / distance)^6),
// so it takes the mid field tau/2 <= distance / size < tau in FP32.
__constant__ float kRadon4Bb[28] = {
    0.1666666666666667f, 0.0506432536617282f, 0.3987134926765437f, 0.0506432536617282f, 0.2350710320525576f,
    0.0298579358948849f, 0.2350710320525576f, 0.6666666666666666f, 0.5506432536617281f, 0.8987134926765437f,
    0.5506432536617281f, 0.7350710320525575f, 0.5298579358948849f, 0.7350710320525576f, 0.1666666666666667f,
    0.0506432536617282f, 0.3987134926765437f, 0.0506432536617282f, 0.2350710320525576f, 0.0298579358948849f,
    0.2350710320525576f, 0.3333333333333334f, 0.4493567463382718f, 0.4493567463382718f, 0.1012865073234563f,
    0.2649289679474425f, 0.2649289679474425f, 0.4701420641051152f};
__constant__ float kRadon4Bc[28] = {
    0.1666666666666667f, 0.0506432536617282f, 0.0506432536617282f, 0.3987134926765437f, 0.2350710320525576f,
    0.2350710320525576f, 0.0298579358948849f, 0.1666666666666667f, 0.0506432536617282f, 0.0506432536617282f,
    0.3987134926765437f, 0.2350710320525576f, 0.2350710320525576f, 0.0298579358948849f, 0.6666666666666667f,
    0.5506432536617282f, 0.5506432536617282f, 0.8987134926765437f, 0.7350710320525575f, 0.7350710320525575f,
    0.5298579358948849f, 0.3333333333333333f, 0.1012865073234563f, 0.4493567463382718f, 0.4493567463382718f,
    0.4701420641051151f, 0.2649289679474425f, 0.2649289679474425f};

// ----------------------------------------------------------- FP32 pieces --
// sqrt for arguments known to be positive and normal (far-field distances):
// r2 * rsqrt(r2), within 2 ulp.
__device__ __forceinline__ float sqrt_pos(float r2) { return r2 * rsqrtf(r2); }

// Lambda of an edge of length L whose end points lie at distances d1, d2
// from the station: the line integral of 1/r along the edge,
//   Lambda = log((d1 + d2 + L) / (d1 + d2 - L)) = 2 atanh(v),  v = L / (d1 + d2),
// equal to the reference's oriented form log((s2 + d2) / (s1 + d1)) because
// d2^2 - d1^2 = s2^2 - s1^2 along the edge's line.  Away from the edge (every
// FP32 pair) d1 + d2 - L does not cancel.  For v <= 0.2 the series
// 2 (v + v^3/3 + ... + v^9/9) (Abramowitz & Stegun 4.1.28), whose first
// omitted term is below 2e-9 v, else log1pf(2v / (1 - v)).  The arguments are
// bounded away from zero and overflow, so the 2-ulp quotient is used.
// atanh(v) for 0 <= v <= 0.2 by the series above (Lambda = 2 atanh(v)).
__device__ __forceinline__ float atanh_series(float v) {
    const float v2 = v * v;
    const float p = fmaf(v2, fmaf(v2, fmaf(v2, fmaf(v2, 1.f / 9.f, 1.f / 7.f), 1.f / 5.f), 1.f / 3.f), 1.f);
    return v * p;
}

__device__ __forceinline__ float lam_f32(float d1, float d2, float L) {
    const float v = __fdividef(L, d1 + d2);
    if (v <= 0.2f) return 2.f * atanh_series(v);
    return log1pf(__fdividef(2.f * v, 1.f - v));
}

// atan(t) for |t| <= 1/8: the Maclaurin series through t^9 (Abramowitz &
// Stegun 4.4.42; first omitted term below 1e-10 t).
__device__ __forceinline__ float atan_series(float t) {
    const float t2 = t * t;
    const float p = fmaf(t2, fmaf(t2, fmaf(t2, fmaf(t2, 1.f / 9.f, -1.f / 7.f), 1.f / 5.f), -1.f / 3.f), 1.f);
    return t * p;
}

// atan2(y, x); for x > 0 and |y| <= x / 8 (every far pair's solid angle)
// atan_series(y / x), else atan2f.
__device__ __forceinline__ float atan2_far(float y, float x) {
    if (x > 0.f && fabsf(y) <= 0.125f * x) return atan_series(__fdividef(y, x));
    return atan2f(y, x);
}

// True when a far pair lies inside both series' ranges on all four terms:
// the solid angle's atan2(ny, den) (den > 0, |ny| <= den / 8) and the three
// edges' atanh (v_i <= 0.2).  Far pairs practically always do, so one test
// replaces four per-term branches; a pair that fails it takes atan2_far /
// lam_f32, which select per term, and both routes give the same bits.
__device__ __forceinline__ bool far_series_ok(float ny, float den, float v0, float v1, float v2) {
    return den > 0.f && fabsf(ny) <= 0.125f * den && fmaxf(v0, fmaxf(v1, v2)) <= 0.2f;
}

// Near pair in FP64, local frame: solidAngle's branch semantics, Lambda in
// the symmetric form (lambda_sym: the reference's value except exactly on an
// edge's line beyond its end, where the reference's branch gives 0).  Adds
// gz and TMI contributions.
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
    double lam0 = (L0 < kEps) ? 0.0 : lambda_sym(la, lb, L0, &live);
    double e1x = M(MC_E1X), e1y = M(MC_E1Y), e2x = M(MC_E2X), e2y = M(MC_E2Y);
    double lam1 = (M(MC_L1) < kEps) ? 0.0 : lambda_sym(lb, lc, M(MC_L1), &live);
    double lam2 = (M(MC_L2) < kEps) ? 0.0 : lambda_sym(lc, la, M(MC_L2), &live);
    // d_perp_i = -(r1 . perp_i), perp_i = z x e_i = (-e_y, e_x, 0)
    double dp0 = y;
    double dp1 = rbx * e1y + y * e1x;
    double dp2 = rcx * e2y - rcy * e2x;
    *gz += M(MC_SGZ) * (dp0 * lam0 + dp1 * lam1 + dp2 * lam2 - h * om);
    *tmi += M(MC_MF) * om + M(MC_MT0) * lam0 + M(MC_MT1) * lam1 + M(MC_MT2) * lam2;
#undef M
}

// ---------------------------------------------------- far-field gradient --
// Sums v[0..31] over the warp, transposed: on return lane L holds the warp
// total of v[L] in v[0] (31 shuffles for 32 sums instead of 32 x 5).
__device__ __forceinline__ float warp_transpose_sum32(float (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
        const bool upper = (lane & step) != 0;
#pragma unroll
        for (int i = 0; i < step; ++i) {
            const float send = upper ? v[i] : v[i + step];
            const float keep = upper ? v[i + step] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, step);
        }
    }
    return v[0];
}

// Class of a (facet, tile) in the far-field gradient: 0 near (the FP64
// kernel's), 1 far (6-point rule), 2 beyond 4 tau x size (3-point rule).
// The near / far decision is tile_far's, operation for operation.
__device__ __forceinline__ int tile_gradient_class(const FarKey& k, const double* __restrict__ bbox) {
    if (k.th2 < 0.0) return 0;
    const double d0 = fmax(0.0, fmax(__dadd_rn(bbox[0], -k.c0), __dadd_rn(k.c0, -bbox[3])));
    const double d1 = fmax(0.0, fmax(__dadd_rn(bbox[1], -k.c1), __dadd_rn(k.c1, -bbox[4])));
    const double d2 = fmax(0.0, fmax(__dadd_rn(bbox[2], -k.c2), __dadd_rn(k.c2, -bbox[5])));
    const double dd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
    return dd >= __dmul_rn(16.0, k.th2) ? 2 : (dd >= k.th2 ? 1 : 0);
}

constexpr int kFarTerms = 23;      // far-field station sums per facet (listed below)
constexpr int kFarFlushTiles = 4;  // far tiles summed per lane in FP32 between warp reductions

// Far-field objective gradient in FP32: one warp per facet, lanes over the
// stations of the facet's far tiles (exactly the tiles k_gradient_warp_fp64
// leaves out: both classify with facet_far_key / tile_far).  gz by Dunavant's
// 6-point rule, the 3-point rule beyond 4 tau x size (tile_gradient_class);
// the point sums are flushed whenever the rule changes.
//  * gz: I = A sum_q w_q / r_q, so
//      sum_s G0 dI/dv = (dA/dv) Q0 - A sum_q beta_qv D_q,
//    Q0 = sum_s G0 sum_q w_q / r_q, D_q = sum_s G0 w_q (p_q - o) / r_q^3
//    (G0 = gravity adjoint x group scale, beta_qv = barycentric weight of
//    point q on vertex v; n_z enters at the end, its own derivative through
//    the shared finalisation);
//  * TMI: the closed-form d Omega / dv and d Lambda / dv of the FP64 kernel.
// Each lane sums up to kFarFlushTiles tiles (8 stations) in FP32; the 23
// sums are then reduced across the warp in one transposed pass and lane k
// adds sum k to its FP64 total.  Lane 0 gathers the totals, forms the facet
// accumulators in FP64 and finalises.  Facet list and station chunks as in
// k_gradient_warp_fp64; part layout [chunk][9][T].
// Sums: 0 Q0; 1-3, 4-6, 7-9 sum_q beta_q{a,b,c} D_q; 10-12, 13-15, 16-18 TMI
// vertex terms of a, b, c; 19 sum Ts Omega; 20-22 sum Ts Lambda_i.
// Four CTAs per SM (at most 128 registers, a few bytes of spill) ran faster
// than the unconstrained 147-register, three-CTA build on every workload
// measured (contact model -1 %, large model -3 %, 256-body batch -7 %).
__global__ void __launch_bounds__(128, 4) k_gradient_warp_far32(int T, const double* __restrict__ gc, int S,
                                                             const double* __restrict__ sta,
                                                             const double* __restrict__ gcoef,
                                                             const double* __restrict__ mcoef,
                                                             const double* __restrict__ tile_box,
                                                             const int16_t* __restrict__ face_group,
                                                             const GroupConst* __restrict__ groups, d3 fdir,
                                                             double tau, const int32_t* __restrict__ facets, int nfacets,
        int tiles_per_chunk, const int32_t* __restrict__ grp_sta_off,
        const int32_t* __restrict__ grp_tile_off, double* __restrict__ part) {
    const int lane = threadIdx.x & 31;
    const int w = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    if (w >= nfacets) return;  // warp-uniform
    const int f = facets[w];
    if (grp_sta_off) {  // batched bodies: only the facet's own body's stations
        const int g = face_group[f], sb = grp_sta_off[g];
        S = grp_sta_off[g + 1] - sb;
        sta += 3 * (size_t)sb;
        if (gcoef) gcoef += sb;
        if (mcoef) mcoef += sb;
        tile_box += 6 * (size_t)grp_tile_off[g];
    }
    // this chunk's station tiles
    const int ntiles_all = (S + kStationTile - 1) / kStationTile;
    const int tbeg = blockIdx.y * tiles_per_chunk, ntiles = min(ntiles_all, tbeg + tiles_per_chunk);
    part += (size_t)blockIdx.y * 9 * T;
    bool active, any = false;
    double tot = 0.0;
    {
        double C[NGC];
#pragma unroll
        for (int k = 0; k < NGC; ++k) C[k] = __ldg(&gc[(size_t)k * T + f]);
        active = facet_grad_active(C);
        if (active) {
            const float L0 = (float)C[GC_L0], cx = (float)C[GC_CX], cy = (float)C[GC_CY];
            const float e1x = (float)C[GC_E1X], e1y = (float)C[GC_E1Y], L1 = (float)C[GC_L1];
            const float e2x = (float)C[GC_E2X], e2y = (float)C[GC_E2Y], L2 = (float)C[GC_L2];
            const float rx0 = (float)C[GC_XX], rx1 = (float)C[GC_XY], rx2 = (float)C[GC_XZ];
            const float ry0 = (float)C[GC_YX], ry1 = (float)C[GC_YY], ry2 = (float)C[GC_YZ];
            const float mf = (float)C[GC_MF], mt0 = (float)C[GC_MT0], mt1 = (float)C[GC_MT1],
                        mt2 = (float)C[GC_MT2];
            const float A2 = L0 * cy;
            const double ax = C[GC_AX], ay = C[GC_AY], az = C[GC_AZ];
            const double zx = C[GC_ZX], zy = C[GC_ZY], zz = C[GC_ZZ];
            const double gsn = C[GC_GS], ms = C[GC_MS];
            float qx[6], qy[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                qx[q] = kDun6Bb[q] * L0 + kDun6Bc[q] * cx;
                qy[q] = kDun6Bc[q] * cy;
            }
            float q0 = 0.f, dqx[6], dqy[6], dqz[6];
            float vax = 0.f, vay = 0.f, vaz = 0.f, vbx = 0.f, vby = 0.f, vbz = 0.f, vcx = 0.f, vcy = 0.f, vcz = 0.f;
            float amf = 0.f, amt0 = 0.f, amt1 = 0.f, amt2 = 0.f;
#pragma unroll
            for (int q = 0; q < 6; ++q) dqx[q] = dqy[q] = dqz[q] = 0.f;
            int pending = 0, rule = 0;  // rule of the pending point sums: 0 six-point, 1 three-point
            auto flush = [&]() {
                float v[32];
                float sa0 = 0.f, sa1 = 0.f, sa2 = 0.f, sb0 = 0.f, sb1 = 0.f, sb2 = 0.f, sc0 = 0.f, sc1 = 0.f, sc2 = 0.f;
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    // slots 0-2 hold the three-point rule's sums when rule == 1 (slots 3-5 are then zero)
                    const float bb = rule ? (q < 3 ? kTri3Bb[q] : 0.f) : kDun6Bb[q];
                    const float bc = rule ? (q < 3 ? kTri3Bc[q] : 0.f) : kDun6Bc[q];
                    const float ba = 1.f - bb - bc;
                    sa0 = fmaf(ba, dqx[q], sa0); sa1 = fmaf(ba, dqy[q], sa1); sa2 = fmaf(ba, dqz[q], sa2);
                    sb0 = fmaf(bb, dqx[q], sb0); sb1 = fmaf(bb, dqy[q], sb1); sb2 = fmaf(bb, dqz[q], sb2);
                    sc0 = fmaf(bc, dqx[q], sc0); sc1 = fmaf(bc, dqy[q], sc1); sc2 = fmaf(bc, dqz[q], sc2);
                    dqx[q] = dqy[q] = dqz[q] = 0.f;
                }
                v[0] = q0;
                v[1] = sa0; v[2] = sa1; v[3] = sa2;
                v[4] = sb0; v[5] = sb1; v[6] = sb2;
                v[7] = sc0; v[8] = sc1; v[9] = sc2;
                v[10] = vax; v[11] = vay; v[12] = vaz;
                v[13] = vbx; v[14] = vby; v[15] = vbz;
                v[16] = vcx; v[17] = vcy; v[18] = vcz;
                v[19] = amf; v[20] = amt0; v[21] = amt1; v[22] = amt2;
#pragma unroll
                for (int k = kFarTerms; k < 32; ++k) v[k] = 0.f;
                tot += (double)warp_transpose_sum32(v);
                q0 = 0.f;
                vax = vay = vaz = vbx = vby = vbz = vcx = vcy = vcz = 0.f;
                amf = amt0 = amt1 = amt2 = 0.f;
            };
            const FarKey key = facet_far_key(C, tau);
            for (int t0 = tbeg; t0 < ntiles; t0 += 32) {
                const int t = t0 + lane;
                const int cls = t < ntiles ? tile_gradient_class(key, tile_box + 6 * (size_t)t) : 0;
                unsigned m = __ballot_sync(0xffffffffu, cls != 0);
                const unsigned mv = __ballot_sync(0xffffffffu, cls == 2);
                any |= m != 0;
                while (m) {
                    const int b = __ffs(m) - 1;
                    m &= m - 1;
                    const int r = (mv >> b) & 1u;  // warp-uniform
                    if (pending && r != rule) {  // the pending sums belong to the other rule
                        flush();
                        pending = 0;
                    }
                    rule = r;
                    const int s0 = (t0 + b) * kStationTile;
#pragma unroll
                    for (int k = 0; k < kStationTile; k += 32) {
                        const int j = s0 + k + lane;
                        float G0 = 0.f, Ts = 0.f;
                        double ox = 0.0, oy = 0.0, oz = 0.0;
                        if (j < S) {
                            G0 = (float)((gcoef ? gcoef[j] : 0.0) * gsn);
                            Ts = (float)((mcoef ? mcoef[j] : 0.0) * ms);
                            ox = sta[3 * j]; oy = sta[3 * j + 1]; oz = sta[3 * j + 2];
                        }
                        if (G0 == 0.f && Ts == 0.f) continue;
                        const double ddx = ox - ax, ddy = oy - ay, ddz = oz - az;
                        const float dx = (float)ddx, dy = (float)ddy, dzf = (float)ddz;
                        const float x = fmaf(dx, rx0, fmaf(dy, rx1, dzf * rx2));
                        const float y = fmaf(dx, ry0, fmaf(dy, ry1, dzf * ry2));
                        const float z = (float)(ddx * zx + ddy * zy + ddz * zz);
                        const float z2 = z * z;
                        if (G0 != 0.f && r) {  // beyond 4 tau: the 3-point rule, weights 1/3
                            float sw = 0.f;
#pragma unroll
                            for (int q = 0; q < 3; ++q) {
                                const float px = fmaf(kTri3Bb[q], L0, fmaf(kTri3Bc[q], cx, -x));
                                const float py = fmaf(kTri3Bc[q], cy, -y);
                                const float rs = rsqrtf(fmaf(px, px, fmaf(py, py, z2)));
                                const float w = (1.f / 3.f) * rs;
                                sw += w;
                                const float g3 = G0 * w * rs * rs;
                                dqx[q] = fmaf(g3, px, dqx[q]);
                                dqy[q] = fmaf(g3, py, dqy[q]);
                                dqz[q] = fmaf(g3, -z, dqz[q]);
                            }
                            q0 = fmaf(G0, sw, q0);
                        } else if (G0 != 0.f) {
                            float sw = 0.f;
#pragma unroll
                            for (int q = 0; q < 6; ++q) {
                                const float px = qx[q] - x, py = qy[q] - y;
                                const float rs = rsqrtf(fmaf(px, px, fmaf(py, py, z2)));
                                const float w = kDun6W[q] * rs;
                                sw += w;
                                const float g3 = G0 * w * rs * rs;
                                dqx[q] = fmaf(g3, px, dqx[q]);
                                dqy[q] = fmaf(g3, py, dqy[q]);
                                dqz[q] = fmaf(g3, -z, dqz[q]);
                            }
                            q0 = fmaf(G0, sw, q0);
                        }
                        if (Ts != 0.f) {
                            const float rbx = L0 - x, rcx = cx - x, rcy = cy - y;
                            const float la = sqrt_pos(fmaf(x, x, fmaf(y, y, z2)));
                            const float lb = sqrt_pos(fmaf(rbx, rbx, fmaf(y, y, z2)));
                            const float lc = sqrt_pos(fmaf(rcx, rcx, fmaf(rcy, rcy, z2)));
                            const float dab = fmaf(-x, rbx, fmaf(y, y, z2));
                            const float dac = fmaf(-x, rcx, fmaf(-y, rcy, z2));
                            const float dbc = fmaf(rbx, rcx, fmaf(-y, rcy, z2));
                            const float den = la * lb * lc + dab * lc + dac * lb + dbc * la;
                            const float ny = -z * A2;
                            const float e0 = __fdividef(L0, la + lb), e1 = __fdividef(L1, lb + lc),
                                        e2 = __fdividef(L2, lc + la);
                            float om, l0, l1, l2;
                            if (far_series_ok(ny, den, e0, e1, e2)) {
                                om = 2.f * atan_series(__fdividef(ny, den));
                                l0 = 2.f * atanh_series(e0);
                                l1 = 2.f * atanh_series(e1);
                                l2 = 2.f * atanh_series(e2);
                            } else {
                                om = 2.f * atan2_far(ny, den);
                                l0 = lam_f32(la, lb, L0);
                                l1 = lam_f32(lb, lc, L1);
                                l2 = lam_f32(lc, la, L2);
                            }
                            const float s11 = fmaf(rbx, e1x, -y * e1y), s21 = fmaf(rcx, e2x, rcy * e2y);
                            const float ia = __fdividef(1.f, la), ib = __fdividef(1.f, lb), ic = __fdividef(1.f, lc);
                            const float kom = Ts * mf;
                            // edge (p1 -> p2): W = L / (d1 d2 + r1.r2), q = r1 - s1 e, Z = e x r1,
                            // P = W (kom Z - kl q); p1 += (P - kl e)/d1, p2 += (P + kl e)/d2
                            auto edge = [&](float r1x, float r1y, float r2x, float r2y, float d1, float d2, float ex,
                                            float ey, float L, float s1, float kl, float i1, float i2, float& g1x,
                                            float& g1y, float& g1z, float& g2x, float& g2y, float& g2z) {
                                const float W = __fdividef(L, fmaf(d1, d2, fmaf(r1x, r2x, fmaf(r1y, r2y, z2))));
                                const float qxv = fmaf(-s1, ex, r1x), qyv = fmaf(-s1, ey, r1y), qzv = -z;
                                const float Zx = -ey * z, Zy = ex * z, Zz = fmaf(ex, r1y, -ey * r1x);  // e x r1
                                const float Px = W * fmaf(kom, Zx, -kl * qxv), Py = W * fmaf(kom, Zy, -kl * qyv),
                                            Pz = W * fmaf(kom, Zz, -kl * qzv);
                                g1x = fmaf(fmaf(-kl, ex, Px), i1, g1x);
                                g1y = fmaf(fmaf(-kl, ey, Py), i1, g1y);
                                g1z = fmaf(Pz, i1, g1z);
                                g2x = fmaf(fmaf(kl, ex, Px), i2, g2x);
                                g2y = fmaf(fmaf(kl, ey, Py), i2, g2y);
                                g2z = fmaf(Pz, i2, g2z);
                            };
                            edge(-x, -y, rbx, -y, la, lb, 1.f, 0.f, L0, -x, Ts * mt0, ia, ib, vax, vay, vaz, vbx, vby,
                                 vbz);
                            edge(rbx, -y, rcx, rcy, lb, lc, e1x, e1y, L1, s11, Ts * mt1, ib, ic, vbx, vby, vbz, vcx,
                                 vcy, vcz);
                            edge(rcx, rcy, -x, -y, lc, la, e2x, e2y, L2, s21, Ts * mt2, ic, ia, vcx, vcy, vcz, vax,
                                 vay, vaz);
                            amf = fmaf(Ts, om, amf);
                            amt0 = fmaf(Ts, l0, amt0);
                            amt1 = fmaf(Ts, l1, amt1);
                            amt2 = fmaf(Ts, l2, amt2);
                        }
                    }
                    if (++pending == kFarFlushTiles) {
                        flush();
                        pending = 0;
                    }
                }
            }
            if (pending) flush();
        }
    }
    double outv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (active && any) {
        double v[kFarTerms];
#pragma unroll
        for (int k = 0; k < kFarTerms; ++k) v[k] = __shfl_sync(0xffffffffu, tot, k);
        if (lane == 0) {
            double C[NGC];
#pragma unroll
            for (int k = 0; k < NGC; ++k) C[k] = __ldcg(&gc[(size_t)k * T + f]);
            const double nz = C[GC_ZZ], L0 = C[GC_L0], cx = C[GC_CX], cy = C[GC_CY];
            const double Ar = 0.5 * L0 * cy, q0 = v[0];
            // dA/da = (-cy, cx - L0, 0)/2, dA/db = (cy, -cx, 0)/2, dA/dc = (0, L0, 0)/2
            GradAcc A;
            grad_acc_zero(A);
            A.va = mk3(nz * (-0.5 * cy * q0 - Ar * v[1]) + v[10], nz * (0.5 * (cx - L0) * q0 - Ar * v[2]) + v[11],
                       nz * (-Ar * v[3]) + v[12]);
            A.vb = mk3(nz * (0.5 * cy * q0 - Ar * v[4]) + v[13], nz * (-0.5 * cx * q0 - Ar * v[5]) + v[14],
                       nz * (-Ar * v[6]) + v[15]);
            A.vc = mk3(nz * (-Ar * v[7]) + v[16], nz * (0.5 * L0 * q0 - Ar * v[8]) + v[17], nz * (-Ar * v[9]) + v[18]);
            A.ai = Ar * q0;
            A.amf = v[19];
            A.amt[0] = v[20]; A.amt[1] = v[21]; A.amt[2] = v[22];
            grad_finalize(C, A, groups[face_group[f]], fdir, outv);
        }
    }
    if (lane == 0)
        for (int k = 0; k < 9; ++k) part[(size_t)k * T + f] = outv[k];
}

// Per station: sum of chunk partials (facet scales are already applied).
// Blocks of 32 stations x 8 chunk lanes: lane y sums chunks y, y+8, ...
// (coalesced over stations), then the 8 lane sums are added in lane order.
// With block_nch, station s sums block_nch[s / block] chunks (the persistent
// patch forward), else nchunks.
__global__ void __launch_bounds__(256) k_forward_reduce_mixed(int S, int nchunks, const double* __restrict__ part_gz,
                                                              const double* __restrict__ part_tmi,
                                                              double* __restrict__ gz, double* __restrict__ tmi,
                                                              const int32_t* __restrict__ block_nch = nullptr,
                                                              int block = 1) {
    __shared__ double sg[8][33], st[8][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int s = blockIdx.x * 32 + tx;
    double g = 0.0, t = 0.0;
    if (block_nch && s < S) nchunks = block_nch[s / block];
    if (s < S) {
        if (part_gz) g = strided_sum8(ty, nchunks, g, [&](int c) { return part_gz[(size_t)c * S + s]; });
        if (part_tmi) t = strided_sum8(ty, nchunks, t, [&](int c) { return part_tmi[(size_t)c * S + s]; });
    }
    sg[ty][tx] = g;
    st[ty][tx] = t;
    __syncthreads();
    if (ty == 0 && s < S) {
        double G = 0.0, Tm = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            G += sg[k][tx];
            Tm += st[k][tx];
        }
        if (gz) gz[s] = G;
        if (tmi) tmi[s] = Tm;
    }
}

}  // namespace litho_b200
