// Per-facet mixed-precision forward (engine LF_FWD_FACET of lf_tuning): one
// FP32 record per facet, written once per evaluation by k_face_prep_mixed,
// streamed through shared memory 32 facets at a time; each (station, facet)
// pair evaluates its three vertex distances, three edge integrals and the
// solid angle on its own.  The patch engine (kernels_patch.cuh) shares the
// vertex distances and edge integrals across the facets of a patch instead;
// lf_autotune picks the faster engine per model.
#pragma once
#include "kernels_mixed.cuh"

namespace litho_b200 {

// FP32 facet record of the far-field forward, written once per evaluation by
// k_face_prep_mixed (array [T] in HBM), copied 32 facets at a time into
// shared memory and read there with 128-bit loads (10 per far pair, 9 per
// very far pair, 8 per mid pair).  The origin and the unit normal stay FP64: the
// height above the facet plane can be tiny next to |o - a| (a far top facet
// seen from 1 m above it).  Row 12 feeds the per-warp near/far test, row 13
// the mid field's analytic gz.
struct __align__(16) FaceF32 {
    float rx0, rx1, rx2, L0;   // local x axis, |ab|
    float ry0, ry1, ry2, cx;   // local y axis, c.x
    float cy, L1, L2, gq;      // c.y, |bc|, |ca|, n_z * gz scale * area
    float mf, mt0, mt1, mt2;   // TMI facet scales, doubled
    float q6[12];              // (x, y) of the 6-point rule's points in the local frame
    float q3[8];               // (x, y) of the 3-point rule's points, pad
    double ax, ay, az, zx, zy, zz;
    float cenx, ceny, cenz;    // centroid
    float size;                // longest edge; -1 for a facet that contributes nothing
    float l2sq, l2l0sq, cxl0;  // |ca|^2, |ca|^2 - |ab|^2, c.x - |ab|
    float g2;                  // 2 n_z * gz scale (0: no gz term)
};
static_assert(sizeof(FaceF32) == 224, "FaceF32 layout");
constexpr int kFaceF32Vec = sizeof(FaceF32) / 16;  // float4 per record

// The far-field record of one facet from its mixed constants m[NMC].
__device__ __forceinline__ void make_face_f32(const double* m, FaceF32& F) {
#define M(k) m[k]
    F.rx0 = (float)M(MC_XX); F.rx1 = (float)M(MC_XY); F.rx2 = (float)M(MC_XZ);
    F.ry0 = (float)M(MC_YX); F.ry1 = (float)M(MC_YY); F.ry2 = (float)M(MC_YZ);
    F.L0 = (float)M(MC_L0); F.cx = (float)M(MC_CX); F.cy = (float)M(MC_CY);
    F.L1 = (float)M(MC_L1); F.L2 = (float)M(MC_L2);
    F.gq = (float)(M(MC_SGZ) * 0.5 * M(MC_L0) * M(MC_CY));
    // TMI scales doubled: the far pair's series give atan2 and atanh (exact)
    F.mf = 2.f * (float)M(MC_MF); F.mt0 = 2.f * (float)M(MC_MT0);
    F.mt1 = 2.f * (float)M(MC_MT1); F.mt2 = 2.f * (float)M(MC_MT2);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        F.q6[2 * q] = kDun6Bb[q] * F.L0 + kDun6Bc[q] * F.cx;
        F.q6[2 * q + 1] = kDun6Bc[q] * F.cy;
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        F.q3[2 * q] = kTri3Bb[q] * F.L0 + kTri3Bc[q] * F.cx;
        F.q3[2 * q + 1] = kTri3Bc[q] * F.cy;
    }
    F.q3[6] = F.q3[7] = 0.f;
    F.ax = M(MC_AX); F.ay = M(MC_AY); F.az = M(MC_AZ);
    F.zx = M(MC_ZX); F.zy = M(MC_ZY); F.zz = M(MC_ZZ);
    F.cenx = (float)M(MC_CENX); F.ceny = (float)M(MC_CENY); F.cenz = (float)M(MC_CENZ);
    F.size = M(MC_VALID) != 0.0 ? (float)M(MC_SIZE) : -1.f;
    F.l2sq = (float)(M(MC_L2) * M(MC_L2));
    F.l2l0sq = (float)(M(MC_L2) * M(MC_L2) - M(MC_L0) * M(MC_L0));
    F.cxl0 = (float)(M(MC_CX) - M(MC_L0));
    F.g2 = (float)(2.0 * M(MC_SGZ));
#undef M
}

__global__ void k_face_prep_mixed(int T, const int32_t* __restrict__ tri, const double* __restrict__ pos,
                                  const int16_t* __restrict__ face_group, const GroupConst* __restrict__ groups, d3 fdir,
                                  double* __restrict__ mc, FaceF32* __restrict__ mf32, int drop_collapsed) {
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
    if (!(area2 < kEps) && !(drop_collapsed && facet_collapsed(v, area2))) {
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
    FaceF32 F;
    make_face_f32(out, F);
    const float4* src = reinterpret_cast<const float4*>(&F);
    float4* dst = reinterpret_cast<float4*>(mf32 + f);
#pragma unroll
    for (int k = 0; k < kFaceF32Vec; ++k) dst[k] = src[k];
}


enum { RULE_TRI3 = 0, RULE_DUN6 = 1, RULE_MID = 2 };

// atanh(v) / v - 1 = v^2/3 + v^4/5 + ... for 0 <= v <= 0.2 (Abramowitz &
// Stegun 4.1.28 through v^8; the first omitted term, v^10/11, is below 1e-8,
// so below 1e-8 of atanh(v) / v).
__device__ __forceinline__ float atanh_q(float v) {
    const float v2 = v * v;
    return v2 * fmaf(v2, fmaf(v2, fmaf(v2, 1.f / 9.f, 1.f / 7.f), 1.f / 5.f), 1.f / 3.f);
}

// (atanh(v) / v - 1) / v^2 = 1/3 + v^2/5 + ... + v^8/11, in v2 = v^2.
__device__ __forceinline__ float atanh_q11(float v2) {
    return fmaf(v2, fmaf(v2, fmaf(v2, fmaf(v2, 1.f / 11.f, 1.f / 9.f), 1.f / 7.f), 1.f / 5.f), 1.f / 3.f);
}

// Q(e) = atanh(e) / e - 1 for 0 < e < 1, without the cancellation of
// "atanh(e) / e - 1" in FP32.  With c = sqrt(1 - e^2) and w = e / (1 + c) =
// tanh(atanh(e) / 2) (the half-argument formula),
//   atanh(e) / e = 2 atanh(w) / e = (2 / (1 + c)) (1 + Q(w)),
// and, as 1 - c = e^2 / (1 + c),  Q(e) = w^2 + (2 / (1 + c)) Q(w): every term
// is positive.  Each step halves atanh(e); atanh_q takes over at 0.2, which
// four steps reach for e below 0.997 -- closer to 1 the log form has no
// cancellation left to fear.
__device__ __forceinline__ float atanh_q_any(float e) {
    if (!(e > 0.2f)) return atanh_q(e);
    float q = 0.f, m = 1.f, v = e;
#pragma unroll 1
    for (int it = 0; it < 4 && v > 0.2f && v < 1.f; ++it) {
        const float r = __fdividef(1.f, 1.f + sqrt_pos((1.f - v) * (1.f + v)));
        v *= r;
        q = fmaf(m, v * v, q);
        m *= 2.f * r;
    }
    if (v <= 0.2f) return fmaf(m, atanh_q(v), q);
    return __fdividef(0.5f * log1pf(__fdividef(2.f * e, 1.f - e)), e) - 1.f;
}

// Far pair, both FP32, o = station (FP64): TMI analytic; gz by quadrature
// (RULE_TRI3 beyond 4 tau, RULE_DUN6 beyond tau) or analytically (RULE_MID,
// the mid field tau/2 <= distance / size < tau).  SHORT (tau >= 3, so very
// far pairs lie beyond 12 x size and far ones beyond 3 x size): series of the
// length those distances need, and no range test.
//
// The mid field's gz: the integral of 1/r over the facet is
//   I = sum_i u_i Lambda_i + z Omega
// (u_i: distance from the station's projection to edge i's line, positive
// inside; Gauss-Green in the facet plane, the same identity as the FP64
// pair's gz).  In FP32 the sum cancels by about distance / size, so it is
// regrouped around sbar = (s0 + s1 + s2) / 3, s_i = the sum of edge i's two
// vertex distances, using sum_i u_i L_i = 2A:
//   I / 2 = 2A / sbar + sum_i (u_i L_i / s_i) (Q_i + (sbar - s_i) / sbar),
// Q_i = atanh(e_i) / e_i - 1, e_i = L_i / s_i; sbar - s_i comes from the
// distance differences l_c - l_a = (l_c^2 - l_a^2) / (l_c + l_a), whose
// numerators are linear in the station.  Every term is then of the size of
// I itself.
template <int RULE, bool SHORT = false>
__device__ __forceinline__ void pair_far_f32(const FaceF32* Fp, double ox, double oy, double oz, float* gz,
                                             float* tmi) {
    const float4* v = reinterpret_cast<const float4*>(Fp);
    const double2* w = reinterpret_cast<const double2*>(Fp);
    const float4 v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3];
    const double2 w0 = w[9], w1 = w[10], w2 = w[11];
    const double ddx = ox - w0.x, ddy = oy - w0.y, ddz = oz - w1.x;
    const float dx = (float)ddx, dy = (float)ddy, dz = (float)ddz;
    const float x = fmaf(dx, v0.x, fmaf(dy, v0.y, dz * v0.z));
    const float y = fmaf(dx, v1.x, fmaf(dy, v1.y, dz * v1.z));
    const float z = (float)(ddx * w1.y + ddy * w2.x + ddz * w2.y);
    const float L0 = v0.w, cx = v1.w, cy = v2.x, L1 = v2.y, L2 = v2.z, gq = v2.w;
    const float z2 = z * z;
    // gz: n_z * gscale * A * sum_q w_q / r_q.  A facet with a horizontal unit
    // normal (n_z == 0 exactly: every vertical face of a voxel-built surface,
    // which z-only vertex moves keep vertical) has gq == 0 and adds exactly
    // zero, as in the reference's n_z * (...) product; its quadrature is
    // skipped.  The facet is the same for every lane, so the branch is
    // warp-uniform.
    if (RULE != RULE_MID) {
        float acc = 0.f;
        if (gq == 0.f) {
        } else if (RULE == RULE_DUN6) {
            const float4 qa = v[4], qb = v[5], qc = v[6];
            const float q[12] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w, qc.x, qc.y, qc.z, qc.w};
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                float px = q[2 * k] - x, py = q[2 * k + 1] - y;
                acc = fmaf(kDun6W[k], rsqrtf(fmaf(px, px, fmaf(py, py, z2))), acc);
            }
        } else {
            const float4 qa = v[7], qb = v[8];
            const float q[6] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float px = q[2 * k] - x, py = q[2 * k + 1] - y;
                acc += rsqrtf(fmaf(px, px, fmaf(py, py, z2)));
            }
            acc *= (1.f / 3.f);
        }
        if (gq != 0.f) *gz += gq * acc;
    }
    // TMI: MF * Omega + sum_i MT_i Lambda_i with Omega = 2 atan2(ny, den) and
    // Lambda_i = 2 atanh(e_i); the record holds 2 MF and 2 MT_i, so the terms
    // below are atan2 and atanh.  Scaling by 2 is exact: the bits equal
    // MF * (2 atan2) + MT_i * (2 atanh).
    float rbx = L0 - x, rcx = cx - x, rcy = cy - y;
    float la = sqrt_pos(fmaf(x, x, fmaf(y, y, z2)));
    float lb = sqrt_pos(fmaf(rbx, rbx, fmaf(y, y, z2)));
    float lc = sqrt_pos(fmaf(rcx, rcx, fmaf(rcy, rcy, z2)));
    float dab = fmaf(-x, rbx, fmaf(y, y, z2));
    float dac = fmaf(-x, rcx, fmaf(-y, rcy, z2));
    float dbc = fmaf(rbx, rcx, fmaf(-y, rcy, z2));
    float den = la * lb * lc + dab * lc + dac * lb + dbc * la;
    const float l0cy = L0 * cy;
    const float ny = -z * l0cy;
    float om, l0, l1, l2;
    if (RULE == RULE_MID) {
        const float s0 = la + lb;
        const float r0 = __fdividef(1.f, s0), r1 = __fdividef(1.f, lb + lc), r2 = __fdividef(1.f, lc + la);
        const float e0 = L0 * r0, e1 = L1 * r1, e2 = L2 * r2;
        float q0, q1, q2;
        if (far_series_ok(ny, den, e0, e1, e2)) {
            om = atan_series(__fdividef(ny, den));
            q0 = atanh_q(e0);
            q1 = atanh_q(e1);
            q2 = atanh_q(e2);
        } else {
            om = atan2_far(ny, den);
            q0 = atanh_q_any(e0);
            q1 = atanh_q_any(e1);
            q2 = atanh_q_any(e2);
        }
        l0 = fmaf(e0, q0, e0);
        l1 = fmaf(e1, q1, e1);
        l2 = fmaf(e2, q2, e2);
        const float4 v13 = v[13];  // |ca|^2, |ca|^2 - |ab|^2, c.x - |ab|, 2 n_z gscale
        if (v13.w != 0.f) {
            const float k = __fdividef(0.5f, s0 + lc);  // 1 / (3 sbar)
            const float tx = x + x, ty = y + y;
            const float dba = L0 * (L0 - tx) * r0;                          // l_b - l_a
            const float dca = fmaf(-cx, tx, fmaf(-cy, ty, v13.x)) * r2;     // l_c - l_a
            const float dcb = fmaf(-v13.z, tx, fmaf(-cy, ty, v13.y)) * r1;  // l_c - l_b
            // u_i L_i / s_i for the edges ab (u = y), bc and ca
            const float w0 = y * L0 * r0, w1 = fmaf(rbx, cy, y * v13.z) * r1, w2 = fmaf(x, cy, -y * cx) * r2;
            float h = w0 * (q0 + (dca + dcb) * k);
            h = fmaf(w1, q1 - (dba + dca) * k, h);
            h = fmaf(w2, q2 + (dba - dcb) * k, h);
            h = fmaf(3.f * l0cy, k, h);  // 2A / sbar
            h = fmaf(z, om, h);          // I / 2
            *gz += v13.w * h;
        }
    } else {
        const float e0 = __fdividef(L0, la + lb), e1 = __fdividef(L1, lb + lc), e2 = __fdividef(L2, lc + la);
        if (SHORT && RULE == RULE_TRI3) {
            // Beyond 12 x size every vertex lies beyond 11.3 x size (a vertex
            // is within 2/3 of a median, so within size, of the centroid):
            // e_i < 0.045 (the series through e^5 leaves 1e-9 of the sum) and
            // the solid angle, below area / distance^2, under 0.0035 (|t| <
            // 0.002: through t^3 leaves 1e-12); den > 0 and the range test
            // holds there.
            const float t = __fdividef(ny, den);
            om = t * fmaf(t * t, -1.f / 3.f, 1.f);
            l0 = e0 * fmaf(e0 * e0, fmaf(e0 * e0, 0.2f, 1.f / 3.f), 1.f);
            l1 = e1 * fmaf(e1 * e1, fmaf(e1 * e1, 0.2f, 1.f / 3.f), 1.f);
            l2 = e2 * fmaf(e2 * e2, fmaf(e2 * e2, 0.2f, 1.f / 3.f), 1.f);
        } else if (SHORT) {
            // Beyond 3 x size every vertex lies beyond 2.33 x size: e_i < 0.215
            // (one term more than atanh_series, through e^11, leaves 8e-10)
            // and |t| < 0.04 (through t^5 leaves 6e-10); the vertices' view
            // angles stay below 25 degrees, so den > 0.
            const float t = __fdividef(ny, den), t2 = t * t;
            om = t * fmaf(t2, fmaf(t2, 0.2f, -1.f / 3.f), 1.f);
            l0 = e0 * fmaf(e0 * e0, atanh_q11(e0 * e0), 1.f);
            l1 = e1 * fmaf(e1 * e1, atanh_q11(e1 * e1), 1.f);
            l2 = e2 * fmaf(e2 * e2, atanh_q11(e2 * e2), 1.f);
        } else if (far_series_ok(ny, den, e0, e1, e2)) {
            om = atan_series(__fdividef(ny, den));
            l0 = atanh_series(e0);
            l1 = atanh_series(e1);
            l2 = atanh_series(e2);
        } else {
            om = atan2_far(ny, den);
            l0 = 0.5f * lam_f32(la, lb, L0);
            l1 = 0.5f * lam_f32(lb, lc, L1);
            l2 = 0.5f * lam_f32(lc, la, L2);
        }
    }
    *tmi += v3.x * om + v3.y * l0 + v3.z * l1 + v3.w * l2;
}


// Station-per-thread forward: CTAs of 128 stations (pre-ordered along a
// Morton curve, so a warp's 32 stations are spatially compact) x facet
// chunks, facets staged 32 at a time in shared memory (their FP32 records,
// written by k_face_prep_mixed, copied by the whole CTA; the FP64 constants
// of a near facet fetched into the warp's own slot when it meets one,
// which is a few per cent of pairs).  The precision class
// is decided per (warp, facet): lane j tests facet j of the stage against the
// warp's station bounding box -- centroid at least 4 tau x size away: very
// far (FP32, 3-point gz); at least tau x size: far (FP32, 6-point gz); at
// least tau/2 x size: mid (FP32, analytic gz); else near (FP64 analytic) --
// and the warp walks each class warp-uniformly.
// One CTA's work: station s (this thread; act = s is a station of the
// block) against facets [fb, fe); out_gz[s] / out_tmi[s] receive the sums.
template <bool GZ, bool TMI, int FT>
__device__ __forceinline__ void forward_mixed_block(FaceF32* __restrict__ smf, double* __restrict__ smn, int s,
                                                    bool act, const double* __restrict__ sta, int T,
                                                    const double* __restrict__ mc, const FaceF32* __restrict__ mf32,
                                                    int fb, int fe, float tau,
                                                    double* __restrict__ out_gz, double* __restrict__ out_tmi,
                                                    unsigned long long* __restrict__ near_pairs) {
    static_assert(FT % 32 == 0, "one facet per lane in each 32-facet half of the near/far test");
    const int lane = threadIdx.x & 31;
    double ox = 0.0, oy = 0.0, oz = 0.0;
    if (act) { ox = sta[3 * s]; oy = sta[3 * s + 1]; oz = sta[3 * s + 2]; }
    // the warp's station bounding box: lo = min, hi = -min(-x)
    float bb[6] = {act ? (float)ox : 3e38f, act ? (float)oy : 3e38f, act ? (float)oz : 3e38f,
                   act ? -(float)ox : 3e38f, act ? -(float)oy : 3e38f, act ? -(float)oz : 3e38f};
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) bb[k] = fminf(bb[k], __shfl_xor_sync(0xffffffffu, bb[k], off));
    double gz = 0.0, tmi = 0.0;
    unsigned long long nearCount = 0;
    for (int f0 = fb; f0 < fe; f0 += FT) {
        const int nf = min(FT, fe - f0);
        __syncthreads();  // the previous stage's records are no longer read
        {
            const float4* __restrict__ src = reinterpret_cast<const float4*>(mf32 + f0);
            float4* dst = reinterpret_cast<float4*>(smf);
            for (int idx = threadIdx.x; idx < nf * kFaceF32Vec; idx += blockDim.x) dst[idx] = __ldg(src + idx);
        }
        __syncthreads();
        for (int h0 = 0; h0 < nf; h0 += 32) {
            const FaceF32* __restrict__ sh = smf + h0;
            // lane j: facet h0 + j of the stage against this warp's box
            bool valid = false, vfar = false, far = false, mid = false;
            if (h0 + lane < nf && !(sh[lane].size < 0.f)) {
                valid = true;
                const float cxw = sh[lane].cenx, cyw = sh[lane].ceny, czw = sh[lane].cenz;
                const float ddx = fmaxf(0.f, fmaxf(bb[0] - cxw, cxw + bb[3]));
                const float ddy = fmaxf(0.f, fmaxf(bb[1] - cyw, cyw + bb[4]));
                const float ddz = fmaxf(0.f, fmaxf(bb[2] - czw, czw + bb[5]));
                const float d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                const float lim = tau * sh[lane].size, limMid = 0.5f * lim;
                vfar = d2 >= 16.f * (lim * lim);
                far = !vfar && d2 >= lim * lim;
                mid = !vfar && !far && d2 >= limMid * limMid;
            }
            const unsigned vfarMask = __ballot_sync(0xffffffffu, valid && vfar);
            const unsigned farMask = __ballot_sync(0xffffffffu, valid && far);
            const unsigned midMask = __ballot_sync(0xffffffffu, valid && mid);
            const unsigned nearMask = __ballot_sync(0xffffffffu, valid && !vfar && !far && !mid);
            if (act) {
                float gacc = 0.f, tacc = 0.f;
                if (tau >= 3.f) {
                    for (unsigned m = vfarMask; m; m &= m - 1) {
                        const int j = __ffs(m) - 1;
                        pair_far_f32<RULE_TRI3, true>(&sh[j], ox, oy, oz, &gacc, &tacc);
                    }
                    for (unsigned m = farMask; m; m &= m - 1) {
                        const int j = __ffs(m) - 1;
                        pair_far_f32<RULE_DUN6, true>(&sh[j], ox, oy, oz, &gacc, &tacc);
                    }
                } else {
                    for (unsigned m = vfarMask; m; m &= m - 1) {
                        const int j = __ffs(m) - 1;
                        pair_far_f32<RULE_TRI3>(&sh[j], ox, oy, oz, &gacc, &tacc);
                    }
                    for (unsigned m = farMask; m; m &= m - 1) {
                        const int j = __ffs(m) - 1;
                        pair_far_f32<RULE_DUN6>(&sh[j], ox, oy, oz, &gacc, &tacc);
                    }
                }
                for (unsigned m = midMask; m; m &= m - 1) {
                    const int j = __ffs(m) - 1;
                    pair_far_f32<RULE_MID>(&sh[j], ox, oy, oz, &gacc, &tacc);
                }
                if (GZ) gz += gacc;
                if (TMI) tmi += tacc;
                nearCount += __popc(nearMask);
            }
            // Near facets (a few per cent of pairs): the warp copies the
            // facet's FP64 constants from HBM into its own slot of shared
            // memory (lane k loads constant k), then every lane reads them.
            double* slot = smn + (threadIdx.x >> 5) * NMC;
            for (unsigned m = nearMask; m; m &= m - 1) {
                const int j = __ffs(m) - 1;
                __syncwarp();
                if (lane < NMC) slot[lane] = __ldg(mc + (size_t)lane * T + f0 + h0 + j);
                __syncwarp();
                if (act) {
                    double g1 = 0.0, t1 = 0.0;
                    pair_near_f64(slot, 0, 1, mk3(ox, oy, oz), &g1, &t1);
                    if (GZ) gz += g1;
                    if (TMI) tmi += t1;
                }
            }
        }
    }
    if (act) {
        if (GZ) out_gz[s] = gz;
        if (TMI) out_tmi[s] = tmi;
        if (near_pairs && nearCount) atomicAdd(near_pairs, nearCount);
    }
}

template <bool GZ, bool TMI, int FT>
__global__ void __launch_bounds__(128) k_forward_mixed(int S, const double* __restrict__ sta, int T,
                                                       const double* __restrict__ mc,
                                                       const FaceF32* __restrict__ mf32,
                                                       const int32_t* __restrict__ chunk_begin,
                                                       const int32_t* __restrict__ chunk_end, float tau,
                                                       double* __restrict__ part_gz, double* __restrict__ part_tmi,
                                                       unsigned long long* __restrict__ near_pairs) {
    __shared__ FaceF32 smf[FT];
    __shared__ double smn[4 * NMC];  // one near-facet slot per warp (128 threads)
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int chunk = blockIdx.y;
    forward_mixed_block<GZ, TMI, FT>(smf, smn, s, s < S, sta, T, mc, mf32, chunk_begin[chunk], chunk_end[chunk], tau,
                                     GZ ? part_gz + (size_t)chunk * S : nullptr,
                                     TMI ? part_tmi + (size_t)chunk * S : nullptr, near_pairs);
}

// Batched bodies (item list as for k_forward_fp64_items).
template <bool GZ, bool TMI, int FT>
__global__ void __launch_bounds__(128) k_forward_mixed_items(const FwdItem* __restrict__ items, int nitems,
                                                             const double* __restrict__ sta, int T,
                                                             const double* __restrict__ mc,
                                                             const FaceF32* __restrict__ mf32, float tau,
                                                             double* __restrict__ part_gz, double* __restrict__ part_tmi,
                                                             unsigned long long* __restrict__ near_pairs) {
    __shared__ FaceF32 smf[FT];
    __shared__ double smn[4 * NMC];  // one near-facet slot per warp (128 threads)
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const FwdItem w = items[it];
        const int s = w.s0 + (int)threadIdx.x;
        forward_mixed_block<GZ, TMI, FT>(smf, smn, s, s < w.s_end, sta, T, mc, mf32, w.fb, w.fe, tau,
                                         GZ ? part_gz + w.out : nullptr, TMI ? part_tmi + w.out : nullptr,
                                         near_pairs);
    }
}


}  // namespace litho_b200
