// FP64 device kernels of the LithoInv hot path (sm_100a).
//
// Forward (station-per-thread, facets staged in shared memory): the per-pair
// arithmetic follows faceNagyContribution / magneticFacet / solidAngle /
// lineIntegralTerm of the reference in the same operation order
// (modules/litho-forward/src/forward/gravity_forward.cpp:13-42,
//  modules/litho-forward/src/forward/magnetic_forward.cpp:312-347,
//  modules/litho-core/src/core/geometry.cpp:10-52); the station-independent
// facet quantities (unit normal, edge vectors, lengths, in-plane edge normals,
// magnetic direction products) are computed once per facet by face_prep_fwd.
//
// Gradient (facet-per-thread, stations staged in shared memory): the
// derivative of every facet term with respect to its three vertices, in
// closed form, contracted with the per-station weighted residual in the same
// pass so the Jacobian is never stored.  Derivation (per facet, local frame
// with origin at vertex a, x along a->b, z along the unit normal):
//   d Lambda_e / d p2 = ( e_hat - q W ) / d2,   d Lambda_e / d p1 = (-e_hat - q W) / d1,
//   d Omega / d p1 += (e_hat x r1) W / d1,      d Omega / d p2 += (e_hat x r1) W / d2,
// with r1 = p1 - o, q = r1 - (r1.e_hat) e_hat, W = L / (d1 d2 + r1.r2); the
// station-independent factors (n_z, n_hat, in-plane edge normals, magnetic
// direction products) are differentiated once per facet from accumulated
// station sums.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace litho_b200 {

constexpr double kEps = 1e-15;
constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------- layouts --
// Forward facet constants, SoA [NFC][T].
enum FwdConst {
    FC_AX = 0, FC_AY, FC_AZ, FC_BX, FC_BY, FC_BZ, FC_CX, FC_CY, FC_CZ,
    FC_NX, FC_NY, FC_NZ,
    FC_E0X, FC_E0Y, FC_E0Z, FC_E1X, FC_E1Y, FC_E1Z, FC_E2X, FC_E2Y, FC_E2Z,
    FC_L0, FC_L1, FC_L2,
    FC_P0X, FC_P0Y, FC_P0Z, FC_P1X, FC_P1Y, FC_P1Z, FC_P2X, FC_P2Y, FC_P2Z,
    FC_MF, FC_MT0, FC_MT1, FC_MT2,
    FC_VALID,
    NFC
};

// Gradient facet constants (local frame), SoA [NGC][T].
enum GradConst {
    GC_AX = 0, GC_AY, GC_AZ,           // origin (vertex a)
    GC_XX, GC_XY, GC_XZ,               // local x axis (global components)
    GC_YX, GC_YY, GC_YZ,               // local y axis
    GC_ZX, GC_ZY, GC_ZZ,               // local z axis = unit normal
    GC_L0, GC_CX, GC_CY,               // b = (L0, 0, 0), c = (CX, CY, 0)
    GC_E1X, GC_E1Y, GC_L1,             // edge b->c direction and length
    GC_E2X, GC_E2Y, GC_L2,             // edge c->a direction and length
    GC_GS,                             // gz scale of the facet's group (0: no gravity)
    GC_MS,                             // TMI scale of the facet's group (0: skipped)
    GC_MF, GC_MT0, GC_MT1, GC_MT2,     // magnetic direction products
    GC_FLAGS,                          // bit0 valid facet, bit1 needs gradient
    NGC
};

struct GroupConst {
    double gscale_fwd;  // G * rho * 1e3 * 1e5 (forward association)
    double gscale_jac;  // (G * 1e3 * 1e5) * rho (Jacobian association)
    double mscale;      // magnetization amplitude * 100 / (4 pi)
    double mdir[3];
    int mag_active;     // amplitude >= 1e-15 (the Jacobian skips weaker groups)
};

// ------------------------------------------------------------- utilities --
struct d3 { double x, y, z; };
__device__ __forceinline__ d3 mk3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator*(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross3(d3 a, d3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double norm3(d3 a) { return sqrt(dot3(a, a)); }

// lineIntegralTerm branch semantics (geometry.cpp:39-51) given s1, s2, d1, d2.
__device__ __forceinline__ double lambda_from(double s1, double s2, double d1, double d2, bool* live) {
    double num = s2 + d2, den = s1 + d1;
    *live = false;
    if (fabs(den) < kEps) return 0.0;  // covers the "both ~0" branch too
    if (num <= 0.0 || den <= 0.0) return 0.0;
    *live = true;
    return log(num / den);
}

// Lambda in the symmetric form log((d1 + d2 + L) / (d1 + d2 - L)) =
// log1p(2 L / (d1 + d2 - L)), equal to lineIntegralTerm's oriented
// log((s2 + d2) / (s1 + d1)) (d2^2 - d1^2 = s2^2 - s1^2 along the edge's
// line) wherever that is live.  The local-frame FP64 kernels (mixed near
// pairs, the analytic derivatives) use it: it depends only on distances,
// so the rounding of the frame change cannot flip a branch.  Where the
// reference's branch returns 0 although the station lies off the segment
// -- exactly on the edge's line, beyond its end point, which synthetic
// station grids can hit when they share the voxel lattice (s1 + d1 is then
// an exact 0 in the reference's global coordinates) -- this is the
// continuous value log(d1 / d2) instead: the reference's forward is
// discontinuous there and its own finite-difference Jacobian undefined.
// The FP64 forward keeps lambda_from, bit for bit.  live = the station is
// not on the segment itself (d1 + d2 > L).
__device__ __forceinline__ double lambda_sym(double d1, double d2, double L, bool* live) {
    const double dsum = d1 + d2, den = dsum - L;
    *live = den > 1e-13 * dsum;
    return *live ? log1p(2.0 * L / den) : 0.0;
}

// ------------------------------------------------------------- scatter ----
// LithologyModel::applyParameterVector (lithology_model.cpp:210-248) step 1:
// every global DOF writes the (vertex, axis) slots it controls.
__global__ void k_scatter_dofs(int np, const double* __restrict__ params, const int32_t* __restrict__ dof_off,
                               const int32_t* __restrict__ ref_vertex, const uint8_t* __restrict__ ref_axis,
                               const double* __restrict__ ref_scale, double* __restrict__ pos) {
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= np) return;
    double val = params[d];
    for (int r = dof_off[d]; r < dof_off[d + 1]; ++r)
        pos[3 * ref_vertex[r] + ref_axis[r]] = __dmul_rn(val, ref_scale[r]);
}

// Step 2: interpolateFromControlPoints (surface_mesh.cpp:610-623); rows only
// read control-point vertices, which are never rows themselves.
__global__ void k_interpolate(int nrows, const int32_t* __restrict__ rows, const int32_t* __restrict__ interp_off,
                              const int32_t* __restrict__ interp_src, const double* __restrict__ interp_w,
                              double* __restrict__ pos) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    int v = rows[i];
    double px = 0.0, py = 0.0, pz = 0.0;
    for (int k = interp_off[v]; k < interp_off[v + 1]; ++k) {
        const double* q = pos + 3 * interp_src[k];
        double w = interp_w[k];
        px = __dadd_rn(px, __dmul_rn(q[0], w));
        py = __dadd_rn(py, __dmul_rn(q[1], w));
        pz = __dadd_rn(pz, __dmul_rn(q[2], w));
    }
    pos[3 * v] = px;
    pos[3 * v + 1] = py;
    pos[3 * v + 2] = pz;
}

// Step 3: shared-vertex averaging groups (lithology_model.cpp:235-247).
__global__ void k_sync_shared(int ns, const int32_t* __restrict__ sync_off, const int32_t* __restrict__ sync_vertex,
                              double* __restrict__ pos) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    int b = sync_off[s], e = sync_off[s + 1];
    if (e - b < 2) return;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int k = b; k < e; ++k) {
        const double* q = pos + 3 * sync_vertex[k];
        ax = __dadd_rn(ax, q[0]);
        ay = __dadd_rn(ay, q[1]);
        az = __dadd_rn(az, q[2]);
    }
    double n = static_cast<double>(e - b);
    ax = __ddiv_rn(ax, n); ay = __ddiv_rn(ay, n); az = __ddiv_rn(az, n);
    for (int k = b; k < e; ++k) {
        double* q = pos + 3 * sync_vertex[k];
        q[0] = ax; q[1] = ay; q[2] = az;
    }
}

// ------------------------------------------------------- facet constants --
// Exact-order helpers: no FMA contraction, the reference's left-to-right
// evaluation.  Facets collapsed by the control-point interpolation have a
// twice-area of ~1e-12 (above the reference's 1e-15 cutoff), so their unit
// normal is pure rounding; the TMI facet term does not vanish with the area,
// so it is reproduced only when the normal is rounded exactly as on the CPU.
__device__ __forceinline__ d3 sub_rn(d3 a, d3 b) { return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)}; }
__device__ __forceinline__ double dot_rn(d3 a, d3 b) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z));
}
__device__ __forceinline__ d3 cross_rn(d3 a, d3 b) {
    return {__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
            __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x))};
}
__device__ __forceinline__ double norm_rn(d3 a) { return __dsqrt_rn(dot_rn(a, a)); }
__device__ __forceinline__ d3 div_rn(d3 a, double s) { return {__ddiv_rn(a.x, s), __ddiv_rn(a.y, s), __ddiv_rn(a.z, s)}; }

// A facet collapsed onto a line: twice-area below 1e-10 x its longest edge
// squared (control-point interpolation produces them).  Its unit normal is
// rounding noise, and the reference's TMI facet term, which does not vanish
// with the area (magnetic_forward.cpp:312-347), is then a discontinuous
// function of the positions.  The derivative kernels always take such facets
// as contributing zero; the forward does too when the context drops them
// (lf_set_collapsed_facets), so that the objective is the function its
// gradient differentiates.  No reference counterpart.
__device__ __forceinline__ bool facet_collapsed(const d3 (&v)[3], double area2) {
    const double l0 = norm_rn(sub_rn(v[1], v[0])), l1 = norm_rn(sub_rn(v[2], v[1])), l2 = norm_rn(sub_rn(v[0], v[2]));
    const double lm = fmax(l0, fmax(l1, l2));
    return area2 < 1e-10 * lm * lm;
}

// Forward constants of one facet (vertices v) in the reference's operation
// order; out[NFC].  drop: collapsed facets contribute nothing.
__device__ __forceinline__ void face_consts_fwd(const d3 (&v)[3], const GroupConst& g, d3 fdir, double (&out)[NFC],
                                                bool drop = false) {
    // faceNagyContribution / magneticFacet: n = (b-a) x (c-a), unit_n = n / |n|
    d3 n = cross_rn(sub_rn(v[1], v[0]), sub_rn(v[2], v[0]));
    double area2 = norm_rn(n);
    bool valid = !(area2 < kEps) && !(drop && facet_collapsed(v, area2));
    d3 un = valid ? div_rn(n, area2) : mk3(0, 0, 0);
    d3 m = mk3(g.mdir[0], g.mdir[1], g.mdir[2]);
    out[FC_AX] = v[0].x; out[FC_AY] = v[0].y; out[FC_AZ] = v[0].z;
    out[FC_BX] = v[1].x; out[FC_BY] = v[1].y; out[FC_BZ] = v[1].z;
    out[FC_CX] = v[2].x; out[FC_CY] = v[2].y; out[FC_CZ] = v[2].z;
    out[FC_NX] = un.x; out[FC_NY] = un.y; out[FC_NZ] = un.z;
    out[FC_MF] = __dmul_rn(dot_rn(m, un), dot_rn(fdir, un));  // mn * fn
    for (int i = 0; i < 3; ++i) {
        d3 e = sub_rn(v[(i + 1) % 3], v[i]);
        double L = norm_rn(e);
        d3 eh = (L < kEps) ? mk3(0, 0, 0) : div_rn(e, L);
        d3 perp = cross_rn(un, eh);
        out[FC_E0X + 3 * i] = e.x; out[FC_E0Y + 3 * i] = e.y; out[FC_E0Z + 3 * i] = e.z;
        out[FC_L0 + i] = L;
        out[FC_P0X + 3 * i] = perp.x; out[FC_P0Y + 3 * i] = perp.y; out[FC_P0Z + 3 * i] = perp.z;
        out[FC_MT0 + i] = __dmul_rn(dot_rn(m, perp), dot_rn(fdir, perp));  // mt * ft
    }
    out[FC_VALID] = valid ? 1.0 : 0.0;
}

__global__ void k_face_prep_fwd(int T, const int32_t* __restrict__ tri, const double* __restrict__ pos,
                                const int16_t* __restrict__ face_group, const GroupConst* __restrict__ groups,
                                d3 fdir, double* __restrict__ fc, int drop_collapsed) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= T) return;
    const double* pa = pos + 3 * tri[3 * f];
    const double* pb = pos + 3 * tri[3 * f + 1];
    const double* pc = pos + 3 * tri[3 * f + 2];
    d3 v[3] = {mk3(pa[0], pa[1], pa[2]), mk3(pb[0], pb[1], pb[2]), mk3(pc[0], pc[1], pc[2])};
    double out[NFC];
    face_consts_fwd(v, groups[face_group[f]], fdir, out, drop_collapsed != 0);
    for (int k = 0; k < NFC; ++k) fc[(size_t)k * T + f] = out[k];
}

// Finite-difference-XY gradient mode (no reference counterpart; the
// reference differentiates every axis by per-facet forward differences with
// h = 1e-4 m, faceNagyWithGradient gravity_forward.cpp:48-85): forward
// constants of each listed facet and of its six copies with one vertex moved
// by +h in x or y, variant k = 1 + 2 * corner + axis.  Layout
// [7][NFC][nf] over the list index.
__global__ void k_face_prep_fdxy(int nf, const int32_t* __restrict__ facets, const int32_t* __restrict__ tri,
                                 const double* __restrict__ pos, const int16_t* __restrict__ face_group,
                                 const GroupConst* __restrict__ groups, d3 fdir, double h, double* __restrict__ fcfd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;  // variant
    if (i >= nf) return;
    const int f = facets[i];
    d3 v[3];
    for (int c = 0; c < 3; ++c) {
        const double* p = pos + 3 * tri[3 * f + c];
        v[c] = mk3(p[0], p[1], p[2]);
    }
    if (k > 0) {
        const int c = (k - 1) >> 1;
        if ((k - 1) & 1) v[c].y = __dadd_rn(v[c].y, h);
        else v[c].x = __dadd_rn(v[c].x, h);
    }
    double out[NFC];
    face_consts_fwd(v, groups[face_group[f]], fdir, out);
    for (int q = 0; q < NFC; ++q) fcfd[((size_t)k * NFC + q) * nf + i] = out[q];
}

__global__ void k_face_prep_grad(int T, const int32_t* __restrict__ tri, const double* __restrict__ pos,
                                 const int16_t* __restrict__ face_group, const GroupConst* __restrict__ groups,
                                 const uint8_t* __restrict__ face_needs, int want_grav, int want_mag, d3 fdir,
                                 double* __restrict__ gc) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= T) return;
    const double* pa = pos + 3 * tri[3 * f];
    const double* pb = pos + 3 * tri[3 * f + 1];
    const double* pc = pos + 3 * tri[3 * f + 2];
    d3 a = mk3(pa[0], pa[1], pa[2]), b = mk3(pb[0], pb[1], pb[2]), c = mk3(pc[0], pc[1], pc[2]);
    d3 n = cross3(b - a, c - a);
    double area2 = norm3(n);
    double L0 = norm3(b - a), L1 = norm3(c - b), L2 = norm3(a - c);
    // Facets collapsed onto a line (twice-area below 1e-10 of the longest edge
    // squared, e.g. by control-point interpolation) carry a kink in their
    // facet term: its central difference is zero and so is their derivative
    // contribution here.
    double Lmax = fmax(L0, fmax(L1, L2));
    bool valid = !(area2 < kEps) && !(L0 < kEps) && !(L1 < kEps) && !(L2 < kEps) && !(area2 < 1e-10 * Lmax * Lmax);
    double out[NGC];
    for (int k = 0; k < NGC; ++k) out[k] = 0.0;
    if (valid) {
        d3 zh = n * (1.0 / area2);
        d3 xh = (b - a) * (1.0 / L0);
        d3 yh = cross3(zh, xh);
        d3 ca = c - a;
        double cx = dot3(ca, xh), cy = dot3(ca, yh);
        const GroupConst& g = groups[face_group[f]];
        d3 m = mk3(g.mdir[0], g.mdir[1], g.mdir[2]);
        out[GC_AX] = a.x; out[GC_AY] = a.y; out[GC_AZ] = a.z;
        out[GC_XX] = xh.x; out[GC_XY] = xh.y; out[GC_XZ] = xh.z;
        out[GC_YX] = yh.x; out[GC_YY] = yh.y; out[GC_YZ] = yh.z;
        out[GC_ZX] = zh.x; out[GC_ZY] = zh.y; out[GC_ZZ] = zh.z;
        out[GC_L0] = L0; out[GC_CX] = cx; out[GC_CY] = cy;
        out[GC_E1X] = (cx - L0) / L1; out[GC_E1Y] = cy / L1; out[GC_L1] = L1;
        out[GC_E2X] = -cx / L2; out[GC_E2Y] = -cy / L2; out[GC_L2] = L2;
        out[GC_GS] = want_grav ? g.gscale_jac : 0.0;
        out[GC_MS] = (want_mag && g.mag_active) ? -g.mscale : 0.0;
        // magnetic direction products in the local frame
        d3 ml = mk3(dot3(m, xh), dot3(m, yh), dot3(m, zh));
        d3 fl = mk3(dot3(fdir, xh), dot3(fdir, yh), dot3(fdir, zh));
        out[GC_MF] = ml.z * fl.z;
        double ex[3] = {1.0, out[GC_E1X], out[GC_E2X]}, ey[3] = {0.0, out[GC_E1Y], out[GC_E2Y]};
        for (int i = 0; i < 3; ++i) {
            // in-plane edge normal perp = z x e = (-ey, ex, 0)
            double mp = -ml.x * ey[i] + ml.y * ex[i], fp = -fl.x * ey[i] + fl.y * ex[i];
            out[GC_MT0 + i] = mp * fp;
        }
        out[GC_FLAGS] = 1.0 + (face_needs[f] ? 2.0 : 0.0);
    }
    for (int k = 0; k < NGC; ++k) gc[(size_t)k * T + f] = out[k];
}

// ------------------------------------------------------------- forward ----
// One pair (station o, facet in shared memory slot j) in the reference's
// operation order.  Adds the gz facet factor to *gz and the TMI facet factor
// to *tmi.
template <bool GZ, bool TMI>
__device__ __forceinline__ void pair_forward_fp64(const double* __restrict__ s, int j, int stride, d3 o,
                                                  double* gz, double* tmi) {
#define F(k) s[(k) * stride + j]
    if (F(FC_VALID) == 0.0) return;
    d3 ra = mk3(F(FC_AX) - o.x, F(FC_AY) - o.y, F(FC_AZ) - o.z);
    d3 rb = mk3(F(FC_BX) - o.x, F(FC_BY) - o.y, F(FC_BZ) - o.z);
    d3 rc = mk3(F(FC_CX) - o.x, F(FC_CY) - o.y, F(FC_CZ) - o.z);
    double la = norm3(ra), lb = norm3(rb), lc = norm3(rc);
    double omega = 0.0;
    if (!(la < kEps || lb < kEps || lc < kEps)) {
        double num = dot3(ra, cross3(rb, rc));
        double den = la * lb * lc + dot3(ra, rb) * lc + dot3(ra, rc) * lb + dot3(rb, rc) * la;
        omega = 2.0 * atan2(num, den);
    }
    d3 un = mk3(F(FC_NX), F(FC_NY), F(FC_NZ));
    double h = dot3(ra, un);
    d3 r[3] = {ra, rb, rc};
    double l[3] = {la, lb, lc};
    double dsum = 0.0, tsum = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double L = F(FC_L0 + i);
        if (L < kEps) continue;
        d3 e = mk3(F(FC_E0X + 3 * i), F(FC_E0Y + 3 * i), F(FC_E0Z + 3 * i));
        d3 r1 = r[i], r2 = r[(i + 1) % 3];
        double s1 = dot3(r1, e) / L, s2 = dot3(r2, e) / L;
        bool live;
        double lam = lambda_from(s1, s2, l[i], l[(i + 1) % 3], &live);
        if (GZ) {
            d3 p = mk3(F(FC_P0X + 3 * i), F(FC_P0Y + 3 * i), F(FC_P0Z + 3 * i));
            double dperp = -dot3(r1, p);
            dsum += dperp * lam;
        }
        if (TMI) tsum += F(FC_MT0 + i) * lam;
    }
    if (GZ) *gz += un.z * (dsum - h * omega);
    if (TMI) *tmi += F(FC_MF) * omega + tsum;
#undef F
}

// Grid: x = station tiles of blockDim.x, y = facet chunks (each inside one
// group).  Writes the chunk's unscaled facet sums per station.
// One CTA's work: station s (act = s is a station of the block) against
// facets [fb, fe); out_gz[s] / out_tmi[s] receive the unscaled sums.
template <bool GZ, bool TMI, int FT>
__device__ __forceinline__ void forward_fp64_block(double* __restrict__ sm, int s, bool act,
                                                   const double* __restrict__ sta, int T,
                                                   const double* __restrict__ fc, int fb, int fe,
                                                   double* __restrict__ out_gz, double* __restrict__ out_tmi) {
    d3 o = mk3(0, 0, 0);
    if (act) o = mk3(sta[3 * s], sta[3 * s + 1], sta[3 * s + 2]);
    double gz = 0.0, tmi = 0.0;
    for (int f0 = fb; f0 < fe; f0 += FT) {
        int nf = min(FT, fe - f0);
        __syncthreads();
        for (int idx = threadIdx.x; idx < NFC * FT; idx += blockDim.x) {
            int k = idx / FT, j = idx % FT;
            sm[idx] = (j < nf) ? fc[(size_t)k * T + f0 + j] : 0.0;
        }
        __syncthreads();
        if (act)
            for (int j = 0; j < nf; ++j) pair_forward_fp64<GZ, TMI>(sm, j, FT, o, &gz, &tmi);
    }
    if (act) {
        if (GZ) out_gz[s] = gz;
        if (TMI) out_tmi[s] = tmi;
    }
}

template <bool GZ, bool TMI, int FT>
__global__ void __launch_bounds__(128) k_forward_fp64(int S, const double* __restrict__ sta, int T,
                                                      const double* __restrict__ fc, const int32_t* __restrict__ chunk_begin,
                                                      const int32_t* __restrict__ chunk_end, double* __restrict__ part_gz,
                                                      double* __restrict__ part_tmi) {
    __shared__ double sm[NFC * FT];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int chunk = blockIdx.y;
    forward_fp64_block<GZ, TMI, FT>(sm, s, s < S, sta, T, fc, chunk_begin[chunk], chunk_end[chunk],
                                    GZ ? part_gz + (size_t)chunk * S : nullptr,
                                    TMI ? part_tmi + (size_t)chunk * S : nullptr);
}

// Batched bodies: a persistent grid walks a list of (station block, facet
// range) items -- one body's stations against one chunk of that body's
// facets -- in the order given (largest first).  Item out: offset added to
// the global station index to address the item's partial slot.
struct FwdItem {
    int32_t s0, s_end, fb, fe;
    int64_t out;
};

template <bool GZ, bool TMI, int FT>
__global__ void __launch_bounds__(128) k_forward_fp64_items(const FwdItem* __restrict__ items, int nitems,
                                                            const double* __restrict__ sta, int T,
                                                            const double* __restrict__ fc,
                                                            double* __restrict__ part_gz, double* __restrict__ part_tmi) {
    __shared__ double sm[NFC * FT];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const FwdItem w = items[it];
        const int s = w.s0 + (int)threadIdx.x;
        forward_fp64_block<GZ, TMI, FT>(sm, s, s < w.s_end, sta, T, fc, w.fb, w.fe,
                                        GZ ? part_gz + w.out : nullptr, TMI ? part_tmi + w.out : nullptr);
    }
}

// acc + v(c0) + v(c0 + 8) + ... (c < n), added in that order with eight
// loads in flight: the chunk reductions below are bound by the latency of
// their partial loads, not by the additions.
template <class F>
__device__ __forceinline__ double strided_sum8(int c0, int n, double acc, F v) {
    int c = c0;
    for (; c + 56 < n; c += 64) {
        double x[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) x[u] = v(c + 8 * u);
#pragma unroll
        for (int u = 0; u < 8; ++u) acc += x[u];
    }
    for (; c < n; c += 8) acc += v(c);
    return acc;
}

// Per station of a batch of bodies: sum of its body's chunk partials
// (grp_part_off[g] + c * n_g + local index, c < grp_nch[g]), times the body's
// group scales when `groups` is given (FP64 path; the mixed partials carry
// their scales).  Lane sums over chunks as in k_forward_reduce.
__global__ void __launch_bounds__(256) k_forward_reduce_groups(int S, const int32_t* __restrict__ sta_group,
                                                               const int32_t* __restrict__ grp_sta_off,
                                                               const int64_t* __restrict__ grp_part_off,
                                                               const int32_t* __restrict__ grp_nch,
                                                               const GroupConst* __restrict__ groups,
                                                               const double* __restrict__ part_gz,
                                                               const double* __restrict__ part_tmi,
                                                               double* __restrict__ gz, double* __restrict__ tmi) {
    __shared__ double sg[8][33], st[8][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int s = blockIdx.x * 32 + tx;
    double g = 0.0, t = 0.0;
    int grp = 0;
    if (s < S) {
        grp = sta_group[s];
        const int n = grp_sta_off[grp + 1] - grp_sta_off[grp], loc = s - grp_sta_off[grp];
        const int64_t base = grp_part_off[grp] + loc;
        const int nch = grp_nch[grp];
        if (part_gz) g = strided_sum8(ty, nch, g, [&](int c) { return part_gz[base + (int64_t)c * n]; });
        if (part_tmi) t = strided_sum8(ty, nch, t, [&](int c) { return part_tmi[base + (int64_t)c * n]; });
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
        if (groups) {
            G = G * groups[grp].gscale_fwd;
            Tm = -groups[grp].mscale * Tm;
        }
        if (gz) gz[s] = G;
        if (tmi) tmi[s] = Tm;
    }
}

// Per body (group) of a batch: data misfit of its stations, gravity + alpha
// x magnetic, from the residual definition of k_residual.
__global__ void k_group_misfit(int G, const int32_t* __restrict__ grp_sta_off, const double* __restrict__ gpred,
                               const double* __restrict__ gobs, const double* __restrict__ gw,
                               const double* __restrict__ mpred, const double* __restrict__ mobs,
                               const double* __restrict__ mw, double alpha, double* __restrict__ out) {
    __shared__ double red[256];
    const int g = blockIdx.x;
    if (g >= G) return;
    double acc = 0.0;
    for (int s = grp_sta_off[g] + threadIdx.x; s < grp_sta_off[g + 1]; s += blockDim.x) {
        if (gpred) {
            const double r = gw[s] * (gobs[s] - gpred[s]);
            acc += 0.5 * r * r;
        }
        if (mpred) {
            const double r = mw[s] * (mobs[s] - mpred[s]);
            acc += alpha * (0.5 * r * r);
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[g] = red[0];
}

// Sums chunk partials with the group scales applied chunk by chunk (a chunk
// lies in one group): gz = sum_c G*rho_g(c)*1e3*1e5 * part (gravityClosedMesh
// :162-178), tmi = sum_c -(amp_g(c)*100/(4 pi)) * part
// (magneticClosedMeshVector :367-386).  Blocks of 32 stations x 8 chunk
// lanes, lane sums added in lane order.
__global__ void __launch_bounds__(256) k_forward_reduce(int S, int nchunks, const int32_t* __restrict__ chunk_group,
                                                        const GroupConst* __restrict__ groups,
                                                        const double* __restrict__ part_gz,
                                                        const double* __restrict__ part_tmi, double* __restrict__ gz,
                                                        double* __restrict__ tmi) {
    __shared__ double sg[8][33], st[8][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int s = blockIdx.x * 32 + tx;
    double g = 0.0, t = 0.0;
    if (s < S) {
        if (part_gz)
            g = strided_sum8(ty, nchunks, g, [&](int c) {
                return part_gz[(size_t)c * S + s] * groups[chunk_group[c]].gscale_fwd;
            });
        if (part_tmi)
            t = strided_sum8(ty, nchunks, t, [&](int c) {
                return -groups[chunk_group[c]].mscale * part_tmi[(size_t)c * S + s];
            });
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

// ----------------------------------------------------------- residuals ----
// ObjectiveFunction misfit (objective.cpp:22-31, 83-105): w = 1/std or 1;
// adjoint c = -alpha * w^2 * (obs - pred); per-block partial misfit sums.
__global__ void k_residual(int S, const double* __restrict__ pred, const double* __restrict__ obs,
                           const double* __restrict__ w, double alpha, double* __restrict__ coef,
                           double* __restrict__ block_misfit) {
    __shared__ double red[256];
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    double mis = 0.0;
    if (s < S) {
        double ws = w[s];
        double r = obs[s] - pred[s];
        double res = ws * r;
        mis = 0.5 * res * res;
        if (coef) coef[s] = -alpha * (ws * ws * r);
    }
    red[threadIdx.x] = mis;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_misfit[blockIdx.x] = red[0];
}

// ------------------------------------------------------------ gradient ----
struct StationTile {
    // per station: x, y, z, gravity adjoint, magnetic adjoint
    double v[5];
};

// Per-facet accumulators over stations (local frame).
struct GradAcc {
    d3 va, vb, vc;      // vertex-direct terms
    double alam[3];     // sum Gs * Lambda_i       (d_perp direct on p1)
    double aom;         // sum Gs * Omega          (h direct on a)
    double ai;          // sum G0 * I              (n_z factor)
    d3 bh;              // sum Gs * Omega * r_a    (h through n_hat)
    d3 bl[3];           // sum Gs * Lambda_i * r1  (d_perp through perp_i)
    double amf;         // sum Ts * Omega          (MF)
    double amt[3];      // sum Ts * Lambda_i       (MT_i)
};

__device__ __forceinline__ void edge_terms(d3 r1, d3 r2, double d1, double d2, double ex, double ey, double L,
                                           double inv1, double inv2, double kom, double Gs, double Ts, double mt,
                                           double dperp, double lam, bool live, d3* g1, d3* g2) {
    // kappa_i = Gs * d_perp + Ts * MT_i
    double kl = live ? (Gs * dperp + Ts * mt) : 0.0;
    double dw = d1 * d2 + dot3(r1, r2);
    double W = dw > 1e-300 ? L / dw : 0.0;
    double s1 = r1.x * ex + r1.y * ey;
    d3 q = mk3(r1.x - s1 * ex, r1.y - s1 * ey, r1.z);
    d3 Z = mk3(ey * r1.z, -ex * r1.z, ex * r1.y - ey * r1.x);  // e_hat x r1, e_hat = (ex, ey, 0)
    d3 P = mk3(W * (kom * Z.x - kl * q.x), W * (kom * Z.y - kl * q.y), W * (kom * Z.z - kl * q.z));
    *g1 = *g1 + mk3((P.x - kl * ex) * inv1, (P.y - kl * ey) * inv1, P.z * inv1);
    *g2 = *g2 + mk3((P.x + kl * ex) * inv2, (P.y + kl * ey) * inv2, P.z * inv2);
}

// Per-facet finalisation in the local frame: differentiates the facet
// constants (n_z, the unit normal, the in-plane edge normals, the magnetic
// direction products, the edge directions) once, from the station sums, and
// returns d(contracted facet terms)/d(a, b, c) in the global frame.
__device__ inline void grad_finalize(const double* C, const GradAcc& A, const GroupConst& g, d3 fdir, double outv[9]) {
    const double L0 = C[GC_L0], cx = C[GC_CX], cy = C[GC_CY];
    const double area2 = L0 * cy;
    d3 xh = mk3(C[GC_XX], C[GC_XY], C[GC_XZ]), yh = mk3(C[GC_YX], C[GC_YY], C[GC_YZ]),
       zh = mk3(C[GC_ZX], C[GC_ZY], C[GC_ZZ]);
    d3 mg = mk3(g.mdir[0], g.mdir[1], g.mdir[2]);
    d3 ml = mk3(dot3(mg, xh), dot3(mg, yh), dot3(mg, zh));
    d3 fl = mk3(dot3(fdir, xh), dot3(fdir, yh), dot3(fdir, zh));
    d3 nh = mk3(0, 0, 1);
    d3 eh[3] = {mk3(1, 0, 0), mk3(C[GC_E1X], C[GC_E1Y], 0), mk3(C[GC_E2X], C[GC_E2Y], 0)};
    double Ls[3] = {L0, C[GC_L1], C[GC_L2]};
    d3 vbar[3] = {A.va, A.vb, A.vc};
    // n_hat adjoint
    d3 nbar = A.bh * -1.0;
    {
        double mn = ml.z, fn = fl.z;
        nbar = nbar + (ml * fn + fl * mn) * A.amf;
        // n_z = n_hat . e_z(global); e_z in local coordinates
        nbar = nbar + mk3(xh.z, yh.z, zh.z) * A.ai;
    }
    // vertex-direct: h on a, d_perp on p1
    vbar[0] = vbar[0] + nh * (-A.aom);
    for (int i = 0; i < 3; ++i) {
        d3 perp = cross3(nh, eh[i]);
        vbar[i] = vbar[i] + perp * (-A.alam[i]);
        double mp = dot3(ml, perp), fp = dot3(fl, perp);
        d3 pbar = A.bl[i] * -1.0 + (ml * fp + fl * mp) * A.amt[i];
        // perp = n x e: n_bar += e x pbar, e_bar = pbar x n
        nbar = nbar + cross3(eh[i], pbar);
        d3 ebar = cross3(pbar, nh);
        double pe = dot3(ebar, eh[i]);
        d3 eraw = (ebar - eh[i] * pe) * (1.0 / Ls[i]);
        vbar[(i + 1) % 3] = vbar[(i + 1) % 3] + eraw;
        vbar[i] = vbar[i] - eraw;
    }
    // n_hat = n / |n|, n = (b-a) x (c-a)
    double pn = dot3(nbar, nh);
    d3 nraw = (nbar - nh * pn) * (1.0 / area2);
    d3 u = mk3(L0, 0, 0), w = mk3(cx, cy, 0);
    d3 ubar = cross3(w, nraw), wbar = cross3(nraw, u);
    vbar[1] = vbar[1] + ubar;
    vbar[2] = vbar[2] + wbar;
    vbar[0] = vbar[0] - ubar - wbar;
    for (int v = 0; v < 3; ++v) {
        d3 gv = xh * vbar[v].x + yh * vbar[v].y + zh * vbar[v].z;
        outv[3 * v] = gv.x; outv[3 * v + 1] = gv.y; outv[3 * v + 2] = gv.z;
    }
}

__device__ __forceinline__ void grad_acc_zero(GradAcc& A) {
    A.va = A.vb = A.vc = mk3(0, 0, 0);
    A.bh = mk3(0, 0, 0);
    for (int i = 0; i < 3; ++i) { A.alam[i] = 0; A.bl[i] = mk3(0, 0, 0); A.amt[i] = 0; }
    A.aom = A.ai = A.amf = 0.0;
}

// Station tiles: kStationTile consecutive stations (Morton order on the
// device), bounding boxes precomputed per station set (tile_box[t][6]:
// min xyz, max xyz).
constexpr int kStationTile = 64;

// Near/far split of the mixed-precision gradient: a facet is far from a
// station tile when its centroid lies at least tau x its longest edge from
// the tile's bounding box.  Every operation is rounded explicitly, so the
// near-field and far-field kernels, compiled separately, classify every
// (facet, tile) identically and each pair is counted exactly once.
// FarKey: the facet's centroid and squared threshold; th2 < 0 means
// "everything near" (tau >= 1e30, the FP64 mode).
struct FarKey {
    double c0, c1, c2, th2;
};

__device__ __forceinline__ FarKey facet_far_key(const double* C, double tau) {
    FarKey k;
    const double L0 = C[GC_L0], cx = C[GC_CX], cy = C[GC_CY];
    const double px = __ddiv_rn(__dadd_rn(L0, cx), 3.0), py = __ddiv_rn(cy, 3.0);
    k.c0 = __dadd_rn(C[GC_AX], __dadd_rn(__dmul_rn(px, C[GC_XX]), __dmul_rn(py, C[GC_YX])));
    k.c1 = __dadd_rn(C[GC_AY], __dadd_rn(__dmul_rn(px, C[GC_XY]), __dmul_rn(py, C[GC_YY])));
    k.c2 = __dadd_rn(C[GC_AZ], __dadd_rn(__dmul_rn(px, C[GC_XZ]), __dmul_rn(py, C[GC_YZ])));
    const double th = __dmul_rn(tau, fmax(L0, fmax(C[GC_L1], C[GC_L2])));
    k.th2 = tau >= 1e30 ? -1.0 : __dmul_rn(th, th);
    return k;
}

__device__ __forceinline__ bool tile_far(const FarKey& k, const double* __restrict__ bbox) {
    if (k.th2 < 0.0) return false;
    const double d0 = fmax(0.0, fmax(__dadd_rn(bbox[0], -k.c0), __dadd_rn(k.c0, -bbox[3])));
    const double d1 = fmax(0.0, fmax(__dadd_rn(bbox[1], -k.c1), __dadd_rn(k.c1, -bbox[4])));
    const double d2 = fmax(0.0, fmax(__dadd_rn(bbox[2], -k.c2), __dadd_rn(k.c2, -bbox[5])));
    const double dd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
    return dd >= k.th2;
}

// One (facet, station) pair of the FP64 gradient: adds the station's terms,
// weighted by its adjoints (gco gravity, mco magnetic), to the facet's
// local-frame accumulators.  gsn / ms: the facet group's gz / TMI scales.
__device__ __forceinline__ void pair_gradient_fp64(const double* C, double gsn, double ms, double ox, double oy,
                                                   double oz, double gco, double mco, GradAcc& A) {
    const double nz = C[GC_ZZ];
    const double L0 = C[GC_L0], cx = C[GC_CX], cy = C[GC_CY];
    const double area2 = L0 * cy;
    double G0 = gco * gsn;  // gravity adjoint x group scale
    double Gs = G0 * nz;    // ... x n_z
    double Ts = mco * ms;   // magnetic adjoint x group TMI scale
    if (Gs == 0.0 && Ts == 0.0 && G0 == 0.0) return;
    d3 dd = mk3(ox - C[GC_AX], oy - C[GC_AY], oz - C[GC_AZ]);
    double x = dd.x * C[GC_XX] + dd.y * C[GC_XY] + dd.z * C[GC_XZ];
    double y = dd.x * C[GC_YX] + dd.y * C[GC_YY] + dd.z * C[GC_YZ];
    double z = dd.x * C[GC_ZX] + dd.y * C[GC_ZY] + dd.z * C[GC_ZZ];
    d3 ra = mk3(-x, -y, -z), rb = mk3(L0 - x, -y, -z), rc = mk3(cx - x, cy - y, -z);
    double z2 = z * z;
    double la = sqrt(x * x + y * y + z2), lb = sqrt(rb.x * rb.x + y * y + z2),
           lc = sqrt(rc.x * rc.x + rc.y * rc.y + z2);
    if (la < kEps || lb < kEps || lc < kEps) return;  // station on a vertex: not differentiable
    double h = -z;
    double Nn = h * area2;
    double Dd = la * lb * lc + dot3(ra, rb) * lc + dot3(ra, rc) * lb + dot3(rb, rc) * la;
    double om = 2.0 * atan2(Nn, Dd);
    double ia = 1.0 / la, ib = 1.0 / lb, ic = 1.0 / lc;
    // edges: 0 a->b (e=(1,0)), 1 b->c, 2 c->a
    double e1x = C[GC_E1X], e1y = C[GC_E1Y], e2x = C[GC_E2X], e2y = C[GC_E2Y];
    bool lv0, lv1, lv2;
    double lam0 = lambda_sym(la, lb, L0, &lv0);
    double lam1 = lambda_sym(lb, lc, C[GC_L1], &lv1);
    double lam2 = lambda_sym(lc, la, C[GC_L2], &lv2);
    // d_perp_i = -r1 . perp_i, perp_i = (-ey, ex, 0)
    double dp0 = y;  // -(r_a.y * 1)
    double dp1 = rb.x * e1y - rb.y * e1x;
    double dp2 = rc.x * e2y - rc.y * e2x;
    double I = dp0 * lam0 + dp1 * lam1 + dp2 * lam2 - h * om;
    double kom = -Gs * h + Ts * C[GC_MF];
    edge_terms(ra, rb, la, lb, 1.0, 0.0, L0, ia, ib, kom, Gs, Ts, C[GC_MT0], dp0, lam0, lv0, &A.va, &A.vb);
    edge_terms(rb, rc, lb, lc, e1x, e1y, C[GC_L1], ib, ic, kom, Gs, Ts, C[GC_MT1], dp1, lam1, lv1, &A.vb, &A.vc);
    edge_terms(rc, ra, lc, la, e2x, e2y, C[GC_L2], ic, ia, kom, Gs, Ts, C[GC_MT2], dp2, lam2, lv2, &A.vc, &A.va);
    A.alam[0] += Gs * lam0; A.alam[1] += Gs * lam1; A.alam[2] += Gs * lam2;
    A.aom += Gs * om;
    A.ai += G0 * I;
    A.bh = A.bh + ra * (Gs * om);
    A.bl[0] = A.bl[0] + ra * (Gs * lam0);
    A.bl[1] = A.bl[1] + rb * (Gs * lam1);
    A.bl[2] = A.bl[2] + rc * (Gs * lam2);
    A.amf += Ts * om;
    A.amt[0] += Ts * lam0; A.amt[1] += Ts * lam1; A.amt[2] += Ts * lam2;
}

__device__ __forceinline__ bool facet_grad_active(const double* C) {
    int flags = static_cast<int>(C[GC_FLAGS]);
    return (flags & 1) && (flags & 2) && (C[GC_GS] != 0.0 || C[GC_MS] != 0.0);
}

// Per-station facet gradients for dense Jacobian rows.  Grid: x = facet
// warps (one facet per thread), y = station chunks of stations_per_chunk
// consecutive stations; part layout [chunk][9][T] (vertex a xyz, b xyz,
// c xyz; global frame).  Stations are warp-uniform loads.
__global__ void __launch_bounds__(32) k_gradient_fp64(int T, const double* __restrict__ gc, int S,
                                                      const double* __restrict__ sta, const double* __restrict__ gcoef,
                                                      const double* __restrict__ mcoef, int stations_per_chunk,
                                                      const int16_t* __restrict__ face_group,
                                                      const GroupConst* __restrict__ groups, d3 fdir,
                                                      double* __restrict__ part) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    int chunk = blockIdx.y;
    int sb = chunk * stations_per_chunk, se = min(S, sb + stations_per_chunk);
    if (f >= T) return;
    double C[NGC];
#pragma unroll
    for (int k = 0; k < NGC; ++k) C[k] = gc[(size_t)k * T + f];
    const bool active = facet_grad_active(C);
    double outv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (active) {
        GradAcc A;
        grad_acc_zero(A);
        const double gsn = C[GC_GS], ms = C[GC_MS];
        for (int j = sb; j < se; ++j)
            pair_gradient_fp64(C, gsn, ms, sta[3 * j], sta[3 * j + 1], sta[3 * j + 2], gcoef ? gcoef[j] : 0.0,
                               mcoef ? mcoef[j] : 0.0, A);
        grad_finalize(C, A, groups[face_group[f]], fdir, outv);
    }
    for (int k = 0; k < 9; ++k) part[((size_t)chunk * 9 + k) * T + f] = outv[k];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

__device__ __forceinline__ void grad_acc_warp_sum(GradAcc& A) {
    A.va = mk3(warp_sum(A.va.x), warp_sum(A.va.y), warp_sum(A.va.z));
    A.vb = mk3(warp_sum(A.vb.x), warp_sum(A.vb.y), warp_sum(A.vb.z));
    A.vc = mk3(warp_sum(A.vc.x), warp_sum(A.vc.y), warp_sum(A.vc.z));
    A.bh = mk3(warp_sum(A.bh.x), warp_sum(A.bh.y), warp_sum(A.bh.z));
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        A.alam[i] = warp_sum(A.alam[i]);
        A.amt[i] = warp_sum(A.amt[i]);
        A.bl[i] = mk3(warp_sum(A.bl[i].x), warp_sum(A.bl[i].y), warp_sum(A.bl[i].z));
    }
    A.aom = warp_sum(A.aom);
    A.ai = warp_sum(A.ai);
    A.amf = warp_sum(A.amf);
}

// Objective gradient, FP64: one warp per facet.  The warp visits the
// facet's near station tiles (every tile when tau >= 1e30), lanes taking
// the tile's stations in turn; per-lane sums are reduced across the warp
// once per facet and lane 0 finalises.  The work of a facet is spread over
// 32 lanes, so facets with many near tiles leave no long tail behind.
// Warps run over `facets` (those with a DOF vertex); grid.y splits the
// station tiles into chunks of tiles_per_chunk so that a model with few such
// facets still fills the GPU.  part layout [chunk][9][T].
__global__ void __launch_bounds__(128, 3) k_gradient_warp_fp64(int T, const double* __restrict__ gc, int S,
                                                            const double* __restrict__ sta,
                                                            const double* __restrict__ gcoef,
                                                            const double* __restrict__ mcoef,
                                                            const double* __restrict__ tile_box,
                                                            const int16_t* __restrict__ face_group,
                                                            const GroupConst* __restrict__ groups, d3 fdir, double tau,
                                                            const int32_t* __restrict__ facets, int nfacets,
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
    // the facet's constants live in shared memory (one row per warp): the
    // per-lane FP64 sums and pair temporaries need the registers
    __shared__ double Csh[4][NGC];
    double* C = Csh[threadIdx.x >> 5];
    if (lane < NGC) C[lane] = gc[(size_t)lane * T + f];
    __syncwarp();
    double outv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (facet_grad_active(C)) {
        GradAcc A;
        grad_acc_zero(A);
        const double gsn = C[GC_GS], ms = C[GC_MS];
        const FarKey key = facet_far_key(C, tau);
        bool any = false;
        for (int t0 = tbeg; t0 < ntiles; t0 += 32) {
            const int t = t0 + lane;
            const bool nearT = t < ntiles && !tile_far(key, tile_box + 6 * (size_t)t);
            unsigned m = __ballot_sync(0xffffffffu, nearT);
            any |= m != 0;
            while (m) {
                const int b = __ffs(m) - 1;
                m &= m - 1;
                const int s0 = (t0 + b) * kStationTile;
#pragma unroll
                for (int k = 0; k < kStationTile; k += 32) {
                    const int j = s0 + k + lane;
                    if (j < S)
                        pair_gradient_fp64(C, gsn, ms, sta[3 * j], sta[3 * j + 1], sta[3 * j + 2],
                                           gcoef ? gcoef[j] : 0.0, mcoef ? mcoef[j] : 0.0, A);
                }
            }
        }
        if (any) {
            grad_acc_warp_sum(A);
            if (lane == 0) grad_finalize(C, A, groups[face_group[f]], fdir, outv);
        }
    }
    if (lane == 0)
        for (int k = 0; k < 9; ++k) part[(size_t)k * T + f] = outv[k];
}

// Finite-difference-XY partials (see k_face_prep_fdxy): one warp per listed
// facet x station chunk (tiles_per_chunk tiles of kStationTile stations),
// lanes over the chunk's stations.  Per station, the facet term of the base
// record and of the six moved copies (pair_forward_fp64, the reference's
// operation order), contracted with the station adjoints and the group
// scales of the analytic kernels (zero for collapsed facets):
//   sum_s (G_s (F_k - F_0) + T_s (M_k - M_0)) / h.
// Writes the x and y partials of the three corners, and zero z, into this
// chunk's slot of part ([chunk][9][T]).
__global__ void __launch_bounds__(128) k_gradient_fdxy(int T, int nf, const int32_t* __restrict__ facets,
                                                       const double* __restrict__ fcfd, const double* __restrict__ gc,
                                                       int S, const double* __restrict__ sta,
                                                       const double* __restrict__ gcoef,
                                                       const double* __restrict__ mcoef,
                                                       const int16_t* __restrict__ face_group, double inv_h,
                                                       int tiles_per_chunk, const int32_t* __restrict__ grp_sta_off,
                                                       double* __restrict__ part) {
    const int lane = threadIdx.x & 31;
    const int w = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    if (w >= nf) return;  // warp-uniform
    const int f = facets[w];
    if (grp_sta_off) {  // batched bodies: only the facet's own body's stations
        const int g = face_group[f], sb = grp_sta_off[g];
        S = grp_sta_off[g + 1] - sb;
        sta += 3 * (size_t)sb;
        if (gcoef) gcoef += sb;
        if (mcoef) mcoef += sb;
    }
    const int s0 = blockIdx.y * tiles_per_chunk * kStationTile;
    const int s1 = min(S, s0 + tiles_per_chunk * kStationTile);
    part += (size_t)blockIdx.y * 9 * T;
    __shared__ double R[4][7 * NFC];
    double* rec = R[threadIdx.x >> 5];
    for (int q = lane; q < 7 * NFC; q += 32) rec[q] = fcfd[(size_t)q * nf + w];
    __syncwarp();
    const double gs = gc[(size_t)GC_GS * T + f], ms = gc[(size_t)GC_MS * T + f];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (gs != 0.0 || ms != 0.0) {
        for (int j = s0 + lane; j < s1; j += 32) {
            const double G = gcoef ? gcoef[j] * gs : 0.0, M = mcoef ? mcoef[j] * ms : 0.0;
            if (G == 0.0 && M == 0.0) continue;
            const d3 o = mk3(sta[3 * (size_t)j], sta[3 * (size_t)j + 1], sta[3 * (size_t)j + 2]);
            double g0 = 0.0, m0 = 0.0;
            pair_forward_fp64<true, true>(rec, 0, 1, o, &g0, &m0);
#pragma unroll 1
            for (int k = 0; k < 6; ++k) {
                double gk = 0.0, mk = 0.0;
                pair_forward_fp64<true, true>(rec + (k + 1) * NFC, 0, 1, o, &gk, &mk);
                acc[k] += G * (gk - g0) + M * (mk - m0);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = warp_sum(acc[k]);
    if (lane == 0)
        for (int c = 0; c < 3; ++c) {
            part[(size_t)(3 * c) * T + f] = acc[2 * c] * inv_h;
            part[(size_t)(3 * c + 1) * T + f] = acc[2 * c + 1] * inv_h;
            part[(size_t)(3 * c + 2) * T + f] = 0.0;
        }
}

// Sums facet partials into vertex gradients: one warp per listed vertex,
// lanes over its (chunk, incident facet corner) items, then a fixed warp
// reduction (deterministic).  Slots from fd_from on hold
// finite-difference-XY partials: when fd_from < nchunks, x and y come from
// those slots only and z from the slots before them.
__global__ void k_vertex_reduce(int nverts, const int32_t* __restrict__ verts, const int32_t* __restrict__ vf_off,
                                const int32_t* __restrict__ vf, int T, int nchunks, int fd_from,
                                const double* __restrict__ part, double* __restrict__ vgrad) {
    const int i = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= nverts) return;  // warp-uniform
    const int v = verts[i];
    const int b = vf_off[v], ninc = vf_off[v + 1] - b;
    const int items = nchunks * ninc;
    double gx = 0, gy = 0, gz = 0;
    for (int it = lane; it < items; it += 32) {
        const int c = it / ninc, k = b + it % ninc;
        const int f = vf[k] / 3, corner = vf[k] % 3;
        const double* p = part + ((size_t)c * 9 + 3 * corner) * T + f;
        const bool xy = fd_from >= nchunks || c >= fd_from;
        if (xy) {
            gx += p[0];
            gy += p[(size_t)T];
        }
        if (c < fd_from) gz += p[(size_t)2 * T];
    }
    gx = warp_sum(gx);
    gy = warp_sum(gy);
    gz = warp_sum(gz);
    if (lane == 0) {
        vgrad[3 * v] = gx;
        vgrad[3 * v + 1] = gy;
        vgrad[3 * v + 2] = gz;
    }
}

// grad[d] = sum_refs vgrad[vertex][axis] * axis scale + reference-model term
// (gather of gravity_forward.cpp:269-289 contracted; reference_model.cpp:22-25).
__global__ void k_dof_gather(int np, const int32_t* __restrict__ dof_off, const int32_t* __restrict__ ref_vertex,
                             const uint8_t* __restrict__ ref_axis, const double* __restrict__ ref_scale,
                             const double* __restrict__ vgrad, const double* __restrict__ params,
                             const double* __restrict__ ref_params, double ref_weight,
                             const double* __restrict__ vgrad_smooth, double smooth_weight,
                             double* __restrict__ grad) {
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= np) return;
    double acc = 0.0;
    for (int r = dof_off[d]; r < dof_off[d + 1]; ++r) acc += vgrad[3 * ref_vertex[r] + ref_axis[r]] * ref_scale[r];
    if (vgrad_smooth) {  // SurfaceSmoothness::gradient gather (smoothness.cpp:231-242), times its weight
        double s = 0.0;
        for (int r = dof_off[d]; r < dof_off[d + 1]; ++r)
            s += vgrad_smooth[3 * ref_vertex[r] + ref_axis[r]] * ref_scale[r];
        acc += smooth_weight * s;
    }
    if (ref_params) acc += ref_weight * (params[d] - ref_params[d]);
    grad[d] = acc;
}

// Chain gather (no reference counterpart; the reference reads the vertex
// gradient at the DOF vertices only, gravity_forward.cpp:270-289).  The
// scatter is DOF writes -> interpolation -> averaging; its adjoint runs the
// transposes in reverse.  The averaging's transpose is the averaging itself
// (k_sync_shared on the gradient: its matrix is symmetric).  The
// interpolation's transpose, out of place: a source receives w x the
// gradient of each row it feeds, a row keeps nothing (its position was
// overwritten), every other vertex keeps its own.  Fixed summation order,
// no atomics.
__global__ void k_interp_adjoint(int V, const int32_t* __restrict__ interp_off, const int32_t* __restrict__ adj_off,
                                 const int32_t* __restrict__ adj_row, const double* __restrict__ adj_w,
                                 const double* __restrict__ vg, double* __restrict__ out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const bool row = interp_off[v + 1] > interp_off[v];
    double g0 = row ? 0.0 : vg[3 * (size_t)v], g1 = row ? 0.0 : vg[3 * (size_t)v + 1],
           g2 = row ? 0.0 : vg[3 * (size_t)v + 2];
    for (int k = adj_off[v]; k < adj_off[v + 1]; ++k) {
        const double w = adj_w[k];
        const double* q = vg + 3 * (size_t)adj_row[k];
        g0 += w * q[0];
        g1 += w * q[1];
        g2 += w * q[2];
    }
    out[3 * (size_t)v] = g0;
    out[3 * (size_t)v + 1] = g1;
    out[3 * (size_t)v + 2] = g2;
}

// y += a x over n doubles (the smoothness vertex gradient into the misfit's
// before the chain gather).
__global__ void k_axpy(size_t n, double a, const double* __restrict__ x, double* __restrict__ y) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}

// Dense Jacobian rows from per-station facet partials (one chunk per
// station): J[s][d] = sum_refs (sum_{(f,c) of v} part) * scale, with the
// reference's |vertex gradient| < 1e-30 skip.
__global__ void k_jacobian_gather(int nst, int np, const int32_t* __restrict__ dof_off,
                                  const int32_t* __restrict__ ref_vertex, const uint8_t* __restrict__ ref_axis,
                                  const double* __restrict__ ref_scale, const int32_t* __restrict__ vf_off,
                                  const int32_t* __restrict__ vf, int T, const double* __restrict__ part,
                                  double* __restrict__ J, int ld) {
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    int s = blockIdx.y;
    if (d >= np || s >= nst) return;
    double acc = 0.0;
    for (int r = dof_off[d]; r < dof_off[d + 1]; ++r) {
        int v = ref_vertex[r], ax = ref_axis[r];
        double pg = 0.0;
        for (int k = vf_off[v]; k < vf_off[v + 1]; ++k) {
            int f = vf[k] / 3, corner = vf[k] % 3;
            pg += part[((size_t)s * 9 + 3 * corner + ax) * T + f];
        }
        if (fabs(pg) < 1e-30) continue;
        acc += pg * ref_scale[r];
    }
    J[(size_t)s * ld + d] = acc;
}

// Final deterministic reduction of block partials and objective assembly:
// out = {grav misfit, mag misfit, reg, 0, total}.
// ---------------------------------------------------------- smoothness ----
// SurfaceSmoothness (modules/litho-regularization/src/regularization/
// smoothness.cpp): every non-fixed vertex against the mean of its
// same-freedom mesh neighbours (nbr: CSR, ascending, built on the host like
// SurfaceMesh::buildNeighbors surface_mesh.cpp:265-286).

// Free axes of a VertexFreedom code (surface_mesh.h:9-19); ALONG_VECTOR is
// rejected on the host.
__device__ __forceinline__ void freedom_mask(int fr, bool m[3]) {
    m[0] = fr == 2 || fr == 5 || fr == 6 || fr == 8;
    m[1] = fr == 3 || fr == 5 || fr == 7 || fr == 8;
    m[2] = fr == 1 || fr == 6 || fr == 7 || fr == 8;
}

// diff_v = p_v - mean_v (evaluate :29-49) and the per-vertex penalty
// 0.5 |mask diff|^2 (:51-99), summed per block; same operation order as the
// reference.
__global__ void k_smooth_diff(int V, const double* __restrict__ pos, const uint8_t* __restrict__ freedom,
                              const int32_t* __restrict__ off, const int32_t* __restrict__ nbr,
                              double* __restrict__ diff, double* __restrict__ block_pen) {
    __shared__ double red[256];
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    double pen = 0.0;
    if (v < V) {
        const int b = off[v], e = off[v + 1];
        double d0 = 0.0, d1 = 0.0, d2 = 0.0;
        if (e > b) {
            double m0 = 0.0, m1 = 0.0, m2 = 0.0;
            for (int i = b; i < e; ++i) {
                const double* q = pos + 3 * (size_t)nbr[i];
                m0 = __dadd_rn(m0, q[0]); m1 = __dadd_rn(m1, q[1]); m2 = __dadd_rn(m2, q[2]);
            }
            const double n = static_cast<double>(e - b);
            m0 = __ddiv_rn(m0, n); m1 = __ddiv_rn(m1, n); m2 = __ddiv_rn(m2, n);
            d0 = __dsub_rn(pos[3 * (size_t)v], m0);
            d1 = __dsub_rn(pos[3 * (size_t)v + 1], m1);
            d2 = __dsub_rn(pos[3 * (size_t)v + 2], m2);
            auto sq = [](double d) { return __dmul_rn(d, d); };
            switch (freedom[v]) {
            case 1: pen = __dmul_rn(__dmul_rn(0.5, d2), d2); break;
            case 2: pen = __dmul_rn(__dmul_rn(0.5, d0), d0); break;
            case 3: pen = __dmul_rn(__dmul_rn(0.5, d1), d1); break;
            case 5: pen = __dmul_rn(0.5, __dadd_rn(sq(d0), sq(d1))); break;
            case 6: pen = __dmul_rn(0.5, __dadd_rn(sq(d0), sq(d2))); break;
            case 7: pen = __dmul_rn(0.5, __dadd_rn(sq(d1), sq(d2))); break;
            case 8: pen = __dmul_rn(0.5, __dadd_rn(__dadd_rn(sq(d0), sq(d1)), sq(d2))); break;
            default: break;
            }
        }
        diff[3 * (size_t)v] = d0; diff[3 * (size_t)v + 1] = d1; diff[3 * (size_t)v + 2] = d2;
    }
    red[threadIdx.x] = pen;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_pen[blockIdx.x] = red[0];
}

// Per-vertex smoothness gradient (gradient :152-242): own term mask(diff_v),
// then -mask(diff_u) / n_u for every same-freedom neighbour u in ascending
// order (the neighbour relation and the freedom filter are symmetric, so the
// vertices that add to v are exactly v's own list).
__global__ void k_smooth_vgrad(int V, const uint8_t* __restrict__ freedom, const int32_t* __restrict__ off,
                               const int32_t* __restrict__ nbr, const double* __restrict__ diff,
                               double* __restrict__ vg) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    const int b = off[v], e = off[v + 1];
    if (e > b) {
        bool m[3];
        freedom_mask(freedom[v], m);
        if (m[0]) g0 = diff[3 * (size_t)v];
        if (m[1]) g1 = diff[3 * (size_t)v + 1];
        if (m[2]) g2 = diff[3 * (size_t)v + 2];
        for (int i = b; i < e; ++i) {
            const int u = nbr[i];
            const double nu = static_cast<double>(off[u + 1] - off[u]);
            if (m[0]) g0 = __dadd_rn(g0, __ddiv_rn(-diff[3 * (size_t)u], nu));
            if (m[1]) g1 = __dadd_rn(g1, __ddiv_rn(-diff[3 * (size_t)u + 1], nu));
            if (m[2]) g2 = __dadd_rn(g2, __ddiv_rn(-diff[3 * (size_t)u + 2], nu));
        }
    }
    vg[3 * (size_t)v] = g0; vg[3 * (size_t)v + 1] = g1; vg[3 * (size_t)v + 2] = g2;
}

// Objective components: misfits from the residual block sums; regularisation
// = smoothness (weight x block penalty sums) + reference-model term, in the
// order the runner registers them (runner.cpp:164-179).
__global__ void k_objective_final(int nbg, const double* __restrict__ bg, int nbm, const double* __restrict__ bm,
                                  double alpha, int np, const double* __restrict__ params,
                                  const double* __restrict__ ref_params, double ref_weight, int nbs,
                                  const double* __restrict__ bs, double smooth_weight, double* __restrict__ out5,
                                  double* __restrict__ f_out) {
    __shared__ double red[256];
    double reg = 0.0;
    if (ref_params)
        for (int d = threadIdx.x; d < np; d += blockDim.x) {
            double dd = params[d] - ref_params[d];
            reg += dd * dd;
        }
    red[threadIdx.x] = reg;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double g = 0.0, m = 0.0;
        for (int i = 0; i < nbg; ++i) g += bg[i];
        for (int i = 0; i < nbm; ++i) m += bm[i];
        double r = ref_params ? 0.5 * ref_weight * red[0] : 0.0;
        if (bs) {
            double sp = 0.0;
            for (int i = 0; i < nbs; ++i) sp += bs[i];
            r = smooth_weight * sp + r;
        }
        double total = g + alpha * m + r;
        out5[0] = g; out5[1] = m; out5[2] = r; out5[3] = 0.0; out5[4] = total;
        if (f_out) *f_out = total;
    }
}

}  // namespace litho_b200
