// Patch forward of the mixed-precision path: the far field evaluated once per
// (station, vertex) and once per (station, edge) instead of three times per
// (station, facet).
//
// For a station o and a facet f of a patch (patches.hpp), the reference's
// facet terms (faceNagyContribution gravity_forward.cpp:13-42, magneticFacet
// magnetic_forward.cpp:312-347) use
//   * d_v = |v - o| for the three corners,
//   * Lambda_e = log((d1 + d2 + L) / (d1 + d2 - L)) = 2 atanh(L / (d1 + d2))
//     for the three edges (the symmetric form of lineIntegralTerm
//     geometry.cpp:32-52, equal to the oriented one because d2^2 - d1^2 =
//     s2^2 - s1^2 along the edge's line),
//   * Omega_f = 2 atan2(r_a . N, d_a d_b d_c + (r_a.r_b) d_c + (r_a.r_c) d_b
//     + (r_b.r_c) d_a) (solidAngle geometry.cpp:10-30) with N = (b-a)x(c-a)
//     and r_a.r_b = (d_a^2 + d_b^2 - |ab|^2) / 2.
// TMI of the far facets is then sum_e MT_e Lambda_e + sum_f MF_f Omega_f,
// where MT_e sums the TMI edge coefficients (m.t_i)(f.t_i) (times the group
// scale) of the patch facets that use edge e: an exact regrouping of the
// reference's per-facet sum.  gz of a far facet is n_z * G rho * the
// integral of 1/r over the facet, by Dunavant's 6-point rule (3-point beyond
// 4 tau x size), skipped when n_z == 0 exactly (a vertical facet: its gz
// term is zero).  All of this runs in FP32 in a frame centred on the patch's
// first vertex (the station is moved into it once per patch in FP64).
// Mid-field facets (tau/2 <= distance / size < tau) keep the per-facet FP32
// record path and near ones the FP64 path of kernels_mixed.cuh; their edge
// shares are masked out of MT_e for the warps that see them that close.
#pragma once
#include "kernels_mixed.cuh"
#include "patches.hpp"

namespace litho_b200 {

struct __align__(16) PatchHead {
    int nv, ne, nf, nbytes;
    double ox, oy, oz, pad;  // frame origin: the patch's first vertex
};
struct __align__(16) PatchVert {
    float x, y, z, pad;  // position - origin
};
struct __align__(16) PatchEdgeA {
    int lv1, lv2;  // local vertex indices
    float L;       // edge length
    float mt;      // doubled TMI edge coefficient, summed over the users
};
struct __align__(16) PatchEdgeB {
    int users;       // lf1 | lf2 << 8 (kNoFacet: none)
    float mt1, mt2;  // each user's share of mt
    int pad;
};
struct __align__(16) PatchFacet {
    uint32_t corners;              // local vertex indices a | b << 8 | c << 16
    float nx, ny, nz;              // N = (b - a) x (c - a) (twice the area times the unit normal)
    float cf;                      // (a - origin) . N
    float mf2;                     // doubled TMI solid-angle coefficient (the series gives atan, not 2 atan)
    float gq;                      // n_z * G rho 1e8 * area (0: no gz term)
    float size;                    // longest edge; -1: contributes nothing
    float l2ab, l2bc, l2ca;        // squared edge lengths
    int gfacet;                    // global facet index (mid / near fallbacks)
    float cenx, ceny, cenz, pad0;  // centroid (absolute): the near/far test
    float q3[9];                   // the 3-point rule's points - origin
    float q6[18];                  // the 6-point rule's points - origin
    float pad1;
};
static_assert(sizeof(PatchHead) == kPatchHeadBytes, "PatchHead");
static_assert(sizeof(PatchVert) == kPatchVertBytes, "PatchVert");
static_assert(sizeof(PatchEdgeA) + sizeof(PatchEdgeB) == kPatchEdgeBytes, "PatchEdge");
static_assert(sizeof(PatchFacet) == kPatchFacetBytes, "PatchFacet");
static_assert(kPatchMaxBytes % 16 == 0, "bulk copies move multiples of 16 bytes");

// Per-evaluation records, part 1: one thread per facet.  The facet's FP64
// constants in the reference's operation order (the SoA mc[NMC][T] that near
// pairs read, kernels_mixed.cuh's MixedConst layout), its patch facet record
// (in its patch's frame) and its doubled, group-scaled TMI edge coefficients
// mt2[3][T] in the facet's own edge order (edge i: v_i -> v_{i+1}).
__global__ void __launch_bounds__(128) k_face_prep_patch(int T, const int32_t* __restrict__ tri,
                                                         const double* __restrict__ pos,
                                                         const int16_t* __restrict__ face_group,
                                                         const GroupConst* __restrict__ groups, d3 fdir,
                                                         const int32_t* __restrict__ facetPatch,
                                                         const int32_t* __restrict__ facetSlot,
                                                         const int32_t* __restrict__ facetOff,
                                                         const uint32_t* __restrict__ corners,
                                                         const int32_t* __restrict__ vertOff,
                                                         const int32_t* __restrict__ verts,
                                                         const int32_t* __restrict__ edgeOff,
                                                         const int32_t* __restrict__ blobOff,
                                                         double* __restrict__ mc, float* __restrict__ mt2,
                                                         unsigned char* __restrict__ blobs, int drop_collapsed) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= T) return;
    d3 v[3];
    for (int k = 0; k < 3; ++k) {
        const double* q = pos + 3 * (size_t)tri[3 * f + k];
        v[k] = mk3(q[0], q[1], q[2]);
    }
    // reference-order normal and magnetic products (bit-identical to the
    // reference, which matters for facets collapsed to a line)
    const d3 n = cross_rn(sub_rn(v[1], v[0]), sub_rn(v[2], v[0]));
    const double area2 = norm_rn(n);
    const bool valid = !(area2 < kEps) && !(drop_collapsed && facet_collapsed(v, area2));
    double out[NMC];
    for (int k = 0; k < NMC; ++k) out[k] = 0.0;
    double mt[3] = {0.0, 0.0, 0.0}, L[3], mfv = 0.0, sgz = 0.0;
    for (int i = 0; i < 3; ++i) L[i] = norm_rn(sub_rn(v[(i + 1) % 3], v[i]));
    if (valid) {
        const d3 un = div_rn(n, area2);
        const GroupConst& g = groups[face_group[f]];
        const d3 m = mk3(g.mdir[0], g.mdir[1], g.mdir[2]);
        const double mf = __dmul_rn(dot_rn(m, un), dot_rn(fdir, un));
        for (int i = 0; i < 3; ++i) {
            const d3 e = sub_rn(v[(i + 1) % 3], v[i]);
            const d3 eh = (L[i] < kEps) ? mk3(0, 0, 0) : div_rn(e, L[i]);
            const d3 perp = cross_rn(un, eh);
            mt[i] = -g.mscale * __dmul_rn(dot_rn(m, perp), dot_rn(fdir, perp));
        }
        mfv = -g.mscale * mf;
        sgz = un.z * g.gscale_fwd;
        int k = 0;  // local frame: rotated so that edge 0 is the longest
        if (L[1] > L[k]) k = 1;
        if (L[2] > L[k]) k = 2;
        const d3 a = v[k], b = v[(k + 1) % 3], c = v[(k + 2) % 3];
        const double L0 = L[k];
        const d3 xh = (b - a) * (1.0 / L0);
        // On a facet collapsed onto a line the reference's unit normal is
        // rounding noise and not perpendicular to the edges; the frame must
        // stay orthonormal for the local coordinates (and so Lambda, which the
        // reference takes from positions alone) to be right.
        d3 zh = un - xh * dot3(un, xh);
        zh = zh * (1.0 / norm3(zh));
        const d3 yh = cross3(zh, xh);
        const d3 ca = c - a;
        const double cx = dot3(ca, xh), cy = dot3(ca, yh);
        const double L1 = L[(k + 1) % 3], L2 = L[(k + 2) % 3];
        out[MC_AX] = a.x; out[MC_AY] = a.y; out[MC_AZ] = a.z;
        out[MC_XX] = xh.x; out[MC_XY] = xh.y; out[MC_XZ] = xh.z;
        out[MC_YX] = yh.x; out[MC_YY] = yh.y; out[MC_YZ] = yh.z;
        out[MC_ZX] = zh.x; out[MC_ZY] = zh.y; out[MC_ZZ] = zh.z;
        out[MC_L0] = L0; out[MC_CX] = cx; out[MC_CY] = cy;
        out[MC_L1] = L1; out[MC_L2] = L2;
        if (!(L1 < kEps)) { out[MC_E1X] = (cx - L0) / L1; out[MC_E1Y] = cy / L1; }
        if (!(L2 < kEps)) { out[MC_E2X] = -cx / L2; out[MC_E2Y] = -cy / L2; }
        out[MC_SGZ] = sgz;
        out[MC_MF] = mfv;
        out[MC_MT0] = mt[k];
        out[MC_MT1] = mt[(k + 1) % 3];
        out[MC_MT2] = mt[(k + 2) % 3];
        out[MC_CENX] = (v[0].x + v[1].x + v[2].x) / 3.0;
        out[MC_CENY] = (v[0].y + v[1].y + v[2].y) / 3.0;
        out[MC_CENZ] = (v[0].z + v[1].z + v[2].z) / 3.0;
        out[MC_SIZE] = L0;
        out[MC_VALID] = 1.0;
    }
    for (int k = 0; k < NMC; ++k) mc[(size_t)k * T + f] = out[k];
    for (int i = 0; i < 3; ++i) mt2[(size_t)i * T + f] = (float)(2.0 * mt[i]);
    // the patch facet record, in the patch's frame
    const int p = facetPatch[f], slot = facetSlot[f];
    const int nv = vertOff[p + 1] - vertOff[p], ne = edgeOff[p + 1] - edgeOff[p];
    const double* o = pos + 3 * (size_t)verts[vertOff[p]];
    const d3 org = mk3(o[0], o[1], o[2]);
    PatchFacet F;
    F.corners = corners[facetOff[p] + slot];
    F.pad0 = 0.f;
    F.pad1 = 0.f;
    F.gfacet = f;
    F.nx = (float)n.x; F.ny = (float)n.y; F.nz = (float)n.z;
    F.cf = (float)dot3(v[0] - org, n);
    F.mf2 = (float)(2.0 * mfv);
    F.gq = (float)(sgz * 0.5 * area2);
    F.size = valid ? (float)fmax(L[0], fmax(L[1], L[2])) : -1.f;
    F.l2ab = (float)(L[0] * L[0]); F.l2bc = (float)(L[1] * L[1]); F.l2ca = (float)(L[2] * L[2]);
    F.cenx = (float)((v[0].x + v[1].x + v[2].x) / 3.0);
    F.ceny = (float)((v[0].y + v[1].y + v[2].y) / 3.0);
    F.cenz = (float)((v[0].z + v[1].z + v[2].z) / 3.0);
    const d3 eb = v[1] - v[0], ec = v[2] - v[0], a0 = v[0] - org;
    for (int q = 0; q < 3; ++q) {
        const d3 pq = a0 + eb * (double)kTri3Bb[q] + ec * (double)kTri3Bc[q];
        F.q3[3 * q] = (float)pq.x; F.q3[3 * q + 1] = (float)pq.y; F.q3[3 * q + 2] = (float)pq.z;
    }
    for (int q = 0; q < 6; ++q) {
        const d3 pq = a0 + eb * (double)kDun6Bb[q] + ec * (double)kDun6Bc[q];
        F.q6[3 * q] = (float)pq.x; F.q6[3 * q + 1] = (float)pq.y; F.q6[3 * q + 2] = (float)pq.z;
    }
    unsigned char* B = blobs + blobOff[p];
    float4* dst = reinterpret_cast<float4*>(B + kPatchHeadBytes + nv * kPatchVertBytes + ne * kPatchEdgeBytes +
                                            slot * kPatchFacetBytes);
    const float4* src = reinterpret_cast<const float4*>(&F);
#pragma unroll
    for (int k = 0; k < kPatchFacetBytes / 16; ++k) dst[k] = src[k];
}

// Per-evaluation records, part 2: one warp per patch writes the header, the
// patch-frame vertices and the edges (length, summed coefficient and the two
// users' shares of it, from the facets' mt2 written by k_face_prep_patch).
__global__ void __launch_bounds__(32) k_patch_prep(int P, const double* __restrict__ pos,
                                                   const int32_t* __restrict__ facetOff,
                                                   const int32_t* __restrict__ facets,
                                                   const int32_t* __restrict__ vertOff,
                                                   const int32_t* __restrict__ verts,
                                                   const int32_t* __restrict__ edgeOff,
                                                   const uint32_t* __restrict__ edgeInfo,
                                                   const uint8_t* __restrict__ edgeSlot,
                                                   const int32_t* __restrict__ blobOff, int T,
                                                   const float* __restrict__ mt2, unsigned char* __restrict__ blobs) {
    const int p = blockIdx.x, lane = threadIdx.x;
    if (p >= P) return;
    const int f0 = facetOff[p], nf = facetOff[p + 1] - f0;
    const int v0 = vertOff[p], nv = vertOff[p + 1] - v0;
    const int e0 = edgeOff[p], ne = edgeOff[p + 1] - e0;
    unsigned char* B = blobs + blobOff[p];
    PatchVert* PV = reinterpret_cast<PatchVert*>(B + kPatchHeadBytes);
    PatchEdgeA* EA = reinterpret_cast<PatchEdgeA*>(B + kPatchHeadBytes + nv * kPatchVertBytes);
    PatchEdgeB* EB = reinterpret_cast<PatchEdgeB*>(EA + ne);
    const double* o = pos + 3 * (size_t)verts[v0];
    const d3 org = mk3(o[0], o[1], o[2]);
    if (lane == 0) {
        PatchHead h;
        h.nv = nv; h.ne = ne; h.nf = nf; h.nbytes = blobOff[p + 1] - blobOff[p];
        h.ox = org.x; h.oy = org.y; h.oz = org.z; h.pad = 0.0;
        *reinterpret_cast<PatchHead*>(B) = h;
    }
    if (lane < nv) {
        const double* q = pos + 3 * (size_t)verts[v0 + lane];
        PatchVert pv;
        pv.x = (float)(q[0] - org.x); pv.y = (float)(q[1] - org.y); pv.z = (float)(q[2] - org.z); pv.pad = 0.f;
        PV[lane] = pv;
    }
    for (int e = lane; e < ne; e += 32) {
        const uint32_t info = edgeInfo[e0 + e], sl = edgeSlot[e0 + e];
        const int lv1 = info & 0xff, lv2 = (info >> 8) & 0xff, lf1 = (info >> 16) & 0xff, lf2 = info >> 24;
        const float m1 = mt2[(size_t)(sl & 3) * T + facets[f0 + lf1]];
        const float m2 = lf2 != kNoFacet ? mt2[(size_t)((sl >> 2) & 3) * T + facets[f0 + lf2]] : 0.f;
        const double* qa = pos + 3 * (size_t)verts[v0 + lv1];
        const double* qb = pos + 3 * (size_t)verts[v0 + lv2];
        PatchEdgeA a;
        a.lv1 = lv1; a.lv2 = lv2;
        a.L = (float)norm3(mk3(qb[0] - qa[0], qb[1] - qa[1], qb[2] - qa[2]));
        a.mt = m1 + m2;
        PatchEdgeB b;
        b.users = lf1 | lf2 << 8; b.mt1 = m1; b.mt2 = m2; b.pad = 0;
        EA[e] = a;
        EB[e] = b;
    }
}

// ------------------------------------------------------- FP32 primitives --
// atanh(L / dsum) (half of Lambda).  For v = L / dsum <= 1/4 the Maclaurin
// series through v^13 (Abramowitz & Stegun 4.1.28), whose first omitted term
// is below 4e-10 v there; larger arguments take 0.5 log1p(2 v / (1 - v)).
__device__ __forceinline__ float atanh_half_lambda(float L, float dsum) {
    const float v = __fdividef(L, dsum);
    if (v <= 0.25f) {
        const float v2 = v * v;
        const float p = fmaf(v2, fmaf(v2, fmaf(v2, fmaf(v2, fmaf(v2, fmaf(v2, 1.f / 13.f, 1.f / 11.f), 1.f / 9.f),
                                                     1.f / 7.f), 1.f / 5.f), 1.f / 3.f), 1.f);
        return v * p;
    }
    return 0.5f * log1pf(__fdividef(2.f * v, 1.f - v));
}

// atanh(v) / v = 1 + v^2/3 + ... + v^12/13 and atan(t) / t = 1 - t^2/3 + ...
// + t^8/9 (Abramowitz & Stegun 4.1.28, 4.4.42) as polynomials in the square:
// below 8e-8 relative for v <= 3/8, below 1e-10 for |t| <= 1/8.
__device__ __forceinline__ float atanh_poly(float v2) {
    return fmaf(v2, fmaf(v2, fmaf(v2, fmaf(v2, fmaf(v2, fmaf(v2, 1.f / 13.f, 1.f / 11.f), 1.f / 9.f), 1.f / 7.f),
                              1.f / 5.f), 1.f / 3.f), 1.f);
}
__device__ __forceinline__ float atan_poly(float t2) {
    return fmaf(t2, fmaf(t2, fmaf(t2, fmaf(t2, 1.f / 9.f, -1.f / 7.f), 1.f / 5.f), -1.f / 3.f), 1.f);
}

// atan(y / x) (half the solid angle): series when x > 0 and |y| <= x / 8,
// else atan2f.
__device__ __forceinline__ float atan_half_omega(float y, float x) {
    if (x > 0.f && fabsf(y) <= 0.125f * x) return atan_series(__fdividef(y, x));
    return atan2f(y, x);
}

constexpr long long kPatchWaitLimit = 1ll << 22;  // mbarrier polls for one patch copy (well under a second)

__device__ __forceinline__ uint32_t patch_smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool patch_wait(uint32_t mbar, uint32_t parity) {
    for (long long i = 0; i < kPatchWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (i > 16) __nanosleep(64);
    }
    return false;
}

// One patch blob into shared memory by the bulk-copy engine (no multicast:
// the source is this GPU's own memory).  Called by one thread.
__device__ __forceinline__ void patch_issue(void* dst, const unsigned char* src, int bytes, uint32_t mbar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier generic reads of the buffer come first
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     patch_smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

template <int NT>
struct PatchSmem {
    unsigned char buf[2][kPatchMaxBytes];
    float dv[kPatchVerts][NT];      // per-station vertex distances of the current patch
    double nearSlot[NT / 32][NMC];  // one near facet's FP64 constants per warp
    unsigned long long mbar[2];
};

// Station block (this thread: station s, live when act) against patches
// [pb, pe); out_gz[s] / out_tmi[s] receive the sums.  Returns false when a
// patch copy did not land within the wait limit (block-uniform): the error
// flag is raised and the block's stations get NaN.
template <bool GZ, bool TMI, int NT>
__device__ __forceinline__ bool forward_patch_block(PatchSmem<NT>& sm, int s, bool act,
                                                    const double* __restrict__ sta,
                                                    const unsigned char* __restrict__ blobs,
                                                    const int32_t* __restrict__ blobOff, int pb, int pe,
                                                    const double* __restrict__ mc, int T, float tau, double* __restrict__ out_gz,
                                                    double* __restrict__ out_tmi,
                                                    unsigned long long* __restrict__ near_pairs,
                                                    unsigned int* __restrict__ err, uint32_t& phases) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, tid = threadIdx.x;
    // inactive lanes evaluate the warp's first live station (results dropped)
    const unsigned live = __ballot_sync(0xffffffffu, act);
    const int src = live ? (s - lane + __ffs(live) - 1) : s;
    double ox = 0.0, oy = 0.0, oz = 0.0;
    if (act) {
        ox = sta[3 * s]; oy = sta[3 * s + 1]; oz = sta[3 * s + 2];
    } else if (live) {
        ox = sta[3 * src]; oy = sta[3 * src + 1]; oz = sta[3 * src + 2];
    }
    float bb[6] = {act ? (float)ox : 3e38f, act ? (float)oy : 3e38f, act ? (float)oz : 3e38f,
                   act ? -(float)ox : 3e38f, act ? -(float)oy : 3e38f, act ? -(float)oz : 3e38f};
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) bb[k] = fminf(bb[k], __shfl_xor_sync(0xffffffffu, bb[k], off));
    float* dvp = &sm.dv[0][tid];
    double gz = 0.0, tmi = 0.0;
    unsigned long long nearCount = 0;
    const int nP = pe - pb;
    const uint32_t mb0 = patch_smem_addr(&sm.mbar[0]), mb1 = patch_smem_addr(&sm.mbar[1]);
    if (tid == 0 && nP > 0) {
        const int o0 = __ldg(blobOff + pb);
        patch_issue(sm.buf[0], blobs + o0, __ldg(blobOff + pb + 1) - o0, mb0);
    }
    for (int i = 0; i < nP; ++i) {
        const int b = i & 1;
        const bool ok = patch_wait(b ? mb1 : mb0, (phases >> b) & 1u);
        if (!__syncthreads_and(ok)) {  // every thread is past the previous patch here
            if (tid == 0) {
                atomicOr(err, 1u);
                patch_wait(b ? mb1 : mb0, (phases >> b) & 1u);  // drain the copy in flight before leaving
            }
            if (act) {  // the station's sums are incomplete: make that visible
                if (GZ) out_gz[s] = __longlong_as_double(0x7ff8000000000000ll);
                if (TMI) out_tmi[s] = __longlong_as_double(0x7ff8000000000000ll);
            }
            return false;
        }
        phases ^= 1u << b;
        if (tid == 0 && i + 1 < nP) {  // the other buffer held patch i - 1, which every warp has finished
            const int o1 = __ldg(blobOff + pb + i + 1);
            patch_issue(sm.buf[b ^ 1], blobs + o1, __ldg(blobOff + pb + i + 2) - o1, b ? mb0 : mb1);
        }
        const unsigned char* B = sm.buf[b];
        const PatchHead& H = *reinterpret_cast<const PatchHead*>(B);
        const int nv = H.nv, ne = H.ne, nf = H.nf;
        const PatchVert* PV = reinterpret_cast<const PatchVert*>(B + kPatchHeadBytes);
        const PatchEdgeA* EA = reinterpret_cast<const PatchEdgeA*>(B + kPatchHeadBytes + nv * kPatchVertBytes);
        const PatchEdgeB* EB = reinterpret_cast<const PatchEdgeB*>(EA + ne);
        const PatchFacet* PF =
            reinterpret_cast<const PatchFacet*>(B + kPatchHeadBytes + nv * kPatchVertBytes + ne * kPatchEdgeBytes);
        // lane j: facet j against this warp's station box
        bool valid = false, vfar = false, far = false, mid = false, hasGz = false;
        if (lane < nf && !(PF[lane].size < 0.f)) {
            valid = true;
            hasGz = PF[lane].gq != 0.f;  // n_z == 0: no gz term
            const float cxw = PF[lane].cenx, cyw = PF[lane].ceny, czw = PF[lane].cenz;
            const float ddx = fmaxf(0.f, fmaxf(bb[0] - cxw, cxw + bb[3]));
            const float ddy = fmaxf(0.f, fmaxf(bb[1] - cyw, cyw + bb[4]));
            const float ddz = fmaxf(0.f, fmaxf(bb[2] - czw, czw + bb[5]));
            const float d2 = ddx * ddx + ddy * ddy + ddz * ddz;
            const float lim = tau * PF[lane].size, limMid = 0.5f * lim;
            vfar = d2 >= 16.f * (lim * lim);
            far = !vfar && d2 >= lim * lim;
            mid = !vfar && !far && d2 >= limMid * limMid;
        }
        const unsigned vfarMask = __ballot_sync(0xffffffffu, valid && vfar);
        const unsigned midMask = __ballot_sync(0xffffffffu, valid && mid);
        const unsigned fastMask = __ballot_sync(0xffffffffu, valid && (vfar || far || mid));
        const unsigned nearMask = __ballot_sync(0xffffffffu, valid && !vfar && !far && !mid);
        const unsigned gzMask = __ballot_sync(0xffffffffu, hasGz);
        if (fastMask) {
            const float xo = (float)(ox - H.ox), yo = (float)(oy - H.oy), zo = (float)(oz - H.oz);
            if (TMI) {
#pragma unroll 4
                for (int v = 0; v < nv; ++v) {
                    const float4 q = *reinterpret_cast<const float4*>(PV + v);
                    const float rx = q.x - xo, ry = q.y - yo, rz = q.z - zo;
                    const float d2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
                    dvp[v * NT] = d2 * rsqrtf(d2);
                }
                float tacc = 0.f;
                // Far facets only (no mid or near facet in this warp's view of the
                // patch): every edge's v = L / (d1 + d2) is below 3/8 and every
                // solid-angle ratio below 1/8 for tau >= 2, so both series run
                // without branches (independent chains the compiler can
                // interleave).  A warp that meets an argument outside those
                // ranges redoes the patch's TMI with the per-term fallbacks.
                bool exact = (midMask | nearMask) != 0u;
                if (!exact) {
                    bool bad = false;
                    float tsum = 0.f;
#pragma unroll 4
                    for (int e = 0; e < ne; ++e) {
                        const PatchEdgeA ea = EA[e];
                        const float v = __fdividef(ea.L, dvp[ea.lv1 * NT] + dvp[ea.lv2 * NT]);
                        bad |= !(v <= 0.375f);
                        tsum = fmaf(ea.mt, v * atanh_poly(v * v), tsum);
                    }
#pragma unroll 2
                    for (unsigned m = fastMask; m; m &= m - 1) {
                        const float4* F4 = reinterpret_cast<const float4*>(PF + (__ffs(m) - 1));
                        const float4 w0 = F4[0], w1 = F4[1], w2 = F4[2];  // corners, N | cf, mf2 | squared edges
                        const uint32_t c = __float_as_uint(w0.x);
                        const float da = dvp[(c & 0xff) * NT], db = dvp[((c >> 8) & 0xff) * NT],
                                    dc = dvp[(c >> 16) * NT];
                        const float da2 = da * da, db2 = db * db, dc2 = dc * dc;
                        const float sab = da2 + db2 - w2.x, sbc = db2 + dc2 - w2.y, sca = dc2 + da2 - w2.z;
                        const float den = fmaf(0.5f, fmaf(sab, dc, fmaf(sbc, da, sca * db)), da * db * dc);
                        const float num = w1.x - fmaf(xo, w0.y, fmaf(yo, w0.z, zo * w0.w));
                        const float t = __fdividef(num, den);
                        bad |= !(den > 0.f && fabsf(t) <= 0.125f);
                        tsum = fmaf(w1.y, t * atan_poly(t * t), tsum);
                    }
                    if (__any_sync(0xffffffffu, bad))
                        exact = true;
                    else
                        tacc = tsum;
                }
                if (exact) {
                    const unsigned excl = nearMask;
                    for (int e = 0; e < ne; ++e) {
                        const PatchEdgeA ea = EA[e];
                        const PatchEdgeB eb = EB[e];
                        const int lf1 = eb.users & 0xff, lf2 = eb.users >> 8;
                        const float m = ((excl >> lf1) & 1u ? 0.f : eb.mt1) +
                                        (lf2 != kNoFacet && !((excl >> lf2) & 1u) ? eb.mt2 : 0.f);
                        if (m != 0.f)
                            tacc = fmaf(m, atanh_half_lambda(ea.L, dvp[ea.lv1 * NT] + dvp[ea.lv2 * NT]), tacc);
                    }
                    for (unsigned m = fastMask; m; m &= m - 1) {
                        const float4* F4 = reinterpret_cast<const float4*>(PF + (__ffs(m) - 1));
                        const float4 w0 = F4[0], w1 = F4[1], w2 = F4[2];
                        const uint32_t c = __float_as_uint(w0.x);
                        const float da = dvp[(c & 0xff) * NT], db = dvp[((c >> 8) & 0xff) * NT],
                                    dc = dvp[(c >> 16) * NT];
                        const float da2 = da * da, db2 = db * db, dc2 = dc * dc;
                        // 2 x the dot products r_a.r_b, r_b.r_c, r_c.r_a from the distances and edge lengths
                        const float sab = da2 + db2 - w2.x, sbc = db2 + dc2 - w2.y, sca = dc2 + da2 - w2.z;
                        const float den = fmaf(0.5f, fmaf(sab, dc, fmaf(sbc, da, sca * db)), da * db * dc);
                        const float num = w1.x - fmaf(xo, w0.y, fmaf(yo, w0.z, zo * w0.w));
                        tacc = fmaf(w1.y, atan_half_omega(num, den), tacc);
                    }
                }
                tmi += tacc;
            }
            if (GZ) {
                float gacc = 0.f;
                // facets with a gz term (n_z != 0), by rule: 3-point beyond 4 tau,
                // 6-point beyond tau, 28-point in the mid field
#pragma unroll 2
                for (unsigned m = fastMask & gzMask & vfarMask; m; m &= m - 1) {
                    const float4* F4 = reinterpret_cast<const float4*>(PF + (__ffs(m) - 1));
                    const float4 w4 = F4[4], w5 = F4[5], w6 = F4[6];  // q3[0..8]
                    const float q[9] = {w4.x, w4.y, w4.z, w4.w, w5.x, w5.y, w5.z, w5.w, w6.x};
                    float acc = 0.f;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float px = q[3 * k] - xo, py = q[3 * k + 1] - yo, pz = q[3 * k + 2] - zo;
                        acc += rsqrtf(fmaf(px, px, fmaf(py, py, pz * pz)));
                    }
                    gacc = fmaf(F4[1].z * (1.f / 3.f), acc, gacc);
                }
#pragma unroll 2
                for (unsigned m = fastMask & gzMask & ~vfarMask & ~midMask; m; m &= m - 1) {
                    const float4* F4 = reinterpret_cast<const float4*>(PF + (__ffs(m) - 1));
                    float q[20];  // floats 24..43 of the record: q3[8], then q6[0..17], pad
#pragma unroll
                    for (int k = 0; k < 5; ++k) {
                        const float4 w = F4[6 + k];
                        q[4 * k] = w.x; q[4 * k + 1] = w.y; q[4 * k + 2] = w.z; q[4 * k + 3] = w.w;
                    }
                    float acc = 0.f;
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        const float px = q[1 + 3 * k] - xo, py = q[2 + 3 * k] - yo, pz = q[3 + 3 * k] - zo;
                        acc = fmaf(kDun6W[k], rsqrtf(fmaf(px, px, fmaf(py, py, pz * pz))), acc);
                    }
                    gacc = fmaf(F4[1].z, acc, gacc);
                }
                for (unsigned m = gzMask & midMask; m; m &= m - 1) {
                    // Radon's 7-point rule on the four midpoint sub-triangles
                    // (28 points), built from the patch-frame corners
                    const float4* F4 = reinterpret_cast<const float4*>(PF + (__ffs(m) - 1));
                    const uint32_t c = __float_as_uint(F4[0].x);
                    const float4 pa = *reinterpret_cast<const float4*>(PV + (c & 0xff));
                    const float4 pb = *reinterpret_cast<const float4*>(PV + ((c >> 8) & 0xff));
                    const float4 pc = *reinterpret_cast<const float4*>(PV + (c >> 16));
                    const float ax = pa.x - xo, ay = pa.y - yo, az = pa.z - zo;
                    const float bx = pb.x - pa.x, by = pb.y - pa.y, bz = pb.z - pa.z;
                    const float cx = pc.x - pa.x, cy = pc.y - pa.y, cz = pc.z - pa.z;
                    float acc = 0.f;
#pragma unroll 7
                    for (int k = 0; k < 28; ++k) {
                        const float u = kRadon4Bb[k], w = kRadon4Bc[k];
                        const float px = fmaf(u, bx, fmaf(w, cx, ax)), py = fmaf(u, by, fmaf(w, cy, ay)),
                                    pz = fmaf(u, bz, fmaf(w, cz, az));
                        acc = fmaf(kRadonW[k % 7], rsqrtf(fmaf(px, px, fmaf(py, py, pz * pz))), acc);
                    }
                    gacc = fmaf(F4[1].z * 0.25f, acc, gacc);
                }
                gz += gacc;
            }
        }
        // near facets: FP64 analytic in the facet's local frame
        double* slot = sm.nearSlot[warp];
        for (unsigned m = nearMask; m; m &= m - 1) {
            const int f = PF[__ffs(m) - 1].gfacet;
            __syncwarp();
            if (lane < NMC) slot[lane] = __ldg(mc + (size_t)lane * T + f);
            __syncwarp();
            double g1 = 0.0, t1 = 0.0;
            pair_near_f64(slot, 0, 1, mk3(ox, oy, oz), &g1, &t1);
            if (GZ) gz += g1;
            if (TMI) tmi += t1;
        }
        nearCount += __popc(nearMask);
    }
    if (act) {
        if (GZ) out_gz[s] = gz;
        if (TMI) out_tmi[s] = tmi;
        if (near_pairs && nearCount) atomicAdd(near_pairs, nearCount);
    }
    return true;
}

template <int NT>
__device__ __forceinline__ PatchSmem<NT>& patch_smem_init() {
    extern __shared__ __align__(128) unsigned char patch_dyn_smem[];
    PatchSmem<NT>& sm = *reinterpret_cast<PatchSmem<NT>*>(patch_dyn_smem);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(patch_smem_addr(&sm.mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(patch_smem_addr(&sm.mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    return sm;
}

// Station blocks of NT stations (blockIdx.x) x patch chunks (blockIdx.y).
template <bool GZ, bool TMI, int NT>
__global__ void __launch_bounds__(NT) k_forward_patch(int S, const double* __restrict__ sta,
                                                      const unsigned char* __restrict__ blobs,
                                                      const int32_t* __restrict__ blobOff,
                                                      const int32_t* __restrict__ chunk_begin,
                                                      const int32_t* __restrict__ chunk_end,
                                                      const double* __restrict__ mc, int T, float tau,
                                                      double* __restrict__ part_gz, double* __restrict__ part_tmi,
                                                      unsigned long long* __restrict__ near_pairs,
                                                      unsigned int* __restrict__ err) {
    PatchSmem<NT>& sm = patch_smem_init<NT>();
    uint32_t phases = 0;
    const int s = blockIdx.x * NT + threadIdx.x;
    const int chunk = blockIdx.y;
    forward_patch_block<GZ, TMI, NT>(sm, s, s < S, sta, blobs, blobOff, chunk_begin[chunk], chunk_end[chunk], mc,
                                     T, tau, GZ ? part_gz + (size_t)chunk * S : nullptr,
                                     TMI ? part_tmi + (size_t)chunk * S : nullptr, near_pairs, err, phases);
}

// Persistent grid (one CTA per resident slot): the (station block, patch)
// units b * P + p, block-major over `nunits` = blocks x P, are split into
// gridDim.x balanced contiguous ranges; a CTA walks its range block by block,
// so each of its blocks is one pipelined patch run.  Block b's partial of CTA
// c goes to slot c - (the CTA holding unit b * P); k_forward_reduce_mixed
// sums block_nch[b] slots for the stations of block b.
__device__ __forceinline__ int patch_unit_owner(long long u, long long nunits, int G) {
    return static_cast<int>(((u + 1) * G - 1) / nunits);
}

template <bool GZ, bool TMI, int NT>
__global__ void __launch_bounds__(NT) k_forward_patch_persistent(int S, const double* __restrict__ sta,
                                                                 const unsigned char* __restrict__ blobs,
                                                                 const int32_t* __restrict__ blobOff, int pbase, int P,
                                                                 long long nunits, const double* __restrict__ mc,
                                                                 int T, float tau, double* __restrict__ part_gz,
                                                                 double* __restrict__ part_tmi,
                                                                 unsigned long long* __restrict__ near_pairs,
                                                                 unsigned int* __restrict__ err) {
    PatchSmem<NT>& sm = patch_smem_init<NT>();
    uint32_t phases = 0;
    const int G = gridDim.x, c = blockIdx.x;
    const long long u0 = (long long)c * nunits / G, u1 = (long long)(c + 1) * nunits / G;
    if (u0 >= u1) return;
    const int b0 = static_cast<int>(u0 / P), b1 = static_cast<int>((u1 - 1) / P);
    for (int b = b0; b <= b1; ++b) {
        const int pb = b == b0 ? static_cast<int>(u0 % P) : 0;
        const int pe = b == b1 ? static_cast<int>((u1 - 1) % P) + 1 : P;
        const int slot = c - patch_unit_owner((long long)b * P, nunits, G);
        const int s = b * NT + (int)threadIdx.x;
        if (!forward_patch_block<GZ, TMI, NT>(sm, s, s < S, sta, blobs, blobOff, pbase + pb, pbase + pe, mc, T, tau,
                                              GZ ? part_gz + (size_t)slot * S : nullptr,
                                              TMI ? part_tmi + (size_t)slot * S : nullptr, near_pairs, err, phases))
            return;
        __syncthreads();  // the next block's first copy reuses buffer 0
    }
}

// Batched bodies: a persistent grid over (body, station block, patch range)
// items; FwdItem's facet range holds the patch range.
template <bool GZ, bool TMI, int NT>
__global__ void __launch_bounds__(NT) k_forward_patch_items(const FwdItem* __restrict__ items, int nitems,
                                                            const double* __restrict__ sta,
                                                            const unsigned char* __restrict__ blobs,
                                                            const int32_t* __restrict__ blobOff,
                                                            const double* __restrict__ mc, int T, float tau,
                                                            double* __restrict__ part_gz,
                                                            double* __restrict__ part_tmi,
                                                            unsigned long long* __restrict__ near_pairs,
                                                            unsigned int* __restrict__ err) {
    PatchSmem<NT>& sm = patch_smem_init<NT>();
    uint32_t phases = 0;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const FwdItem w = items[it];
        const int s = w.s0 + (int)threadIdx.x;
        if (!forward_patch_block<GZ, TMI, NT>(sm, s, s < w.s_end, sta, blobs, blobOff, w.fb, w.fe, mc, T,
                                              tau, GZ ? part_gz + w.out : nullptr, TMI ? part_tmi + w.out : nullptr,
                                              near_pairs, err, phases))
            return;  // a copy did not land (block-uniform): leave the remaining items untouched
        __syncthreads();  // the next item's first copy reuses buffer 0
    }
}

}  // namespace litho_b200
