/*
 * litho_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded FP64 restatement of LithoInv's forward /
 * Jacobian / parameter-scatter path.  It is the checker that the CUDA
 * implementation is compared against; nothing in the product library links,
 * loads or calls it.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may use it.
 *
 * Parity of this restatement is pinned against the reference's own C++
 * sources compiled unmodified (oracle/Makefile -> oracle/_ref/) by
 * tests/test_oracle_pin.py, and against the committed golden vectors in
 * tests/golden/.
 *
 * Every function cites the reference function it restates (paths are
 * relative to the reference project root).  The arithmetic is written in the
 * same operation order as the reference so that, compiled without FMA
 * contraction, results agree with the reference to the last bit or close.
 *
 * Data layout shared by every model-level function (row-major, int32 indices):
 *   pos[V*3]            vertex positions (metres), one slot per (mesh, vertex)
 *   tri[T*3]            triangles as global vertex indices, grouped by lithology
 *   grp_tri_off[G+1]    triangles of group g are tri[grp_tri_off[g] .. grp_tri_off[g+1])
 *   sta[S*3]            observation stations
 *   dof_off[np+1]       global DOF d owns refs dof_off[d] .. dof_off[d+1]
 *   ref_vertex/axis/scale  per ref: global vertex, axis (0,1,2), axis scale
 *   interp_off[V+1], interp_src, interp_w   control-point interpolation rows
 *   sync_off[ns+1], sync_vertex             shared-vertex averaging groups
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define LO_EPS 1e-15
#define LO_PI 3.14159265358979323846

/* gravity_forward.h:37-41 */
#define LO_G_SI 6.67430e-11
#define LO_DENSITY_SCALE 1000.0
#define LO_M_S2_TO_MGAL 1e5

typedef struct { double x, y, z; } v3;

static inline v3 mk(const double *p) { v3 r = {p[0], p[1], p[2]}; return r; }
static inline v3 sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline v3 add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline v3 scl(v3 a, double s) { v3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static inline v3 dvs(v3 a, double s) { v3 r = {a.x / s, a.y / s, a.z / s}; return r; }
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline double norm(v3 a) { return sqrt(dot(a, a)); }
static inline double comp(v3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
static inline void setc(v3 *a, int k, double v) {
    if (k == 0) a->x = v; else if (k == 1) a->y = v; else a->z = v;
}

/* ------------------------------------------------------------------------ */
/* Geometry primitives: modules/litho-core/src/core/geometry.cpp            */
/* ------------------------------------------------------------------------ */

/* solidAngle, geometry.cpp:10-30 (van Oosterom & Strackee). */
static double solid_angle(v3 a, v3 b, v3 c, v3 o) {
    v3 ra = sub(a, o), rb = sub(b, o), rc = sub(c, o);
    double la = norm(ra), lb = norm(rb), lc = norm(rc);
    if (la < LO_EPS || lb < LO_EPS || lc < LO_EPS) return 0.0;
    /* tripleProduct(a,b,c) = a.dot(b.cross(c)), core/geometry.h:7-9 */
    double num = dot(ra, cross(rb, rc));
    double den = la * lb * lc + dot(ra, rb) * lc + dot(ra, rc) * lb + dot(rb, rc) * la;
    return 2.0 * atan2(num, den);
}

/* lineIntegralTerm, geometry.cpp:32-52. */
static double line_integral_term(v3 a, v3 b, v3 o) {
    v3 ra = sub(a, o), rb = sub(b, o), e = sub(b, a);
    double L = norm(e);
    if (L < LO_EPS) return 0.0;
    double s1 = dot(ra, e) / L;
    double s2 = dot(rb, e) / L;
    double d1 = norm(ra), d2 = norm(rb);
    double num = s2 + d2, den = s1 + d1;
    if (fabs(den) < LO_EPS && fabs(num) < LO_EPS) return 0.0;
    if (fabs(den) < LO_EPS) return 0.0;
    if (num <= 0.0 || den <= 0.0) return 0.0;
    return log(num / den);
}

/* faceNagyContribution, modules/litho-forward/src/forward/gravity_forward.cpp:13-42.
 * Returns n_z * (sum_i d_perp_i * Lambda_i - h * Omega). */
static double face_nagy(v3 obs, v3 a, v3 b, v3 c) {
    v3 n = cross(sub(b, a), sub(c, a));
    double area_x2 = norm(n);
    if (area_x2 < LO_EPS) return 0.0;
    v3 un = dvs(n, area_x2);
    double nz = un.z;
    double omega = solid_angle(a, b, c, obs);
    double h = dot(sub(a, obs), un);
    double d_sum = 0.0;
    v3 vs[3] = {a, b, c};
    for (int i = 0; i < 3; ++i) {
        v3 p1 = vs[i], p2 = vs[(i + 1) % 3];
        v3 e = sub(p2, p1);
        double L = norm(e);
        if (L < LO_EPS) continue;
        v3 eh = dvs(e, L);
        v3 perp = cross(un, eh);
        double dperp = dot(sub(obs, p1), perp);
        double lam = line_integral_term(p1, p2, obs);
        d_sum += dperp * lam;
    }
    return nz * (d_sum - h * omega);
}

/* MagneticForward::magneticFacet, modules/litho-forward/src/forward/magnetic_forward.cpp:312-347. */
static double magnetic_facet(v3 obs, v3 a, v3 b, v3 c, v3 mdir, v3 fdir) {
    v3 n = cross(sub(b, a), sub(c, a));
    double area_x2 = norm(n);
    if (area_x2 < LO_EPS) return 0.0;
    v3 nh = dvs(n, area_x2);
    double omega = solid_angle(a, b, c, obs);
    double mn = dot(mdir, nh), fn = dot(fdir, nh);
    double contribution = mn * fn * omega;
    v3 vs[3] = {a, b, c};
    for (int i = 0; i < 3; ++i) {
        v3 p1 = vs[i], p2 = vs[(i + 1) % 3];
        v3 e = sub(p2, p1);
        double L = norm(e);
        if (L < LO_EPS) continue;
        v3 eh = dvs(e, L);
        v3 t = cross(nh, eh);
        double mt = dot(mdir, t), ft = dot(fdir, t);
        double lam = line_integral_term(p1, p2, obs);
        contribution += mt * ft * lam;
    }
    return contribution;
}

/* Face evaluation selector used by the per-face finite-difference gradient. */
typedef struct { int kind; v3 mdir, fdir; } facefn;

static double face_eval(const facefn *f, v3 obs, v3 a, v3 b, v3 c) {
    return f->kind == 0 ? face_nagy(obs, a, b, c) : magnetic_facet(obs, a, b, c, f->mdir, f->fdir);
}

/* faceNagyWithGradient, gravity_forward.cpp:48-85, and
 * magneticFacetWithGradient, magnetic_forward.cpp:14-50: value plus forward
 * differences with h = 1e-4 m on each of the 9 vertex coordinates. */
static void face_with_fd_gradient(const facefn *f, v3 obs, v3 a, v3 b, v3 c,
                                  double *value, v3 *ga, v3 *gb, v3 *gc) {
    const double h = 1e-4;
    double v = face_eval(f, obs, a, b, c);
    *value = v;
    for (int k = 0; k < 3; ++k) {
        v3 p = a; setc(&p, k, comp(a, k) + h);
        setc(ga, k, (face_eval(f, obs, p, b, c) - v) / h);
    }
    for (int k = 0; k < 3; ++k) {
        v3 p = b; setc(&p, k, comp(b, k) + h);
        setc(gb, k, (face_eval(f, obs, a, p, c) - v) / h);
    }
    for (int k = 0; k < 3; ++k) {
        v3 p = c; setc(&p, k, comp(c, k) + h);
        setc(gc, k, (face_eval(f, obs, a, b, p) - v) / h);
    }
}

/* The x and y derivatives of the finite-difference-XY gradient mode (no
 * reference counterpart; its step is a parameter, h = 0.5 m in the
 * large-inversion configuration): forward differences of the reference's
 * facet formula as in face_with_fd_gradient, written into the x and y slots
 * of ga, gb, gc. */
static void face_xy_forward_difference(const facefn *f, v3 obs, v3 a, v3 b, v3 c, double h, v3 *ga, v3 *gb,
                                       v3 *gc) {
    double v = face_eval(f, obs, a, b, c);
    for (int k = 0; k < 2; ++k) {
        v3 p = a; setc(&p, k, comp(a, k) + h);
        setc(ga, k, (face_eval(f, obs, p, b, c) - v) / h);
        p = b; setc(&p, k, comp(b, k) + h);
        setc(gb, k, (face_eval(f, obs, a, p, c) - v) / h);
        p = c; setc(&p, k, comp(c, k) + h);
        setc(gc, k, (face_eval(f, obs, a, b, p) - v) / h);
    }
}

/* ------------------------------------------------------------------------ */
/* The "true derivative" (NOT part of the reference; the analytic device   */
/* gradient is checked against it): a central difference with one           */
/* Richardson step (error O(h^4)) of the same facet formulas evaluated in   */
/* x87 extended precision (64-bit significand).  The reference's oriented   */
/* line-integral form loses digits for edges nearly collinear with the      */
/* station, and a central difference divides that rounding by h; with 11    */
/* more bits the step can follow the facet's own scale (see lo_jacobian)    */
/* instead of being held large to keep the rounding down.                   */
/* ------------------------------------------------------------------------ */
typedef long double ld;
typedef struct { ld x, y, z; } l3;

static inline l3 lmk(v3 a) { l3 r = {a.x, a.y, a.z}; return r; }
static inline l3 lsub(l3 a, l3 b) { l3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline l3 ldvs(l3 a, ld s) { l3 r = {a.x / s, a.y / s, a.z / s}; return r; }
static inline ld ldot(l3 a, l3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline l3 lcross(l3 a, l3 b) {
    l3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline ld lnorm(l3 a) { return sqrtl(ldot(a, a)); }

static ld l_solid_angle(l3 a, l3 b, l3 c, l3 o) {
    l3 ra = lsub(a, o), rb = lsub(b, o), rc = lsub(c, o);
    ld la = lnorm(ra), lb = lnorm(rb), lc = lnorm(rc);
    if (la < LO_EPS || lb < LO_EPS || lc < LO_EPS) return 0.0L;
    ld num = ldot(ra, lcross(rb, rc));
    ld den = la * lb * lc + ldot(ra, rb) * lc + ldot(ra, rc) * lb + ldot(rb, rc) * la;
    return 2.0L * atan2l(num, den);
}

static ld l_line_integral_term(l3 a, l3 b, l3 o) {
    l3 ra = lsub(a, o), rb = lsub(b, o), e = lsub(b, a);
    ld L = lnorm(e);
    if (L < LO_EPS) return 0.0L;
    ld s1 = ldot(ra, e) / L, s2 = ldot(rb, e) / L;
    ld d1 = lnorm(ra), d2 = lnorm(rb);
    ld num = s2 + d2, den = s1 + d1;
    if (fabsl(den) < LO_EPS) return 0.0L;
    if (num <= 0.0L || den <= 0.0L) return 0.0L;
    return logl(num / den);
}

/* face_nagy / magnetic_facet above, term for term. */
static ld l_face_eval(const facefn *f, l3 obs, l3 a, l3 b, l3 c) {
    l3 n = lcross(lsub(b, a), lsub(c, a));
    ld area_x2 = lnorm(n);
    if (area_x2 < LO_EPS) return 0.0L;
    l3 un = ldvs(n, area_x2);
    ld omega = l_solid_angle(a, b, c, obs);
    l3 md = lmk(f->mdir), fd = lmk(f->fdir);
    ld acc = f->kind == 0 ? -ldot(lsub(a, obs), un) * omega : ldot(md, un) * ldot(fd, un) * omega;
    l3 vs[3] = {a, b, c};
    for (int i = 0; i < 3; ++i) {
        l3 p1 = vs[i], p2 = vs[(i + 1) % 3];
        l3 e = lsub(p2, p1);
        ld L = lnorm(e);
        if (L < LO_EPS) continue;
        l3 perp = lcross(un, ldvs(e, L));
        ld lam = l_line_integral_term(p1, p2, obs);
        acc += (f->kind == 0 ? ldot(lsub(obs, p1), perp) : ldot(md, perp) * ldot(fd, perp)) * lam;
    }
    return f->kind == 0 ? un.z * acc : acc;
}

static ld lcomp(l3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
static void lsetc(l3 *a, int k, ld v) {
    if (k == 0) a->x = v; else if (k == 1) a->y = v; else a->z = v;
}

static ld face_central(const facefn *f, l3 obs, l3 a, l3 b, l3 c, int which, int k, ld h) {
    l3 vp[3] = {a, b, c}, vm[3] = {a, b, c};
    lsetc(&vp[which], k, lcomp(vp[which], k) + h);
    lsetc(&vm[which], k, lcomp(vm[which], k) - h);
    ld fp = l_face_eval(f, obs, vp[0], vp[1], vp[2]);
    ld fm = l_face_eval(f, obs, vm[0], vm[1], vm[2]);
    return (fp - fm) / (2.0L * h);
}

/* Distance from o to the triangle abc (closest point by the Voronoi regions
 * of the vertices, edges and face: Ericson, Real-Time Collision Detection,
 * sec. 5.1.5).  Sizes the adaptive step of the true derivative. */
static double point_triangle_distance(v3 o, v3 a, v3 b, v3 c) {
    v3 ab = sub(b, a), ac = sub(c, a), ap = sub(o, a);
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return norm(ap);
    v3 bp = sub(o, b);
    double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) return norm(bp);
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return norm(sub(ap, scl(ab, d1 / (d1 - d3))));
    v3 cp = sub(o, c);
    double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) return norm(cp);
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return norm(sub(ap, scl(ac, d2 / (d2 - d6))));
    double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return norm(sub(bp, scl(sub(c, b), w)));
    }
    double den = va + vb + vc;
    if (!(fabs(den) > 0.0)) return norm(ap); /* degenerate triangle */
    double v = vb / den, w = vc / den;
    return norm(sub(ap, add(scl(ab, v), scl(ac, w))));
}

static void face_true_gradient(const facefn *f, v3 obs, v3 a, v3 b, v3 c, double h,
                               v3 *ga, v3 *gb, v3 *gc) {
    v3 *out[3] = {ga, gb, gc};
    l3 lo = lmk(obs), la = lmk(a), lb = lmk(b), lc = lmk(c);
    for (int w = 0; w < 3; ++w)
        for (int k = 0; k < 3; ++k) {
            ld d1 = face_central(f, lo, la, lb, lc, w, k, h);
            ld d2 = face_central(f, lo, la, lb, lc, w, k, 0.5L * h);
            setc(out[w], k, (double)((4.0L * d2 - d1) / 3.0L));
        }
}

/* Smallest altitude of the triangle abc (twice-area / longest edge): the
 * scale on which its unit normal, and with it the facet term, turns. */
static double min_altitude(v3 a, v3 b, v3 c) {
    double lm = fmax(norm(sub(b, a)), fmax(norm(sub(c, b)), norm(sub(a, c))));
    return lm > 0.0 ? norm(cross(sub(b, a), sub(c, a))) / lm : 0.0;
}

/* A facet collapsed onto a line (twice-area < 1e-10 * longest edge^2): its
 * facet term has a kink (the unit normal flips with the side it opens to), the
 * central difference there is zero, and the truth takes it as zero. */
static int collapsed(v3 a, v3 b, v3 c) {
    double l0 = norm(sub(b, a)), l1 = norm(sub(c, b)), l2 = norm(sub(a, c));
    double lm = fmax(l0, fmax(l1, l2));
    return norm(cross(sub(b, a), sub(c, a))) < 1e-10 * lm * lm;
}

/* ------------------------------------------------------------------------ */
/* Exported primitives (for pinning and golden vectors)                     */
/* ------------------------------------------------------------------------ */

double lo_solid_angle(const double *a, const double *b, const double *c, const double *o) {
    return solid_angle(mk(a), mk(b), mk(c), mk(o));
}
double lo_line_integral_term(const double *a, const double *b, const double *o) {
    return line_integral_term(mk(a), mk(b), mk(o));
}
double lo_face_nagy(const double *o, const double *a, const double *b, const double *c) {
    return face_nagy(mk(o), mk(a), mk(b), mk(c));
}
double lo_magnetic_facet(const double *o, const double *a, const double *b, const double *c,
                         const double *mdir, const double *fdir) {
    return magnetic_facet(mk(o), mk(a), mk(b), mk(c), mk(mdir), mk(fdir));
}
/* grad9 = (ga, gb, gc) as 9 doubles; kind 0 = gravity face, 1 = magnetic facet */
double lo_face_fd_gradient(int kind, const double *o, const double *a, const double *b,
                           const double *c, const double *mdir, const double *fdir, double *grad9) {
    facefn f; f.kind = kind;
    if (kind) { f.mdir = mk(mdir); f.fdir = mk(fdir); }
    double v; v3 ga, gb, gc;
    face_with_fd_gradient(&f, mk(o), mk(a), mk(b), mk(c), &v, &ga, &gb, &gc);
    double g[9] = {ga.x, ga.y, ga.z, gb.x, gb.y, gb.z, gc.x, gc.y, gc.z};
    memcpy(grad9, g, sizeof g);
    return v;
}
void lo_face_true_gradient(int kind, const double *o, const double *a, const double *b,
                           const double *c, const double *mdir, const double *fdir, double h,
                           double *grad9) {
    facefn f; f.kind = kind;
    if (kind) { f.mdir = mk(mdir); f.fdir = mk(fdir); }
    v3 ga, gb, gc;
    face_true_gradient(&f, mk(o), mk(a), mk(b), mk(c), h, &ga, &gb, &gc);
    double g[9] = {ga.x, ga.y, ga.z, gb.x, gb.y, gb.z, gc.x, gc.y, gc.z};
    memcpy(grad9, g, sizeof g);
}

/* ------------------------------------------------------------------------ */
/* Magnetization: MagneticForward ctor magnetic_forward.cpp:57-67 and       */
/* buildGroupMagnetization :100-134                                          */
/* ------------------------------------------------------------------------ */

/* Field unit vector (cosI cosD, cosI sinD, -sinI). */
void lo_field_unit_vector(double inc_deg, double dec_deg, double *out3) {
    double I = inc_deg * LO_PI / 180.0, D = dec_deg * LO_PI / 180.0;
    double cI = cos(I);
    out3[0] = cI * cos(D);
    out3[1] = cI * sin(D);
    out3[2] = -sin(I);
}

/* mode 0 = EffectiveSusceptibility, 1 = FixedVectorPerGroup, 2 = VectorPerGroup. */
void lo_group_magnetization(double susceptibility, double field_nT, const double *fdir, int mode,
                            double rem_mag, double rem_inc, double rem_dec, const double *rem_vec,
                            double *amp, double *dir3) {
    v3 F = mk(fdir);
    double induced = susceptibility * field_nT / 100.0;
    v3 M = scl(F, induced);
    if (mode == 1) {
        double I = rem_inc * LO_PI / 180.0, D = rem_dec * LO_PI / 180.0;
        double cI = cos(I);
        v3 R = {cI * cos(D), cI * sin(D), -sin(I)};
        M = add(M, scl(R, rem_mag));
    } else if (mode == 2) {
        M = add(M, mk(rem_vec));
    }
    double a = norm(M);
    *amp = a;
    v3 d = (a < LO_EPS) ? F : dvs(M, a);
    dir3[0] = d.x; dir3[1] = d.y; dir3[2] = d.z;
}

/* ------------------------------------------------------------------------ */
/* Parameter scatter: LithologyModel::applyParameterVector                 */
/* modules/litho-model/src/litho/lithology_model.cpp:210-248, with          */
/* SurfaceMesh::interpolateFromControlPoints surface_mesh.cpp:610-623.      */
/* ------------------------------------------------------------------------ */
void lo_scatter(int np, const double *params, const int32_t *dof_off, const int32_t *ref_vertex,
                const uint8_t *ref_axis, const double *ref_scale, int V, const int32_t *interp_off,
                const int32_t *interp_src, const double *interp_w, int ns, const int32_t *sync_off,
                const int32_t *sync_vertex, double *pos) {
    /* 1. each global DOF writes every (mesh, local DOF) it controls */
    for (int d = 0; d < np; ++d) {
        double val = params[d];
        for (int r = dof_off[d]; r < dof_off[d + 1]; ++r)
            pos[3 * ref_vertex[r] + ref_axis[r]] = val * ref_scale[r];
    }
    /* 2. non-control-point vertices of CP meshes = sum w * CP position.
     * Rows only read control-point vertices, which are never rows. */
    if (interp_off) {
        for (int v = 0; v < V; ++v) {
            int b = interp_off[v], e = interp_off[v + 1];
            if (b == e) continue;
            v3 p = {0.0, 0.0, 0.0};
            for (int k = b; k < e; ++k) p = add(p, scl(mk(pos + 3 * interp_src[k]), interp_w[k]));
            pos[3 * v] = p.x; pos[3 * v + 1] = p.y; pos[3 * v + 2] = p.z;
        }
    }
    /* 3. shared-vertex averaging groups (lithology_model.cpp:235-247) */
    for (int s = 0; s < ns; ++s) {
        int b = sync_off[s], e = sync_off[s + 1];
        if (e - b < 2) continue;
        v3 avg = {0.0, 0.0, 0.0};
        for (int k = b; k < e; ++k) avg = add(avg, mk(pos + 3 * sync_vertex[k]));
        avg = dvs(avg, (double)(e - b));
        for (int k = b; k < e; ++k) {
            pos[3 * sync_vertex[k]] = avg.x;
            pos[3 * sync_vertex[k] + 1] = avg.y;
            pos[3 * sync_vertex[k] + 2] = avg.z;
        }
    }
}

/* Adjoint of lo_scatter (no reference counterpart: the reference gathers   */
/* vertex derivatives at the DOF vertices only, gravity_forward.cpp:270-289 */
/* and magnetic_forward.cpp's copy of it).  Maps a gradient with respect to */
/* the scattered positions, vg[3V], to the parameters: the three steps of   */
/* lo_scatter transposed in reverse order.  vg is overwritten (scratch).    */
/*  3'. averaging: every member of a group of >= 2 receives the mean of the  */
/*      group's gradients (the averaging matrix is symmetric);              */
/*  2'. interpolation: a row's gradient moves to its sources with the row's  */
/*      weights, and the row keeps none (its position is overwritten);      */
/*  1'. DOF writes: grad[d] = sum over d's slots of scale x vg[slot].        */
/* ------------------------------------------------------------------------ */
void lo_chain_gather(int V, double *vg, int np, const int32_t *dof_off, const int32_t *ref_vertex,
                     const uint8_t *ref_axis, const double *ref_scale, const int32_t *interp_off,
                     const int32_t *interp_src, const double *interp_w, int ns, const int32_t *sync_off,
                     const int32_t *sync_vertex, double *grad) {
    for (int s = 0; s < ns; ++s) {
        int b = sync_off[s], e = sync_off[s + 1];
        if (e - b < 2) continue;
        v3 sum = {0.0, 0.0, 0.0};
        for (int k = b; k < e; ++k) sum = add(sum, mk(vg + 3 * sync_vertex[k]));
        sum = dvs(sum, (double)(e - b));
        for (int k = b; k < e; ++k) {
            vg[3 * sync_vertex[k]] = sum.x;
            vg[3 * sync_vertex[k] + 1] = sum.y;
            vg[3 * sync_vertex[k] + 2] = sum.z;
        }
    }
    if (interp_off) {
        for (int v = 0; v < V; ++v) {
            int b = interp_off[v], e = interp_off[v + 1];
            if (b == e) continue;
            v3 g = mk(vg + 3 * v);
            for (int k = b; k < e; ++k) {
                double *q = vg + 3 * interp_src[k];
                q[0] += interp_w[k] * g.x;
                q[1] += interp_w[k] * g.y;
                q[2] += interp_w[k] * g.z;
            }
            vg[3 * v] = vg[3 * v + 1] = vg[3 * v + 2] = 0.0;
        }
    }
    for (int d = 0; d < np; ++d) {
        double acc = 0.0;
        for (int r = dof_off[d]; r < dof_off[d + 1]; ++r) acc += ref_scale[r] * vg[3 * ref_vertex[r] + ref_axis[r]];
        grad[d] = acc;
    }
}

/* ------------------------------------------------------------------------ */
/* Forward: GravityForward::compute gravity_forward.cpp:105-118 ->          */
/* computeUnitGravity :124-130 -> gravityClosedMesh :162-178.                */
/* ------------------------------------------------------------------------ */
void lo_forward_gz(int S, const double *sta, int G, const int32_t *grp_tri_off,
                   const int32_t *tri, const double *pos, const double *rho, double *gz) {
    for (int s = 0; s < S; ++s) {
        v3 o = mk(sta + 3 * s);
        double acc = 0.0;
        for (int g = 0; g < G; ++g) {
            if (grp_tri_off[g + 1] == grp_tri_off[g]) continue;
            double total = 0.0;
            for (int t = grp_tri_off[g]; t < grp_tri_off[g + 1]; ++t)
                total += face_nagy(o, mk(pos + 3 * tri[3 * t]), mk(pos + 3 * tri[3 * t + 1]),
                                   mk(pos + 3 * tri[3 * t + 2]));
            double scale = LO_G_SI * rho[g] * LO_DENSITY_SCALE * LO_M_S2_TO_MGAL;
            acc += total * scale;
        }
        gz[s] = acc;
    }
}

/* MagneticForward::compute magnetic_forward.cpp:81-94 -> computeUnitMagnetic
 * :136-146 -> magneticClosedMeshVector :367-386. */
void lo_forward_tmi(int S, const double *sta, int G, const int32_t *grp_tri_off,
                    const int32_t *tri, const double *pos, const double *mag_amp,
                    const double *mag_dir, const double *fdir, double *tmi) {
    v3 F = mk(fdir);
    for (int s = 0; s < S; ++s) {
        v3 o = mk(sta + 3 * s);
        double acc = 0.0;
        for (int g = 0; g < G; ++g) {
            if (grp_tri_off[g + 1] == grp_tri_off[g]) continue;
            v3 m = mk(mag_dir + 3 * g);
            double gf = 0.0;
            for (int t = grp_tri_off[g]; t < grp_tri_off[g + 1]; ++t)
                gf += magnetic_facet(o, mk(pos + 3 * tri[3 * t]), mk(pos + 3 * tri[3 * t + 1]),
                                     mk(pos + 3 * tri[3 * t + 2]), m, F);
            double scale = mag_amp[g] * 100.0 / (4.0 * LO_PI);
            acc += -scale * gf;
        }
        tmi[s] = acc;
    }
}

/* ------------------------------------------------------------------------ */
/* Dense Jacobian with the reference's semantics:                           */
/* computeGravityAnalyticJacobian gravity_forward.cpp:184-292 and           */
/* computeMagneticAnalyticJacobian magnetic_forward.cpp:196-306.            */
/*  - per (station, face): forward-FD gradient, h = 1e-4 (kind < 2) or the  */
/*    Richardson central "true" derivative (kind >= 2, test truth only;     */
/*    step true_h, or -true_h x min(station-triangle distance, smallest    */
/*    altitude) if < 0; extended precision); kind 4 / 5: z the truth with  */
/*    step -3e-3, x and y forward differences with step true_h (the        */
/*    finite-difference-XY mode of the device gradient);                   */
/*  - vertex gradients accumulated per mesh with faceScale;                 */
/*  - gather: J(i, dof) += vg[vertex][axis] * axisScale for each ref,       */
/*    skipping |vg| < 1e-30 (reference semantics, kind < 2 only).           */
/* J is row-major S x np.  `kind`: 0 gravity-FD, 1 magnetic-FD,             */
/* 2 gravity-true, 3 magnetic-true.                                          */
/* ------------------------------------------------------------------------ */
void lo_jacobian(int kind, int S, const double *sta, int G, const int32_t *grp_tri_off,
                 const int32_t *tri, int V, const double *pos, const double *rho,
                 const double *mag_amp, const double *mag_dir, const double *fdir, int np,
                 const int32_t *dof_off, const int32_t *ref_vertex, const uint8_t *ref_axis,
                 const double *ref_scale, double true_h, double *J) {
    int mag = kind & 1, truth = kind >= 2, fdxy = kind >= 4;
    double *vg = (double *)calloc((size_t)V * 3, sizeof(double));
    const double gscale = LO_G_SI * LO_DENSITY_SCALE * LO_M_S2_TO_MGAL;
    const double kInv4Pi = 1.0 / (4.0 * LO_PI);
    facefn f; f.kind = mag;
    if (mag) f.fdir = mk(fdir);
    for (int s = 0; s < S; ++s) {
        v3 o = mk(sta + 3 * s);
        memset(vg, 0, sizeof(double) * (size_t)V * 3);
        for (int g = 0; g < G; ++g) {
            if (grp_tri_off[g + 1] == grp_tri_off[g]) continue;
            double faceScale;
            if (mag) {
                if (mag_amp[g] < LO_EPS) continue;
                faceScale = -mag_amp[g] * 100.0 * kInv4Pi;
                f.mdir = mk(mag_dir + 3 * g);
            } else {
                faceScale = gscale * rho[g];
            }
            for (int t = grp_tri_off[g]; t < grp_tri_off[g + 1]; ++t) {
                int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
                v3 ga = {0, 0, 0}, gb = {0, 0, 0}, gc = {0, 0, 0};
                double val;
                if (truth && collapsed(mk(pos + 3 * ia), mk(pos + 3 * ib), mk(pos + 3 * ic))) continue;
                if (truth) {
                    /* true_h > 0: that step; true_h < 0: |true_h| x the
                     * smaller of the station-triangle distance and the
                     * triangle's smallest altitude (floor 1e-9 m), the two
                     * scales of the facet term, so that the O(h^4)
                     * truncation stays small for near, far and thin facets
                     * alike; the extended-precision evaluation keeps the
                     * 1/h rounding below it */
                    double h = fdxy ? -3e-3 : true_h;
                    if (h < 0.0) {
                        v3 pa = mk(pos + 3 * ia), pb = mk(pos + 3 * ib), pc = mk(pos + 3 * ic);
                        h = -h * fmin(point_triangle_distance(o, pa, pb, pc), min_altitude(pa, pb, pc));
                        if (h < 1e-9) h = 1e-9;
                    }
                    face_true_gradient(&f, o, mk(pos + 3 * ia), mk(pos + 3 * ib), mk(pos + 3 * ic), h, &ga,
                                       &gb, &gc);
                }
                else if (!truth)
                    face_with_fd_gradient(&f, o, mk(pos + 3 * ia), mk(pos + 3 * ib),
                                          mk(pos + 3 * ic), &val, &ga, &gb, &gc);
                if (fdxy) /* x and y of each vertex: forward difference with step true_h */
                    face_xy_forward_difference(&f, o, mk(pos + 3 * ia), mk(pos + 3 * ib), mk(pos + 3 * ic),
                                               true_h, &ga, &gb, &gc);
                int ids[3] = {ia, ib, ic};
                v3 gs[3] = {ga, gb, gc};
                for (int w = 0; w < 3; ++w) {
                    v3 c = scl(gs[w], faceScale);
                    vg[3 * ids[w]] += c.x;
                    vg[3 * ids[w] + 1] += c.y;
                    vg[3 * ids[w] + 2] += c.z;
                }
            }
        }
        double *row = J + (size_t)s * np;
        for (int d = 0; d < np; ++d) {
            double acc = 0.0;
            for (int r = dof_off[d]; r < dof_off[d + 1]; ++r) {
                double pg = vg[3 * ref_vertex[r] + ref_axis[r]];
                if (!truth && fabs(pg) < 1e-30) continue;
                acc += pg * ref_scale[r];
            }
            row[d] = acc;
        }
    }
    free(vg);
}

/* ------------------------------------------------------------------------ */
/* Objective: ObjectiveFunction modules/litho-inversion/src/inversion/      */
/* objective.cpp:22-55; w = 1/std if std > 0 else 1.                         */
/* ------------------------------------------------------------------------ */
double lo_misfit(int S, const double *pred, const double *obs, const double *std) {
    double m = 0.0;
    for (int i = 0; i < S; ++i) {
        double w = (std[i] > 0) ? (1.0 / std[i]) : 1.0;
        double res = w * (obs[i] - pred[i]);
        m += 0.5 * res * res;
    }
    return m;
}

/* dataMisfitGradient objective.cpp:42-55: -J^T (w^2 r); alpha scales the
 * result as JointObjective::gradient does for magnetics (joint_objective.cpp:46-58). */
void lo_misfit_gradient(int S, int np, const double *J, const double *pred, const double *obs,
                        const double *std, double alpha, double *grad_accum) {
    for (int i = 0; i < S; ++i) {
        double w = (std[i] > 0) ? (1.0 / std[i]) : 1.0;
        double wr = w * w * (obs[i] - pred[i]);
        const double *row = J + (size_t)i * np;
        for (int d = 0; d < np; ++d) grad_accum[d] += -alpha * row[d] * wr;
    }
}

/* ------------------------------------------------------------------------
 * SurfaceSmoothness (modules/litho-regularization/src/regularization/
 * smoothness.cpp:20-105 evaluate, :107-390 gradient).
 *
 * Neighbours: SurfaceMesh::buildNeighbors (modules/litho-surface/src/surface/
 * surface_mesh.cpp:265-286) -- every other vertex of every triangle that
 * contains the vertex, sorted ascending, duplicates removed.  Only neighbours
 * with the vertex's own freedom count; FIXED vertices take no part.
 * penalty_v = 0.5 |mask_v(p_v - mean_v)|^2, mask_v = the vertex's free axes
 * (ALONG_VECTOR is not represented here).  Value = weight * sum_v penalty_v,
 * summed over vertices in order.  Gradient per vertex (the CP-stride branch,
 * :152-242; the plain branch :243-384 gives the same numbers for axis
 * freedoms): own term mask_v(diff_v), then, for every same-freedom neighbour
 * u in ascending order, -mask_u(diff_u) / n_u; gathered to DOFs as
 * weight * sum_refs vgrad[v][axis] * scale.
 * ------------------------------------------------------------------------ */
static int lo_cmp_i32(const void *a, const void *b) {
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* free axes of a VertexFreedom (surface_mesh.h:9-19) */
static void lo_axis_mask(int freedom, int m[3]) {
    m[0] = m[1] = m[2] = 0;
    switch (freedom) {
    case 1: m[2] = 1; break;            /* Z_ONLY */
    case 2: m[0] = 1; break;            /* X_ONLY */
    case 3: m[1] = 1; break;            /* Y_ONLY */
    case 5: m[0] = m[1] = 1; break;     /* XY_FREE */
    case 6: m[0] = m[2] = 1; break;     /* XZ_FREE */
    case 7: m[1] = m[2] = 1; break;     /* YZ_FREE */
    case 8: m[0] = m[1] = m[2] = 1; break; /* XYZ_FREE */
    default: break;
    }
}

/* Same-freedom neighbour CSR (caller frees *off and *nbr). */
static void lo_same_neighbours(int V, int T, const int32_t *tri, const uint8_t *freedom, int32_t **off_out,
                               int32_t **nbr_out) {
    int32_t *cnt = (int32_t *)calloc((size_t)V + 1, sizeof(int32_t));
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < 3; ++k) cnt[tri[3 * t + k] + 1] += 2;
    for (int v = 0; v < V; ++v) cnt[v + 1] += cnt[v];
    int32_t *raw = (int32_t *)malloc(sizeof(int32_t) * ((size_t)cnt[V] + 1));
    int32_t *fill = (int32_t *)malloc(sizeof(int32_t) * ((size_t)V + 1));
    memcpy(fill, cnt, sizeof(int32_t) * (size_t)V);
    for (int t = 0; t < T; ++t) {
        int32_t a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
        raw[fill[a]++] = b; raw[fill[a]++] = c;
        raw[fill[b]++] = a; raw[fill[b]++] = c;
        raw[fill[c]++] = a; raw[fill[c]++] = b;
    }
    int32_t *off = (int32_t *)calloc((size_t)V + 1, sizeof(int32_t));
    int32_t *nbr = (int32_t *)malloc(sizeof(int32_t) * ((size_t)cnt[V] + 1));
    int k = 0;
    for (int v = 0; v < V; ++v) {
        int32_t *l = raw + cnt[v];
        int n = cnt[v + 1] - cnt[v];
        qsort(l, (size_t)n, sizeof(int32_t), lo_cmp_i32);
        off[v] = k;
        if (freedom[v] != 0)
            for (int i = 0; i < n; ++i) {
                if (i > 0 && l[i] == l[i - 1]) continue;
                if (freedom[l[i]] == freedom[v]) nbr[k++] = l[i];
            }
    }
    off[V] = k;
    free(cnt); free(raw); free(fill);
    *off_out = off;
    *nbr_out = nbr;
}

/* Value (weight * penalty) and DOF gradient of the smoothness term at the
 * positions pos[V*3] (after the scatter).  Either output may be NULL. */
void lo_smoothness(int V, const double *pos, const uint8_t *freedom, int T, const int32_t *tri, double weight,
                   int np, const int32_t *dof_off, const int32_t *ref_vertex, const uint8_t *ref_axis,
                   const double *ref_scale, double *value, double *grad) {
    int32_t *off, *nbr;
    lo_same_neighbours(V, T, tri, freedom, &off, &nbr);
    double *diff = (double *)calloc((size_t)V * 3, sizeof(double));
    double *vg = (double *)calloc((size_t)V * 3, sizeof(double));
    double pen = 0.0;
    for (int v = 0; v < V; ++v) {
        int n = off[v + 1] - off[v];
        if (n == 0) continue;
        double mean[3] = {0.0, 0.0, 0.0};
        for (int i = off[v]; i < off[v + 1]; ++i)
            for (int k = 0; k < 3; ++k) mean[k] += pos[3 * nbr[i] + k];
        for (int k = 0; k < 3; ++k) mean[k] /= (double)n;
        for (int k = 0; k < 3; ++k) diff[3 * v + k] = pos[3 * v + k] - mean[k];
        double d0 = diff[3 * v], d1 = diff[3 * v + 1], d2 = diff[3 * v + 2];
        switch (freedom[v]) {
        case 1: pen += 0.5 * d2 * d2; break;
        case 2: pen += 0.5 * d0 * d0; break;
        case 3: pen += 0.5 * d1 * d1; break;
        case 5: pen += 0.5 * (d0 * d0 + d1 * d1); break;
        case 6: pen += 0.5 * (d0 * d0 + d2 * d2); break;
        case 7: pen += 0.5 * (d1 * d1 + d2 * d2); break;
        case 8: pen += 0.5 * (d0 * d0 + d1 * d1 + d2 * d2); break;
        default: break;
        }
    }
    if (value) *value = weight * pen;
    if (grad) {
        for (int v = 0; v < V; ++v) {
            if (off[v + 1] == off[v]) continue;
            int m[3];
            lo_axis_mask(freedom[v], m);
            for (int k = 0; k < 3; ++k)
                if (m[k]) vg[3 * v + k] = diff[3 * v + k];
        }
        for (int u = 0; u < V; ++u) {
            int n = off[u + 1] - off[u];
            if (n == 0) continue;
            int m[3];
            double contrib[3];
            lo_axis_mask(freedom[u], m);
            for (int k = 0; k < 3; ++k) contrib[k] = m[k] ? -diff[3 * u + k] / (double)n : 0.0;
            for (int i = off[u]; i < off[u + 1]; ++i)
                for (int k = 0; k < 3; ++k) vg[3 * nbr[i] + k] += contrib[k];
        }
        for (int d = 0; d < np; ++d) {
            double g = 0.0;
            for (int r = dof_off[d]; r < dof_off[d + 1]; ++r) g += vg[3 * ref_vertex[r] + ref_axis[r]] * ref_scale[r];
            grad[d] = weight * g;
        }
    }
    free(off); free(nbr); free(diff); free(vg);
}
