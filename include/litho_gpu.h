/*
 * litho_gpu.h -- C ABI of the B200 LithoInv hot path.
 *
 * The library replaces the reference's forward-operator hot path:
 *   - the polyhedron gz / TMI forward over every station x triangle pair
 *     (GravityForward::compute, modules/litho-forward/src/forward/gravity_forward.cpp:105-118;
 *      MagneticForward::compute, modules/litho-forward/src/forward/magnetic_forward.cpp:81-94),
 *   - the vertex Jacobian (computeGravityAnalyticJacobian gravity_forward.cpp:184-292;
 *      computeMagneticAnalyticJacobian magnetic_forward.cpp:196-306),
 *   - its contraction into the objective gradient (ObjectiveFunction::dataMisfitGradient
 *      modules/litho-inversion/src/inversion/objective.cpp:42-55; JointObjective::gradient
 *      modules/litho-inversion/src/inversion/joint_objective.cpp:42-111),
 *   - the parameter scatter (LithologyModel::applyParameterVector
 *      modules/litho-model/src/litho/lithology_model.cpp:210-248) and DOF gather
 *      (gravity_forward.cpp:269-289),
 *   - the projected L-BFGS driver (LBFGSBOptimizer::minimize
 *      modules/litho-inversion/src/inversion/lbfgsb_optimizer.cpp:162-263) on the host.
 *
 * Conventions: plain pointers and sizes; every call returns an lf_status.
 * Host arrays are copied in; device buffers belong to the context.  Each
 * context owns one CUDA stream that orders all its work (lf_stream); in
 * mixed precision the far-field gradient kernel runs on a second, internal
 * stream that forks from and joins back into it within the same call, so
 * results are complete in lf_stream order.  A context must not be used by
 * two threads at once
 * (the reference operators are not re-entrant either).  No CPU fallback:
 * without a usable CUDA device, lf_create returns LF_ECUDA.
 */
#ifndef LITHO_GPU_H
#define LITHO_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    LF_OK = 0,
    LF_EINVAL = 1,    /* bad argument (null pointer, size, index, NaN/Inf input) */
    LF_ECUDA = 2,     /* CUDA runtime error or no device */
    LF_ENOMEM = 3,    /* device allocation failed */
    LF_ESTATE = 4,    /* call out of order (e.g. no model set) */
    LF_ETIMEOUT = 5,  /* a bounded device wait expired */
    LF_ENUMERIC = 6   /* non-finite result detected */
} lf_status;

/* VertexFreedom numbering of modules/litho-surface/include/litho_invert/surface/surface_mesh.h:9-19 */
enum { LF_FIXED = 0, LF_Z_ONLY, LF_X_ONLY, LF_Y_ONLY, LF_ALONG_VECTOR, LF_XY_FREE, LF_XZ_FREE,
       LF_YZ_FREE, LF_XYZ_FREE };

/* RemanentMagnetizationMode, modules/litho-model/include/litho_invert/litho/litho_group.h:7-11 */
enum { LF_REM_EFFECTIVE_SUSCEPTIBILITY = 0, LF_REM_FIXED_VECTOR = 1, LF_REM_VECTOR = 2 };

/* Precision modes for lf_set_precision. */
enum {
    LF_PREC_FP64 = 0,   /* FP64 throughout, reference operation order (parity mode) */
    LF_PREC_MIXED = 1   /* FP32 bulk, FP64 where the conditioning test asks for it */
};

/* Which data type a per-type call addresses. */
enum { LF_GRAVITY = 0, LF_MAGNETIC = 1 };

/* ------------------------------------------------------------------------ */
/* Host model builder (setup time).                                         */
/* Mirrors LithologyModel / SurfaceMesh setup semantics.                    */
/* ------------------------------------------------------------------------ */
typedef struct lf_model lf_model;

lf_status lf_model_create(lf_model** out);
void lf_model_destroy(lf_model* m);

/* LithologyModel::addGroup (lithology_model.cpp:17-28) + LithoGroup fields
 * (litho_group.h:13-34).  rem_vec may be NULL.  *out_index receives the group
 * index; duplicate ids are rejected with LF_EINVAL. */
lf_status lf_model_add_group(lf_model* m, int id, double density_gcc, double susceptibility_si,
                             double rem_magnitude, double rem_inclination_deg,
                             double rem_declination_deg, const double* rem_vec3, int* out_index);

/* LithologyModel::setGroupMesh (lithology_model.cpp:62-69) of a closed mesh:
 * nv vertices (xyz[3*nv], freedom[nv] in LF_* numbering), nt triangles
 * (tri[3*nt], mesh-local, CCW seen from outside). */
lf_status lf_model_set_group_mesh(lf_model* m, int group_index, int nv, const double* xyz,
                                  const uint8_t* freedom, int nt, const int32_t* tri);

/* SurfaceMesh::setAxisScale / setBounds (surface_mesh.cpp:180-182, 250-253)
 * for one group's mesh, or every mesh when group_index < 0. */
lf_status lf_model_set_axis_scale(lf_model* m, int group_index, int axis, double scale);
lf_status lf_model_set_depth_bounds(lf_model* m, int group_index, double min_z, double max_z);
/* SurfaceMesh::setInteriorGrid (surface_mesh.cpp:671-674) */
lf_status lf_model_set_interior_grid(lf_model* m, int group_index, int interior_dim, int padding_rings);

/* LithologyModel::setControlPointStride (lithology_model.cpp:864-1040). */
lf_status lf_model_set_control_point_stride(lf_model* m, int stride, int* out_dof_count);
/* SurfaceMesh::setControlPointStride, regular N x N grid path (surface_mesh.cpp:319-431). */
lf_status lf_model_set_mesh_control_point_stride(lf_model* m, int group_index, int stride,
                                                 int* out_cp_count);
/* LithologyModel::buildSharedVertexSync (lithology_model.cpp:585-618). */
lf_status lf_model_build_shared_vertex_sync(lf_model* m);
/* LithologyModel::applyModelBounds (lithology_model.cpp:808-850). */
lf_status lf_model_apply_model_bounds(lf_model* m, double margin_multiplier);

/* Counts: groups, vertices, triangles, global DOFs (totalDofCount), refs,
 * interpolation entries, shared-sync groups, shared-sync entries. */
typedef struct {
    int n_groups, n_vertices, n_triangles, n_dofs, n_refs, n_interp, n_sync, n_sync_entries;
} lf_model_info;
lf_status lf_model_get_info(lf_model* m, lf_model_info* info);

/* LithologyModel::assembleParameterVector (lithology_model.cpp:194-208) and
 * getBounds (:250-282); arrays of n_dofs. */
lf_status lf_model_assemble_parameters(lf_model* m, double* params);
lf_status lf_model_get_bounds(lf_model* m, double* lower, double* upper);
/* Host copy of the scatter (applyParameterVector) and the current positions
 * (all meshes, group order, xyz[3*n_vertices]). */
lf_status lf_model_apply_parameters(lf_model* m, const double* params);
lf_status lf_model_get_positions(lf_model* m, double* xyz);

/* Flat tables (sizes from lf_model_get_info).  Any pointer may be NULL. */
/* Facet patches of the mixed-precision forward (no reference counterpart;
 * host only, no device needed): groups of at most 32 facets of one group with
 * at most 32 distinct corner vertices, over which the forward evaluates each
 * vertex distance and each edge line integral once per station.  Fills
 * *n_patches and, for arrays that are not NULL, the patch of every facet
 * (patch_of_facet[nt]) and each patch's distinct vertex and edge counts
 * (patch_verts / patch_edges, at least nt entries each). */
lf_status lf_facet_patches(int nv, const double* xyz, int nt, const int32_t* tri, int n_groups,
                           const int32_t* grp_tri_off, int* n_patches, int32_t* patch_of_facet,
                           int32_t* patch_verts, int32_t* patch_edges);
lf_status lf_model_export_tables(lf_model* m, double* pos, int32_t* tri, int32_t* grp_tri_off,
                                 int32_t* dof_off, int32_t* ref_vertex, uint8_t* ref_axis,
                                 double* ref_scale, int32_t* interp_off, int32_t* interp_src,
                                 double* interp_w, int32_t* sync_off, int32_t* sync_vertex);

/* ------------------------------------------------------------------------ */
/* Device context.                                                          */
/* ------------------------------------------------------------------------ */
typedef struct lf_ctx lf_ctx;

/* Creates a context on CUDA device `device` with its own stream (and the
 * internal side stream of the mixed gradient). */
lf_status lf_create(lf_ctx** out, int device);
void lf_destroy(lf_ctx* ctx);
/* Last error message of this context (static storage owned by ctx). */
const char* lf_last_error(const lf_ctx* ctx);
/* The cudaStream_t (as void*) that orders this context's work: every call's
 * results are complete once this stream reaches the point after it. */
void* lf_stream(lf_ctx* ctx);

/* Uploads geometry, group properties and DOF tables from a host model. */
lf_status lf_set_model(lf_ctx* ctx, lf_model* m);

/* Same, from raw tables (for integrators that build the tables from their
 * own LithologyModel).  group arrays have n_groups entries; interp_* and
 * sync_* may be NULL (no control points / no shared vertices). */
lf_status lf_set_model_tables(lf_ctx* ctx, int n_groups, const double* density,
                              const double* susceptibility, const double* rem_magnitude,
                              const double* rem_inclination, const double* rem_declination,
                              const double* rem_vec3, int nv, const double* xyz, int nt,
                              const int32_t* tri, const int32_t* grp_tri_off, int n_dofs,
                              const int32_t* dof_off, const int32_t* ref_vertex,
                              const uint8_t* ref_axis, const double* ref_scale,
                              const int32_t* interp_off, const int32_t* interp_src,
                              const double* interp_w, int n_sync, const int32_t* sync_off,
                              const int32_t* sync_vertex);

/* MagneticForward ctor (magnetic_forward.cpp:57-67) + setRemanenceMode. */
lf_status lf_set_field(lf_ctx* ctx, double inc_deg, double dec_deg, double field_nt,
                       int remanence_mode);

/* Station sets (GravityPoint / MagneticPoint, core/common.h:16-41): xyz[3n],
 * observed data and standard deviations (std <= 0 means weight 1). obs/std
 * may be NULL (zero data, unit weights).  n may be 0 (data type unused). */
lf_status lf_set_gravity_data(lf_ctx* ctx, int n, const double* xyz, const double* obs,
                              const double* std);
lf_status lf_set_magnetic_data(lf_ctx* ctx, int n, const double* xyz, const double* obs,
                               const double* std);

/* JointObjective weights (joint_objective.h:31-49): alpha_mag; reference-model
 * regularisation ReferenceModelRegularization (reference_model.cpp:16-25)
 * with weight ref_weight around ref_params (NULL or ref_weight <= 0: off). */
lf_status lf_set_objective(lf_ctx* ctx, double alpha_mag, double ref_weight,
                           const double* ref_params);

/* SurfaceSmoothness regularisation (smoothness.cpp:20-390), added to the
 * objective and its gradient ahead of the reference-model term, as the
 * runner registers them (runner.cpp:164-179): weight * sum over non-fixed
 * vertices of 0.5 |free axes of (p - mean of same-freedom mesh neighbours)|^2,
 * gradient gathered to DOFs with the reference's control-point semantics.
 * freedom[n_vertices]: VertexFreedom code per vertex in the tables' order;
 * NULL takes the freedoms of the model given to lf_set_model.  weight 0
 * turns it off.  LF_EINVAL for ALONG_VECTOR vertices (their move vectors are
 * not part of the tables).  Reset by every lf_set_model*. */
lf_status lf_set_smoothness(lf_ctx* ctx, double weight, const uint8_t* freedom);

lf_status lf_set_precision(lf_ctx* ctx, int mode);

/* Mixed path: a facet whose centroid lies at least tau x its longest edge
 * from a station tile's bounding box is evaluated in FP32 (quadrature for gz,
 * analytic TMI); nearer facets in FP64.  Default 3.  tau <= 0: every facet in
 * FP64 (local frame). */
lf_status lf_set_far_field_ratio(lf_ctx* ctx, double tau);
/* Station-facet pairs the mixed forward evaluated in FP64 since lf_set_model
 * or the last lf_reset_counters. */
lf_status lf_get_near_pairs(lf_ctx* ctx, unsigned long long* n);

/* Forward at params (host arrays): gz[n_grav] mGal, tmi[n_mag] nT; either
 * output may be NULL. */
lf_status lf_forward(lf_ctx* ctx, const double* params, double* gz, double* tmi);

/* Launch shapes of the hot kernels (no reference counterpart).
 *  fwd_target_blocks     forward CTAs per launch (in 128-station units):
 *                        station blocks x facet (patch) chunks; more chunks =
 *                        more CTAs, each over fewer facets
 *                        (candidates 148 x {4, 8, 16, 32, 64, 128}); 0 (patch
 *                        engine only) = a persistent grid of one CTA per
 *                        resident slot, each over a balanced contiguous range
 *                        of (station block, patch) units
 *  grad_target_warps     gradient warps per launch: DOF facets x station chunks
 *                        (148 x {16, 32, 64, 128, 256})
 *  near_tiles_per_chunk  mixed near-field gradient: 64-station tiles per warp
 *                        (0: the grad_target_warps split; candidates 0, 1, 2, 4, 8)
 *  patch_threads         stations per CTA of the patch engine (128 or 256;
 *                        each CTA walks 32-facet patches, so this is the
 *                        station x facet tile of one shared-memory stage)
 *  fwd_engine            mixed-precision forward: LF_FWD_FACET (one FP32 record
 *                        per facet; every pair evaluates its own three vertex
 *                        distances, edge integrals and solid angle) or
 *                        LF_FWD_PATCH (32-facet patches: vertex distances and
 *                        edge integrals once per station and patch, shared by
 *                        the patch's facets); lf_autotune times both
 *  far_ratio             mixed precision: facet-distance / facet-size ratio tau
 *                        beyond which a pair is FP32 far field (FP32 mid field
 *                        from tau/2, FP64 nearer); the same value as
 *                        lf_set_far_field_ratio.  lf_autotune tries
 *                        {2, 2.5, 3, 4} and accepts a ratio only if the mixed
 *                        gz and TMI stay within 0.3e-6 (norm-wise relative) of
 *                        the FP64 path at params and the gradient within
 *                        max(0.3e-5, 1.5 x the error at the current ratio)
 * lf_autotune measures candidates on the context's own model, stations and
 * precision, at params, and keeps the fastest; lf_set_tuning / lf_get_tuning
 * set and read them directly.  Results do not depend on the launch shapes
 * beyond the summation order of partial sums (far_ratio changes which pairs
 * run in FP32, within the tolerances above). */
enum { LF_FWD_FACET = 0, LF_FWD_PATCH = 1 };
typedef struct {
    int fwd_target_blocks;
    int grad_target_warps;
    int near_tiles_per_chunk;
    int patch_threads;
    double far_ratio;
    int fwd_engine;
} lf_tuning;
lf_status lf_set_tuning(lf_ctx* ctx, const lf_tuning* t);
lf_status lf_get_tuning(lf_ctx* ctx, lf_tuning* t);
/* Times each candidate over `repeats` objective+gradient evaluations (device
 * events) and keeps the fastest; *best_ms (may be NULL) = its time per
 * evaluation.  Needs the model and the data set. */
lf_status lf_autotune(lf_ctx* ctx, const double* params, int repeats, lf_tuning* chosen, double* best_ms);

/* Batched bodies (no reference counterpart: the reference inverts one model
 * at a time).  Many independent closed bodies are given as the groups of one
 * model (lf_set_model / lf_set_model_tables, one group per body), and their
 * station grids as one concatenated list: counts[g] stations of body g, in
 * group order, in both data sets.  Each body's facets then see only its own
 * stations; the forward runs as one persistent launch over (body, station
 * block, facet chunk) items ordered largest first, and the gradient as one
 * launch over every body's facets.  The objective is the sum of the bodies'
 * objectives (the gradient is separable: each body's DOFs see only its own
 * misfit); lf_get_group_objectives returns the per-body data misfits of the
 * last evaluation.  Call before setting the station data (it clears them);
 * counts = NULL turns batching off.  Dense Jacobian rows and unit responses
 * are not available in this mode (LF_ESTATE). */
lf_status lf_set_station_groups(lf_ctx* ctx, int n_groups, const int32_t* counts);
lf_status lf_get_group_objectives(lf_ctx* ctx, double* out);

/* Warm-start MLP (no reference counterpart: the reference has no learned
 * component).  A ReLU network n_in -> width x depth -> n_out trained and run
 * on the device with hand-written BF16 tensor-core GEMMs (FP32 accumulate),
 * Adam on FP32 master weights.  width and batch must be multiples of 128.
 * Inputs and targets are device fp32 arrays [rows][n_in] / [rows][n_out];
 * the loss is 0.5 x mean squared error over the batch and the n_out
 * outputs.  Parameters (get/set/gradients) in the order: for every layer W
 * [out][in] row-major, then b [out]. */
typedef struct lf_mlp lf_mlp;
lf_status lf_mlp_create(int device, int n_in, int width, int depth, int n_out, int batch, unsigned seed,
                        lf_mlp** out);
void lf_mlp_destroy(lf_mlp* m);
const char* lf_mlp_last_error(lf_mlp* m);
lf_status lf_mlp_train_step(lf_mlp* m, const float* d_x, const float* d_y, float lr, float* loss);
lf_status lf_mlp_predict(lf_mlp* m, const float* d_x, int rows, float* d_y);
lf_status lf_mlp_param_count(lf_mlp* m, size_t* n);
lf_status lf_mlp_get_params(lf_mlp* m, float* host);
lf_status lf_mlp_set_params(lf_mlp* m, const float* host);
lf_status lf_mlp_gradients(lf_mlp* m, const float* d_x, const float* d_y, float* loss, float* host_grads);
/* GEMM engine of the network:
 *  LF_GEMM_MMA_SYNC: warp-level mma.sync m16n8k16 with ldmatrix, cp.async
 *    double buffering;
 *  LF_GEMM_TCGEN05: 5th-generation tensor cores, tcgen05.mma from
 *    shared-memory descriptors, accumulator in tensor memory, 128 x 256 or
 *    128 x 128 tiles, operands staged by cp.async;
 *  LF_GEMM_TCGEN05_TMA: the same MMA fed by TMA (2-D tensor maps, 128-byte
 *    swizzle, no multicast) in a warp-specialised pipeline (one producer
 *    warp, one MMA warp, every warp in the epilogue);
 *  LF_GEMM_AUTO (default): per GEMM, LF_GEMM_TCGEN05_TMA for K >= 2048 and
 *    LF_GEMM_MMA_SYNC below (measured faster on each side of that line).
 * All give the same results to FP32 summation order. */
enum { LF_GEMM_TCGEN05 = 0, LF_GEMM_MMA_SYNC = 1, LF_GEMM_TCGEN05_TMA = 2, LF_GEMM_AUTO = 3 };
lf_status lf_mlp_set_engine(lf_mlp* m, int engine);
/* The network's BF16 GEMM on device buffers: C[M x N] = A[M x K] . B[K x N]
 * with A stored [M][K] (a_trans = 0) or [K][M] (a_trans = 1), B stored
 * [K][N] (b_trans = 0) or [N][K] (b_trans = 1), row lengths lda / ldb / ldc
 * (multiples of 8 elements, operands 16-byte aligned), FP32 accumulation;
 * epilogue 0: C fp32, 1: bf16 relu(C + bias[n]), 2: fp32 C + bias[n],
 * 3: bf16 C.  M and N multiples of 128, K of 64 (tcgen05) or 32 (mma.sync).
 * Runs on `stream` (NULL = default stream) and synchronises it; returns
 * LF_ETIMEOUT if a tensor-core mbarrier wait expired. */
lf_status lf_gemm_bf16(int engine, int a_trans, int b_trans, int epilogue, int M, int N, int K, const void* A,
                       int lda, const void* B, int ldb, const float* bias, void* C, int ldc, void* stream);
/* Poll limit of the tensor-core GEMM's main-loop mbarrier waits on the
 * current device (default 2^24 polls, well under a second; a negative value
 * restores it).  No counterpart in the reference: failure detection.  A wait
 * that reaches the limit makes the kernel stop issuing work, wait (with the
 * full limit) for its own MMAs, free its tensor memory and raise the error
 * flag that lf_gemm_bf16 / the lf_mlp_* calls report as LF_ETIMEOUT; with 0,
 * every such wait expires at once, which is how the tests exercise that path.
 * The device stays usable afterwards. */
lf_status lf_set_device_wait_limit(long long polls);

/* Stateless parameter scatter (off by default).  The reference's
 * applyParameterVector averages shared vertices from their current positions
 * (lithology_model.cpp:235-247), and vertices that the DOFs and the
 * control-point interpolation do not rewrite keep what earlier calls left,
 * so the model after evaluating p depends on the parameters evaluated before
 * (reproduced bit for bit by default; on x/y-free models a line-search trial
 * far away can displace such vertices by hundreds of metres for every later
 * evaluation).  Enabled, every scatter starts from the model's positions as
 * given to lf_set_model, so the evaluation at p depends on p alone. */
lf_status lf_set_scatter_stateless(lf_ctx* ctx, int enabled);

/* Gradient gather of the objective gradient (lf_objective_grad,
 * lf_objective_grad_device, graph mode).  No reference counterpart.
 *  LF_GATHER_REFERENCE (default): the reference's gather -- the vertex
 *    gradient read at each DOF's own (vertex, axis) slots times the axis scale
 *    (gravity_forward.cpp:270-289, magnetic_forward.cpp's copy).  With
 *    control-point interpolation or shared-vertex averaging this is not the
 *    derivative of the objective: vertices that follow the control points
 *    contribute nothing, and a line search along it can fail to descend.
 *  LF_GATHER_CHAIN: the exact derivative of the objective with respect to
 *    the parameters through the whole scatter -- the vertex gradient (misfit
 *    plus weighted smoothness) mapped back through the averaging and the
 *    interpolation, then gathered as above.  The gradient is computed at
 *    every vertex whose position depends on the parameters, so the gradient
 *    kernels cover more facets.  With lf_set_scatter_stateless it is the
 *    gradient of a function of p alone.
 * lf_jacobian and the calibration products keep the reference's gather. */
enum { LF_GATHER_REFERENCE = 0, LF_GATHER_CHAIN = 1 };
lf_status lf_set_gradient_gather(lf_ctx* ctx, int mode);

/* x / y vertex derivatives of the objective gradient.
 *  LF_XY_ANALYTIC (default): closed-form derivatives on every axis.
 *  LF_XY_FORWARD_DIFFERENCE: x and y by per-facet forward differences of the
 *    reference's facet formula with the given step (metres; the
 *    large-inversion configuration uses 0.5), z analytic -- the reference's
 *    per-facet differencing (faceNagyWithGradient gravity_forward.cpp:48-85,
 *    magneticFacetWithGradient magnetic_forward.cpp:14-50, there with
 *    h = 1e-4 on every axis) restricted to x and y.  Evaluated in FP64 in
 *    both precision modes (six moved copies of each gradient facet per
 *    station).  Facets collapsed onto a line contribute zero, as in the
 *    analytic path.  lf_jacobian keeps its analytic derivatives.
 * step is ignored for LF_XY_ANALYTIC; otherwise it must be positive. */
enum { LF_XY_ANALYTIC = 0, LF_XY_FORWARD_DIFFERENCE = 1 };
lf_status lf_set_xy_derivative(lf_ctx* ctx, int mode, double step);

/* Facets collapsed onto a line (twice-area below 1e-10 x the longest edge
 * squared; the control-point interpolation produces them).  No reference
 * counterpart.
 *  LF_COLLAPSED_KEEP (default): the forward evaluates them as the reference
 *    does.  Their unit normal is rounding noise and the reference's TMI facet
 *    term (magnetic_forward.cpp:312-347) does not vanish with the area, so
 *    their TMI contribution is reproduced bit for bit but is a discontinuous
 *    function of the positions: central differences of the objective jump
 *    by orders of magnitude between steps of 1e-1 and 1e-3 m.
 *  LF_COLLAPSED_DROP: they contribute nothing to the forward either (the
 *    gradient kernels always take them as zero), so that the objective is
 *    the function its gradient differentiates.
 * Applies to every forward of the context (both precisions and engines,
 * unit responses included). */
enum { LF_COLLAPSED_KEEP = 0, LF_COLLAPSED_DROP = 1 };
lf_status lf_set_collapsed_facets(lf_ctx* ctx, int mode);

/* Graph mode (no reference counterpart: the reference evaluates on one CPU
 * thread).  When enabled, lf_objective, lf_objective_grad and
 * lf_objective_grad_device replay a CUDA graph of the whole evaluation
 * (scatter, forward, residuals, objective, gradient) instead of launching its
 * kernels one by one: the first call with a given set of buffers runs
 * normally and captures the sequence, later calls replay it.  Any setter,
 * and any call that grows a device buffer, invalidates the graph.  Results
 * are identical to the direct launches.  Profiling (lf_set_profiling) turns
 * replay off while it is enabled. */
lf_status lf_set_graph_mode(lf_ctx* ctx, int enabled);

/* Objective components at params: out5 = {gravity misfit, magnetic misfit,
 * regularisation, constraint penalty (0), total} (JointComponents,
 * joint_objective.h:55-63). */
lf_status lf_objective(lf_ctx* ctx, const double* params, double* out5);

/* Objective and its gradient in one fused evaluation (the Jacobian is never
 * formed): *f = total objective, grad[n_dofs]. */
lf_status lf_objective_grad(lf_ctx* ctx, const double* params, double* f, double* grad);

/* Data-weight calibration (JointObjective::calibrateDataWeights,
 * joint_objective.cpp:281-393), matrix-free: power iteration for the largest
 * eigenvalue of J^T W^2 J of each data type with J v from a central
 * difference of the FP64 forward and J^T w from the gradient kernels (the
 * reference forms both dense Jacobians); alpha_mag *= clip(lambda_grav /
 * lambda_mag, 1e-6, 1e6), or the gradient-norm ratio when degenerate.  Updates
 * the context's alpha_mag like the reference; no-op without magnetic data or
 * with alpha_mag <= 0.  seed: start vector.  Any output pointer may be NULL. */
lf_status lf_calibrate_data_weights(lf_ctx* ctx, const double* params, unsigned seed, double* alpha_mag,
                                    double* eig_grav, double* eig_mag);

/* Per-group unit responses at params (positions as after lf_forward), for
 * property inversion: the forward of group `group` alone with
 *  LF_UNIT_GRAVITY    unit density (mGal per g/cc) at the gravity stations
 *                     (GravityForward::computeGroupUnitResponse,
 *                     gravity_forward.cpp:132-146);
 *  LF_UNIT_INDUCED    unit susceptibility under the inducing field (nT per SI)
 *                     at the magnetic stations (MagneticForward::
 *                     computeGroupUnitResponse, magnetic_forward.cpp:148-162);
 *  LF_UNIT_DIRECTION  unit magnetisation along dir[3] (as given, not
 *                     normalised) (computeGroupUnitResponseDirection :164-178);
 *  LF_UNIT_REMANENCE  unit magnetisation along the group's remanence
 *                     inclination/declination (computeGroupUnitRemanenceResponse
 *                     :180-190).
 * out[n_stations] in caller station order. */
enum { LF_UNIT_GRAVITY = 0, LF_UNIT_INDUCED = 1, LF_UNIT_DIRECTION = 2, LF_UNIT_REMANENCE = 3 };
lf_status lf_unit_response(lf_ctx* ctx, const double* params, int kind, int group, const double* dir,
                           double* out);

/* Property step of the alternating inversion (InversionRunner::
 * runPropertyInversion, modules/litho-inversion/src/inversion/
 * runner.cpp:708-917, parts A and B): at the geometry `params`, the
 * per-group unit responses (one lf_unit_response column each) form U, and
 * the small bounded least-squares problem
 *   min_d 0.5 sum_i (w_i (obs_i - (U d)_i))^2 / rms^2 + 0.5 damping |d - d0|^2,
 *   rms = sqrt(max(mean(obs^2), 1)),
 * is solved on the host by the projected L-BFGS of lf_lbfgsb_minimize
 * (history min(5, n), the given iteration limit and tolerance).  Part A:
 * densities from the gravity data; part B (when magnetic data are set):
 * per group chi, plus the remanence magnitude (LF_REM_FIXED_VECTOR) or the
 * remanence vector (LF_REM_VECTOR), bounds as the runner's options.  The
 * results are written back into the context's groups (as the reference
 * writes them into its model) and returned: density[G], magnetic[p G] with
 * p = 1, 2 or 4 parameters per group (NULL to skip). */
typedef struct {
    double density_min, density_max;                            /* propertyDensityMin / Max */
    double susceptibility_min, susceptibility_max;              /* propertySusceptibilityMin / Max */
    double remanence_min, remanence_max;                        /* propertyRemanenceMin / Max */
    double remanence_component_min, remanence_component_max;    /* propertyRemanenceComponentMin / Max */
    double damping;                                             /* propertyDamping */
    int max_iterations;                                         /* propertyInversionMaxIter */
    double tolerance;                                           /* tolerance */
} lf_property_options;
lf_status lf_property_inversion(lf_ctx* ctx, const double* params, const lf_property_options* opt, double* density,
                                double* magnetic);

/* Dense Jacobian J[n_data x n_dofs] (row-major) of gravity (which = LF_GRAVITY)
 * or TMI (LF_MAGNETIC) at params, with the reference's DOF gather semantics:
 * each DOF collects its control-point vertices' own derivative times the axis
 * scale.  Analytic derivative (the reference uses forward differences with
 * h = 1e-4 m).  Intended for small problems and parity checks. */
lf_status lf_jacobian(lf_ctx* ctx, const double* params, int which, double* J);

/* Current device vertex positions after the last scatter, xyz[3*n_vertices]
 * (the reference leaves the shared LithologyModel at the last parameters:
 * gravity_forward.cpp:106). */
lf_status lf_get_positions(lf_ctx* ctx, double* xyz);

/* Device-resident variants: the same evaluations on device pointers (inputs
 * already in HBM, results left in HBM, stream-ordered on lf_stream). */
lf_status lf_forward_device(lf_ctx* ctx, const double* d_params, double* d_gz, double* d_tmi);
lf_status lf_objective_grad_device(lf_ctx* ctx, const double* d_params, double* d_f,
                                   double* d_grad);

/* Projected L-BFGS ("L-BFGS-B") on the device objective; semantics of
 * LBFGSBOptimizer (lbfgsb_optimizer.cpp:33-263, options lbfgsb_optimizer.h:13-57). */
typedef struct {
    int max_iterations;      /* default 500 (optimizer.h:36) */
    double tolerance;        /* ftol, default 1e-6 (optimizer.h:35) */
    int history_size;        /* default 10 */
    double armijo_c1;        /* default 1e-4 */
    int line_search_max_iter;/* default 50 */
    int disable_line_search; /* default 0 */
    double initial_gamma;    /* > 0: H0 = gamma*I for the first step (warm start); 0 = steepest descent */
    double target_value;     /* > 0: stop once the objective is at or below it (no reference
                                counterpart; e.g. the chi^2 = N data misfit); 0 = off */
} lf_lbfgsb_options;
typedef struct {
    int iterations;
    int converged;
    int evaluations;         /* objective-only evaluations */
    int gradients;           /* objective+gradient evaluations */
    double final_value;
    char message[96];
} lf_lbfgsb_result;
void lf_lbfgsb_default_options(lf_lbfgsb_options* opt);
lf_status lf_lbfgsb_minimize(lf_ctx* ctx, const double* x0, const double* lower,
                             const double* upper, const lf_lbfgsb_options* opt, double* x_out,
                             lf_lbfgsb_result* result);

/* Work counters since the last reset: station-facet pairs evaluated by the
 * forward (every facet) and by the gradient (facets with at least one
 * DOF-referenced vertex; the others have no derivative to contribute), and
 * kernel launches. */
typedef struct {
    uint64_t forward_pairs, gradient_pairs, launches;
} lf_counters;
lf_status lf_get_counters(lf_ctx* ctx, lf_counters* c);
/* Zeroes the counters and the near-pair count (lf_get_near_pairs). */
lf_status lf_reset_counters(lf_ctx* ctx);

/* Kernel timing on the context's stream: when enabled, every launch of the
 * forward pair kernel and of the gradient pair kernels is bracketed by CUDA
 * events (the two mixed gradient kernels then run one after the other on
 * the context's stream rather than concurrently).  lf_get_kernel_times synchronises the stream and returns the summed
 * durations (ms) and launch counts since profiling was (re)enabled. */
lf_status lf_set_profiling(lf_ctx* ctx, int enabled);
lf_status lf_get_kernel_times(lf_ctx* ctx, double* forward_ms, int* forward_launches,
                              double* gradient_ms, int* gradient_launches);

/* ---------------------------------------- point classification, constraints */
/* LithologyModel::setLabelGrid (modules/litho-model/src/litho/
 * lithology_model.cpp:89-103): labels[(iz*ny + iy)*nx + ix] = group id of
 * voxel (ix, iy, iz) with corner (x0, y0, z0) and spacing (dx, dy, dz); a
 * voxel holding a negative id falls back to ray casting.  nx, ny or nz <= 0
 * or labels == NULL removes the grid.  Spacings must be non-zero. */
lf_status lf_set_label_grid(lf_ctx* ctx, int nx, int ny, int nz, double x0, double y0, double z0, double dx,
                            double dy, double dz, const int32_t* labels);
/* LithologyModel::setBottomDepth (lithology_model.cpp:856-858): points below
 * it classify as -1.  Default -5000. */
lf_status lf_set_bottom_depth(lf_ctx* ctx, double depth);
/* LithologyModel::classifyPoint (lithology_model.cpp:288-363) for n points
 * xyz[3n]: group[i] = the group whose closed mesh contains the point (label
 * grid first, then a +x ray cast against every group mesh in group order,
 * first odd crossing count wins), -1 outside every mesh or below the bottom
 * depth.  With params != NULL the parameters are applied first
 * (applyParameterVector); with NULL the positions of the last call are used.
 * Same answers as the reference, bit for bit (the ray test is evaluated in
 * FP64 in the reference's operation order). */
lf_status lf_classify_points(lf_ctx* ctx, const double* params, int n, const double* xyz, int32_t* group);
/* ConstraintHandler(model, constraints) + setWeight (modules/
 * litho-inversion/src/inversion/constraint_handler.cpp:7-13,
 * include/.../constraint_handler.h:16): n borehole intervals, xy[2n] column
 * positions, z_top / z_bottom depths positive down, group = lithology known
 * in the interval.  The reference's default weight is 1e6. */
lf_status lf_set_constraints(lf_ctx* ctx, int n, const double* xy, const double* z_top, const double* z_bottom,
                             const int32_t* group, double weight);
/* ConstraintHandler::evaluate (constraint_handler.cpp:31-42): weight x sum
 * of squared violations, a violation being |z_bottom - z_top| when the
 * interval midpoint does not classify as its group.  Applies params. */
lf_status lf_constraint_penalty(lf_ctx* ctx, const double* params, double* value);
/* ConstraintHandler::gradient (constraint_handler.cpp:44-66): central
 * differences with a 1 m step over every parameter (2 np evaluations, each a
 * scatter + classification of every interval midpoint on the GPU), scaled
 * by the weight as the reference does (the evaluations already carry it, so
 * the result carries weight^2).  Leaves the positions at the last perturbed
 * parameters, as the reference leaves its model.  The ObjectiveFunction
 * with a constraint handler (objective.cpp:61-73, 97-101) is lf_objective /
 * lf_objective_grad plus these two. */
lf_status lf_constraint_gradient(lf_ctx* ctx, const double* params, double* grad);

/* LithologyModel::validate (modules/litho-model/src/litho/
 * lithology_model.cpp:624-803) at params (NULL: the current positions): the
 * shared-vertex gap, adjacent and non-adjacent overlap (every vertex
 * classified as in lf_classify_points, on the GPU), edge-tearing, bounding
 * box and spike checks in the reference's order; *passed = 0 with the
 * reference's failure text in reason[reason_len] and its worst violation in
 * *worst for the first check that fails.  freedom[n_vertices] (NULL: the
 * builder's) marks the boundary vertices of the tearing check (not
 * LF_XYZ_FREE).  The overlap baselines are the runner's (runner.cpp:494-516:
 * counts of the initial model, obtainable with lf_classify_points). */
lf_status lf_validate_model(lf_ctx* ctx, const double* params, const uint8_t* freedom,
                            unsigned long long overlap_baseline, unsigned long long adjacent_overlap_baseline,
                            int* passed, double* worst, char* reason, int reason_len);

/* InversionRunner::smoothGradient (modules/litho-inversion/src/inversion/
 * runner.cpp:643-706), the runner's optional gradient smoothing: every
 * DOF-mapped vertex axis blends its gradient with the mean over its mesh
 * neighbours carrying the same axis, (1 - weight) g + weight mean, and each
 * DOF takes the value of its last (mesh, local DOF) reference.  weight <= 0
 * returns the gradient unchanged.  Host arrays (lf_smooth_gradient) or device
 * buffers on the context's stream (lf_smooth_gradient_device; in and out may
 * be the same buffer). */
lf_status lf_smooth_gradient(lf_ctx* ctx, double weight, const double* grad_in, double* grad_out);
lf_status lf_smooth_gradient_device(lf_ctx* ctx, double weight, const double* d_grad_in, double* d_grad_out);

/* ---------------------------------------------------------------- surfaces */
/* loadSurfaceMesh (modules/litho-io/src/io/surface_loader.cpp:163-181):
 * a GOCAD TSurf (.ts: VRTX / PVRTX vertices in file order, TRGL 1-based
 * triangles, HEADER blocks, comments and GOCAD / TFACE / TRIANGLES lines
 * skipped, END stops) or OBJ (.obj: v, f / fo with polygons fanned from the
 * first vertex) surface.  Call with xyz = tri = NULL for the counts, then
 * with xyz[3 n_vertices] and tri[3 n_triangles] (0-based).  LF_EINVAL for an
 * unreadable file, another extension, a file without vertices or a triangle
 * naming a vertex the file does not have (the reference returns that mesh
 * unchecked). */
lf_status lf_read_surface(const char* path, int* n_vertices, int* n_triangles, double* xyz, int32_t* tri);
/* InversionExporter::exportTS (modules/litho-io/src/io/exporters.cpp:116-151):
 * writes a GOCAD TSurf with header name `name`, vertices in %.8e form and
 * 1-based triangles. */
lf_status lf_write_tsurf(const char* path, const char* name, int n_vertices, const double* xyz, int n_triangles,
                         const int32_t* tri);

/* ------------------------------------------------------------------------ */
/* Allocation-free forward.  No counterpart in the reference: for callers    */
/* that cannot call cudaMalloc (a host framework owning all device memory   */
/* through its own pool, a fixed memory budget, a real-time loop that must  */
/* not allocate).                                                            */
/* ------------------------------------------------------------------------ */
/* gz (mGal) and TMI (nT) of one closed triangulated body (induced
 * magnetisation, density contrast density_gcc, susceptibility_si, inducing
 * field inc/dec/field_nt) at ns stations -- the single-group case of
 * lf_forward.  Every array is caller-owned DEVICE memory: d_xyz[3*nv],
 * d_tri[3*nt], d_sta[3*ns], d_gz[ns], d_tmi[ns] (either output may be NULL).
 * Allocates nothing: its scratch is one 8 MiB __device__ array inside the
 * library, so 38*nt + 2*ns must not exceed 1,048,544 (e.g. nt <= 16384 facets
 * with ns <= 212,000 stations); larger sizes return LF_EINVAL.  The first
 * call on a device looks the scratch address up (cudaGetSymbolAddress) and
 * keeps it for the life of the process, so calls after a cudaDeviceReset of
 * that device are not supported.  Every call reads an error flag back to the
 * host and waits for its stream, so no call may be made on a stream that is
 * being captured into a CUDA graph: a capturing stream returns LF_EINVAL.  An
 * error already pending on the calling thread returns LF_ECUDA (left pending)
 * before any work is queued.  Calls share the scratch, so calls that overlap
 * on the GPU race: serialise them.  Triangle indices outside [0, nv) return
 * LF_EINVAL.  Runs on `stream` (a cudaStream_t, NULL = default stream) and
 * returns after the stream has finished the call. */
lf_status lf_forward_noalloc(int nv, const double* d_xyz, int nt, const int32_t* d_tri, int ns,
                             const double* d_sta, double density_gcc, double susceptibility_si,
                             double inc_deg, double dec_deg, double field_nt, double* d_gz,
                             double* d_tmi, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LITHO_GPU_H */
