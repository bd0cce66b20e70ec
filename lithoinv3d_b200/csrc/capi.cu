// C ABI implementation: contexts, device buffers and the launch sequence of
// one forward / objective / objective+gradient evaluation.
#include "../../include/litho_gpu.h"
#include "kernels_classify.cuh"
#include "kernels_mixed.cuh"
#include "kernels_facet.cuh"
#include "kernels_patch.cuh"
#include "lbfgsb.hpp"
#include "model_builder.hpp"
#include "patches.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <random>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace litho_b200;

struct lf_model {
    LithologyModelHost host;
};

namespace {

// Bumped by every device (re)allocation in the process: a captured CUDA
// graph holds raw buffer addresses and is re-captured when this moves.
static uint64_t& reallocAll() {
    static uint64_t n = 0;
    return n;
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t reserve(size_t count) {
        if (count <= n && p) return cudaSuccess;
        release();
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) { p = nullptr; return e; }
        n = count;
        ++reallocAll();
        return cudaSuccess;
    }
};

struct GroupProps {
    double density, chi, remMag, remInc, remDec, remVec[3];
};

// A station set lives on the device in Morton order of (x, y), so that a
// tile of consecutive stations is spatially compact (the mixed-precision
// near/far test is per tile).  perm[i] = caller index of device slot i.
struct StationSet {
    int n = 0;
    std::vector<double> xyz, obs, w;  // caller order
    std::vector<int32_t> perm;
    DevBuf<double> d_xyz, d_obs, d_w, d_pred, d_coef, d_out, d_tileBox;
    DevBuf<int32_t> d_perm;
};

constexpr double kGSI = 6.67430e-11, kDensityScale = 1000.0, kMs2ToMgal = 1e5;

}  // namespace

struct lf_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    // Second stream of the mixed gradient: the FP32 far-field kernel runs
    // beside the FP64 near-field one (fork and join by events; inside a
    // captured graph these become two parallel branches).
    cudaStream_t side = nullptr;
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    std::string err;
    int precision = LF_PREC_FP64;

    // model
    bool hasModel = false;
    int G = 0, V = 0, T = 0, np = 0;
    std::vector<GroupProps> groups;
    std::vector<int32_t> grpTriOff;
    double inc = 90.0, dec = 0.0, fieldNT = 50000.0;
    int remMode = 0;
    d3 fdir{0, 0, -1};
    std::vector<GroupConst> gconst;

    DevBuf<double> d_pos, d_fc, d_gc, d_mc, d_params, d_grad, d_vgrad, d_out5, d_f, d_refp;
    DevBuf<FaceF32> d_mf32;  // per-facet FP32 records of the facet engine [T]
    DevBuf<unsigned long long> d_nearPairs;
    float tau = 3.0f;  // far-field ratio of the mixed path

    // patch forward of the mixed path (kernels_patch.cuh): topology built
    // once per model, record blobs rewritten every evaluation
    PatchTopology ptopo;
    DevBuf<int32_t> d_pFacetOff, d_pFacets, d_pVertOff, d_pVerts, d_pEdgeOff, d_pBlobOff, d_pChunkBegin, d_pChunkEnd,
        d_pFacetPatch, d_pFacetSlot;
    DevBuf<float> d_mt2;  // doubled TMI edge coefficients of every facet [3][T]
    DevBuf<uint32_t> d_pCorners, d_pEdgeInfo;
    DevBuf<uint8_t> d_pEdgeSlot, d_blobs;
    DevBuf<unsigned int> d_patchErr;
    std::vector<int32_t> pchunkBegin, pchunkEnd;
    int pchunkS = 0, pchunkFilter = -2, pchunkThreads = 0;
    int64_t pchunkFacets = 0;
    bool pchunksDirty = true;
    int patchThreads = 128;  // stations per CTA of the patch forward (lf_tuning.patch_threads)
    DevBuf<FwdItem> d_pItems;
    DevBuf<int64_t> d_pGrpPartOff;
    DevBuf<int32_t> d_pGrpNch;
    int npItems = 0;
    int64_t pPartTotal = 0, pItemPairs = 0;
    uint64_t pItemsEpoch = ~0ull;
    int pItemsThreads = 0;
    // persistent schedule (tune.fwd_target_blocks == 0): per-block slot counts
    DevBuf<int32_t> d_pBlockNch;
    long long pPersistKey = -1;
    int pPersistSlots = 0, pPersistGrid = 0;
    DevBuf<int32_t> d_tri, d_dofOff, d_refVertex, d_interpOff, d_interpSrc, d_interpRows, d_syncOff,
        d_syncVertex, d_vfOff, d_vf, d_gradVerts, d_gradFacets, d_chunkBegin, d_chunkEnd, d_chunkGroup;
    DevBuf<uint8_t> d_refAxis, d_faceNeeds;
    DevBuf<double> d_refScale, d_interpW;
    DevBuf<int16_t> d_faceGroup;
    DevBuf<GroupConst> d_groups;
    int nInterpRows = 0, nSync = 0, nGradVerts = 0, nGradFacets = 0;
    double maxRefScale = 0.0;
    bool statelessScatter = false;  // lf_set_scatter_stateless
    DevBuf<double> d_pos0;          // the model's positions as given
    DevBuf<double> d_vel, d_posSave, d_tmpP, d_tmpS;  // matrix-free products (calibration)
    std::vector<int32_t> hGradFacets;
    // Gradient gather (lf_set_gradient_gather): LF_GATHER_REFERENCE reads the
    // vertex gradient at the DOF vertices only; LF_GATHER_CHAIN first maps it
    // back through the shared-vertex averaging and the control-point
    // interpolation.  The vertex / facet sets each mode needs, per model.
    int gatherMode = 0;
    std::vector<int32_t> hGvertsRef, hGvertsChain, hGfacetsRef, hGfacetsChain;
    std::vector<uint8_t> hFneedRef, hFneedChain;
    DevBuf<int32_t> d_adjOff, d_adjRow;  // interpolation transposed: source -> (row, weight)
    DevBuf<double> d_adjW, d_vgrad2;
    // lf_set_xy_derivative: x and y vertex derivatives of the objective
    // gradient by per-facet forward differences with step xyStep (FP64)
    int dropCollapsed = 0;  // lf_set_collapsed_facets
    int xyMode = 0;
    double xyStep = 0.5;
    DevBuf<double> d_fcfd;  // [7][NFC][nGradFacets] moved-facet constants

    // forward chunking (plan cached per station count and group filter;
    // uploaded only when it changes)
    std::vector<int32_t> chunkBegin, chunkEnd, chunkGroup;
    int chunkCapacityS = 0, chunkFilter = -1, groupFilter = -1;
    int64_t chunkFacets = 0;
    bool chunksDirty = true;

    // data
    StationSet grav, mag;
    bool sameStations = false;
    double alphaMag = 1.0, refWeight = 0.0;
    bool hasRef = false;

    // SurfaceSmoothness regularisation (off unless lf_set_smoothness)
    std::vector<uint8_t> vertexFreedom;  // from lf_set_model's builder
    std::vector<int32_t> grpVertOff;     // vertex range of each group mesh (lf_set_model's builder)
    bool smoothOn = false;
    double smoothWeight = 0.0;
    DevBuf<int32_t> d_smOff, d_smNbr;
    DevBuf<uint8_t> d_freedom;
    DevBuf<double> d_smDiff, d_smVgrad, d_blockS;

    // workspaces
    DevBuf<double> d_partG, d_partM, d_partGrad, d_blockG, d_blockM, d_ones, d_jac;

    // point classification and the constraint penalty (lf_set_label_grid,
    // lf_set_bottom_depth, lf_set_constraints)
    double bottomDepth = -5000.0;  // LithologyModel's default
    LabelGridDev labelGrid;        // labels -> d_labels.p when a grid is set
    DevBuf<int32_t> d_labels, d_grpTriOffDev, d_cGroup, d_cCls, d_ptCls;
    DevBuf<unsigned long long> d_clsMask;  // per-point crossing parities (one bit per group)
    DevBuf<double> d_cMid, d_cThick, d_cPar, d_cPar0, d_cFp, d_cFm, d_cGrad, d_cOut, d_pts;
    int nCons = 0;
    double consWeight = 1e6;  // ConstraintHandler's default weight

    // gradient smoothing (lf_smooth_gradient): mesh neighbour lists, built on first use
    bool gnReady = false;
    DevBuf<int32_t> d_gnOff, d_gnList;
    DevBuf<double> d_gsVg, d_gsSg, d_gsIn;
    DevBuf<uint8_t> d_gsHas;

    lf_counters counters{0, 0, 0};

    // CUDA graph replay of whole evaluations (lf_set_graph_mode).  epoch is
    // bumped by every setter; a cached graph is valid for one (epoch,
    // allocation count, buffer addresses) and is re-captured otherwise.
    struct GraphCache {
        cudaGraphExec_t exec = nullptr;
        uint64_t epoch = ~0ull, reallocs = ~0ull;
        const double* params = nullptr;
        double *f = nullptr, *grad = nullptr;
        lf_counters delta{0, 0, 0};
    };
    static constexpr int kGraphSlots = 4;  // buffer sets replayed without re-capture (e.g. ping-pong params)
    struct GraphSet {
        GraphCache slot[kGraphSlots];
        int next = 0;
        uint64_t failedEpoch = ~0ull;
    };
    bool graphMode = false;
    uint64_t epoch = 0;
    GraphSet gObjGrad, gObj, gCons;

    // launch shapes chosen by lf_autotune (defaults: the autotuner's choice
    // on the 19k-facet, 4096-station contact model)
    lf_tuning tune{148 * 128, 148 * 32, 0, 128, 3.0, LF_FWD_FACET};

    // Batched bodies (lf_set_station_groups): each group is one body and
    // sees only its own station range [grpStaOff[g], grpStaOff[g+1]) of both
    // data sets.  The forward runs a persistent item list (body, station
    // block, facet chunk), planned when planEpoch moves.
    bool partitioned = false;
    std::vector<int32_t> grpStaOff, grpTileOff;
    DevBuf<int32_t> d_grpStaOff, d_grpTileOff, d_staGroup, d_grpNch;
    DevBuf<int64_t> d_grpPartOff;
    DevBuf<FwdItem> d_items;
    DevBuf<double> d_grpF;
    int nItems = 0, maxGroupStations = 0;
    int64_t partTotal = 0, itemPairs = 0;
    uint64_t planEpoch = 0, itemsEpoch = ~0ull;

    // optional per-kernel timing (events on `stream`)
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evFwd, evGrad;
    size_t nFwd = 0, nGrad = 0;
};

static void clear_events(std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v) {
    for (auto& e : v) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    v.clear();
}

// Records a begin event for a profiled launch; returns the slot or -1.
static int prof_begin(lf_ctx* c, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v, size_t& n) {
    if (!c->profiling) return -1;
    if (n == v.size()) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess) return -1;
        if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return -1; }
        v.push_back({a, b});
    }
    cudaEventRecord(v[n].first, c->stream);
    return static_cast<int>(n++);
}
static void prof_end(lf_ctx* c, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v, int slot) {
    if (slot >= 0) cudaEventRecord(v[slot].second, c->stream);
}

#define LF_TRY_CUDA(ctx, expr)                                                           \
    do {                                                                                 \
        cudaError_t e__ = (expr);                                                        \
        if (e__ != cudaSuccess) {                                                        \
            (ctx)->err = std::string(#expr) + ": " + cudaGetErrorString(e__);            \
            return e__ == cudaErrorMemoryAllocation ? LF_ENOMEM : LF_ECUDA;              \
        }                                                                                \
    } while (0)

#define LF_CHECK_LAUNCH(ctx) LF_TRY_CUDA(ctx, cudaGetLastError())

#define LF_RET_IF(x)                      \
    do {                                  \
        lf_status s__ = (x);              \
        if (s__ != LF_OK) return s__;     \
    } while (0)

static lf_status fail(lf_ctx* ctx, lf_status st, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return st;
}

static bool finite_all(const double* p, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

template <typename T>
static cudaError_t upload(DevBuf<T>& b, const T* h, size_t n, cudaStream_t s) {
    cudaError_t e = b.reserve(n);
    if (e != cudaSuccess || n == 0) return e;
    return cudaMemcpyAsync(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice, s);
}

static inline int cdiv(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

// ------------------------------------------------------------------ model --
extern "C" lf_status lf_model_create(lf_model** out) {
    if (!out) return LF_EINVAL;
    *out = new (std::nothrow) lf_model();
    return *out ? LF_OK : LF_ENOMEM;
}
extern "C" void lf_model_destroy(lf_model* m) { delete m; }

extern "C" lf_status lf_model_add_group(lf_model* m, int id, double density, double chi, double remMag,
                                        double remInc, double remDec, const double* remVec, int* outIndex) {
    if (!m || !std::isfinite(density) || !std::isfinite(chi)) return LF_EINVAL;
    Group g;
    g.id = id;
    g.density = density;
    g.susceptibility = chi;
    g.remMagnitude = remMag;
    g.remInclination = remInc;
    g.remDeclination = remDec;
    if (remVec) g.remVector = {remVec[0], remVec[1], remVec[2]};
    int idx = m->host.addGroup(g);
    if (outIndex) *outIndex = idx;
    return idx < 0 ? LF_EINVAL : LF_OK;
}

extern "C" lf_status lf_model_set_group_mesh(lf_model* m, int gi, int nv, const double* xyz, const uint8_t* freedom,
                                             int nt, const int32_t* tri) {
    if (!m || gi < 0 || gi >= m->host.groupCount() || nv < 0 || nt < 0) return LF_EINVAL;
    if ((nv && (!xyz || !freedom)) || (nt && !tri)) return LF_EINVAL;
    if (!finite_all(xyz, static_cast<size_t>(nv) * 3)) return LF_EINVAL;
    Mesh mesh;
    mesh.pos.resize(nv);
    mesh.freedom.assign(freedom, freedom + nv);
    for (int v = 0; v < nv; ++v) {
        mesh.pos[v] = {xyz[3 * v], xyz[3 * v + 1], xyz[3 * v + 2]};
        if (freedom[v] > XYZ_FREE) return LF_EINVAL;
    }
    mesh.tri.resize(static_cast<size_t>(nt) * 3);
    for (int k = 0; k < 3 * nt; ++k) {
        if (tri[k] < 0 || tri[k] >= nv) return LF_EINVAL;
        mesh.tri[k] = static_cast<uint32_t>(tri[k]);
    }
    return m->host.setGroupMesh(gi, std::move(mesh)) == 0 ? LF_OK : LF_EINVAL;
}

template <typename Fn>
static lf_status for_meshes(lf_model* m, int gi, Fn fn) {
    if (!m) return LF_EINVAL;
    if (gi >= 0) {
        Mesh* mesh = m->host.mesh(gi);
        if (!mesh) return LF_EINVAL;
        fn(*mesh);
    } else {
        for (int g = 0; g < m->host.meshCount(); ++g)
            if (Mesh* mesh = m->host.mesh(g)) fn(*mesh);
    }
    m->host.markDirty();
    return LF_OK;
}

extern "C" lf_status lf_model_set_axis_scale(lf_model* m, int gi, int axis, double scale) {
    if (axis < 0 || axis > 2 || !(scale != 0.0) || !std::isfinite(scale)) return LF_EINVAL;
    return for_meshes(m, gi, [&](Mesh& me) { me.axisScale[axis] = scale; });
}
extern "C" lf_status lf_model_set_depth_bounds(lf_model* m, int gi, double minZ, double maxZ) {
    return for_meshes(m, gi, [&](Mesh& me) { me.minDepth = minZ; me.maxDepth = maxZ; });
}
extern "C" lf_status lf_model_set_interior_grid(lf_model* m, int gi, int dim, int rings) {
    if (dim < 0 || rings < 0) return LF_EINVAL;
    return for_meshes(m, gi, [&](Mesh& me) {
        me.interiorGridDim = dim;
        me.paddingRings = rings;
        me.rebuildDofMappings();
    });
}
extern "C" lf_status lf_model_set_control_point_stride(lf_model* m, int stride, int* outDofs) {
    if (!m) return LF_EINVAL;
    uint32_t n = m->host.setControlPointStride(stride);
    if (outDofs) *outDofs = static_cast<int>(n);
    return LF_OK;
}
extern "C" lf_status lf_model_set_mesh_control_point_stride(lf_model* m, int gi, int stride, int* outCp) {
    if (!m || gi < 0) return LF_EINVAL;
    Mesh* mesh = m->host.mesh(gi);
    if (!mesh) return LF_EINVAL;
    uint32_t n = mesh->setControlPointStrideGrid(stride);
    mesh->rebuildDofMappings();
    m->host.markDirty();
    if (outCp) *outCp = static_cast<int>(n);
    return LF_OK;
}
extern "C" lf_status lf_model_build_shared_vertex_sync(lf_model* m) {
    if (!m) return LF_EINVAL;
    m->host.buildSharedVertexSync();
    return LF_OK;
}
extern "C" lf_status lf_model_apply_model_bounds(lf_model* m, double margin) {
    if (!m) return LF_EINVAL;
    m->host.applyModelBounds(margin);
    return LF_OK;
}
extern "C" lf_status lf_model_get_info(lf_model* m, lf_model_info* info) {
    if (!m || !info) return LF_EINVAL;
    ModelTables t = m->host.tables();
    info->n_groups = t.nGroups;
    info->n_vertices = t.nVertices;
    info->n_triangles = t.nTriangles;
    info->n_dofs = t.nDofs;
    info->n_refs = static_cast<int>(t.refVertex.size());
    info->n_interp = static_cast<int>(t.interpSrc.size());
    info->n_sync = static_cast<int>(t.syncOff.size()) - 1;
    info->n_sync_entries = static_cast<int>(t.syncVertex.size());
    return LF_OK;
}
extern "C" lf_status lf_model_assemble_parameters(lf_model* m, double* params) {
    if (!m || !params) return LF_EINVAL;
    auto p = m->host.assembleParameterVector();
    std::copy(p.begin(), p.end(), params);
    return LF_OK;
}
extern "C" lf_status lf_model_get_bounds(lf_model* m, double* lo, double* hi) {
    if (!m || !lo || !hi) return LF_EINVAL;
    std::vector<double> l, h;
    m->host.getBounds(l, h);
    std::copy(l.begin(), l.end(), lo);
    std::copy(h.begin(), h.end(), hi);
    return LF_OK;
}
extern "C" lf_status lf_model_apply_parameters(lf_model* m, const double* params) {
    if (!m || !params) return LF_EINVAL;
    uint32_t n = m->host.totalDofCount();
    if (!finite_all(params, n)) return LF_EINVAL;
    m->host.applyParameterVector(std::vector<double>(params, params + n));
    return LF_OK;
}
extern "C" lf_status lf_model_get_positions(lf_model* m, double* xyz) {
    if (!m || !xyz) return LF_EINVAL;
    ModelTables t = m->host.tables();
    std::copy(t.pos.begin(), t.pos.end(), xyz);
    return LF_OK;
}
extern "C" lf_status lf_model_export_tables(lf_model* m, double* pos, int32_t* tri, int32_t* grpTriOff, int32_t* dofOff,
                                            int32_t* refVertex, uint8_t* refAxis, double* refScale, int32_t* interpOff,
                                            int32_t* interpSrc, double* interpW, int32_t* syncOff, int32_t* syncVertex) {
    if (!m) return LF_EINVAL;
    ModelTables t = m->host.tables();
    auto cp = [](auto* dst, const auto& v) {
        if (dst) std::copy(v.begin(), v.end(), dst);
    };
    cp(pos, t.pos); cp(tri, t.tri); cp(grpTriOff, t.grpTriOff); cp(dofOff, t.dofOff);
    cp(refVertex, t.refVertex); cp(refAxis, t.refAxis); cp(refScale, t.refScale);
    cp(interpOff, t.interpOff); cp(interpSrc, t.interpSrc); cp(interpW, t.interpW);
    cp(syncOff, t.syncOff); cp(syncVertex, t.syncVertex);
    return LF_OK;
}

// Facet patches of the mixed forward for a triangle set (host only; the
// context builds the same patches in lf_set_model_tables).
extern "C" lf_status lf_facet_patches(int nv, const double* xyz, int nt, const int32_t* tri, int G,
                                      const int32_t* grpTriOff, int* nPatches, int32_t* patchOfFacet,
                                      int32_t* patchVerts, int32_t* patchEdges) {
    if (nv <= 0 || nt <= 0 || G <= 0 || !xyz || !tri || !grpTriOff || !nPatches) return LF_EINVAL;
    if (grpTriOff[0] != 0 || grpTriOff[G] != nt) return LF_EINVAL;
    for (int g = 0; g < G; ++g)
        if (grpTriOff[g + 1] < grpTriOff[g]) return LF_EINVAL;
    for (int k = 0; k < 3 * nt; ++k)
        if (tri[k] < 0 || tri[k] >= nv) return LF_EINVAL;
    const PatchTopology pt = build_patches(nv, xyz, nt, tri, G, grpTriOff);
    *nPatches = pt.P;
    for (int p = 0; p < pt.P; ++p) {
        if (patchOfFacet)
            for (int k = pt.facetOff[p]; k < pt.facetOff[p + 1]; ++k) patchOfFacet[pt.facets[k]] = p;
        if (patchVerts) patchVerts[p] = pt.vertOff[p + 1] - pt.vertOff[p];
        if (patchEdges) patchEdges[p] = pt.edgeOff[p + 1] - pt.edgeOff[p];
    }
    return LF_OK;
}

// ---------------------------------------------------------------- context --
extern "C" lf_status lf_create(lf_ctx** out, int device) {
    if (!out) return LF_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return LF_ECUDA;
    }
    if (device < 0 || device >= n) return LF_EINVAL;
    lf_ctx* c = new (std::nothrow) lf_ctx();
    if (!c) return LF_ENOMEM;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return LF_ECUDA;
    }
    if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->evFork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->evJoin, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();  // without them the two gradient kernels run one after the other
        if (c->evFork) cudaEventDestroy(c->evFork);
        if (c->side) cudaStreamDestroy(c->side);
        c->side = nullptr;
        c->evFork = c->evJoin = nullptr;
    }
    *out = c;
    return LF_OK;
}

static void drop_graph(lf_ctx::GraphSet& set) {
    for (auto& g : set.slot) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = lf_ctx::GraphCache{};
    }
    set.next = 0;
    set.failedEpoch = ~0ull;
}

extern "C" void lf_destroy(lf_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c->gObjGrad);
    drop_graph(c->gObj);
    drop_graph(c->gCons);
    clear_events(c->evFwd);
    clear_events(c->evGrad);
    if (c->side) cudaStreamSynchronize(c->side);
    if (c->evFork) cudaEventDestroy(c->evFork);
    if (c->evJoin) cudaEventDestroy(c->evJoin);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" const char* lf_last_error(const lf_ctx* c) { return c ? c->err.c_str() : "null context"; }
extern "C" void* lf_stream(lf_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

// Group magnetisation (MagneticForward ctor magnetic_forward.cpp:57-67 and
// buildGroupMagnetization :100-134) and gravity scales (gravity_forward.cpp:176, :230).
static void compute_group_consts(lf_ctx* c) {
    double I = c->inc * kPi / 180.0, D = c->dec * kPi / 180.0;
    double cI = std::cos(I);
    c->fdir = {cI * std::cos(D), cI * std::sin(D), -std::sin(I)};
    c->gconst.resize(c->G);
    for (int g = 0; g < c->G; ++g) {
        const GroupProps& p = c->groups[g];
        GroupConst& k = c->gconst[g];
        k.gscale_fwd = kGSI * p.density * kDensityScale * kMs2ToMgal;
        k.gscale_jac = (kGSI * kDensityScale * kMs2ToMgal) * p.density;
        double induced = p.chi * c->fieldNT / 100.0;
        double M[3] = {induced * c->fdir.x, induced * c->fdir.y, induced * c->fdir.z};
        if (c->remMode == LF_REM_FIXED_VECTOR) {
            double Ir = p.remInc * kPi / 180.0, Dr = p.remDec * kPi / 180.0, cr = std::cos(Ir);
            double R[3] = {cr * std::cos(Dr), cr * std::sin(Dr), -std::sin(Ir)};
            for (int i = 0; i < 3; ++i) M[i] += p.remMag * R[i];
        } else if (c->remMode == LF_REM_VECTOR) {
            for (int i = 0; i < 3; ++i) M[i] += p.remVec[i];
        }
        double amp = std::sqrt(M[0] * M[0] + M[1] * M[1] + M[2] * M[2]);
        if (amp < kEps) {
            k.mdir[0] = c->fdir.x; k.mdir[1] = c->fdir.y; k.mdir[2] = c->fdir.z;
        } else {
            for (int i = 0; i < 3; ++i) k.mdir[i] = M[i] / amp;
        }
        k.mscale = amp * 100.0 / (4.0 * kPi);
        k.mag_active = amp < kEps ? 0 : 1;
    }
}

static lf_status upload_groups(lf_ctx* c) {
    compute_group_consts(c);
    LF_TRY_CUDA(c, upload(c->d_groups, c->gconst.data(), c->gconst.size(), c->stream));
    return LF_OK;
}

// Vertex / facet sets of the current gather mode onto the device.
static lf_status apply_gather_sets(lf_ctx* c) {
    const bool chain = c->gatherMode == LF_GATHER_CHAIN;
    const std::vector<int32_t>& gv = chain ? c->hGvertsChain : c->hGvertsRef;
    const std::vector<int32_t>& gf = chain ? c->hGfacetsChain : c->hGfacetsRef;
    const std::vector<uint8_t>& fn = chain ? c->hFneedChain : c->hFneedRef;
    c->nGradVerts = static_cast<int>(gv.size());
    c->nGradFacets = static_cast<int>(gf.size());
    c->hGradFacets = gf;
    if (!gf.empty()) LF_TRY_CUDA(c, upload(c->d_gradFacets, gf.data(), gf.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_gradVerts, gv.data(), gv.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_faceNeeds, fn.data(), fn.size(), c->stream));
    c->epoch++;
    return LF_OK;
}

extern "C" lf_status lf_set_model_tables(lf_ctx* c, int G, const double* density, const double* chi,
                                         const double* remMag, const double* remInc, const double* remDec,
                                         const double* remVec, int nv, const double* xyz, int nt, const int32_t* tri,
                                         const int32_t* grpTriOff, int np, const int32_t* dofOff,
                                         const int32_t* refVertex, const uint8_t* refAxis, const double* refScale,
                                         const int32_t* interpOff, const int32_t* interpSrc, const double* interpW,
                                         int nSync, const int32_t* syncOff, const int32_t* syncVertex) {
    if (!c) return LF_EINVAL;
    c->epoch++;
    if (G <= 0 || G > 32000 || nv <= 0 || nt <= 0 || np < 0 || !density || !xyz || !tri || !grpTriOff ||
        (np > 0 && (!dofOff || !refVertex || !refAxis || !refScale)))
        return fail(c, LF_EINVAL, "lf_set_model_tables: bad sizes or null arrays");
    if (!finite_all(xyz, (size_t)nv * 3)) return fail(c, LF_EINVAL, "non-finite vertex position");
    if (grpTriOff[0] != 0 || grpTriOff[G] != nt) return fail(c, LF_EINVAL, "grp_tri_off must span [0, nt]");
    for (int g = 0; g < G; ++g)
        if (grpTriOff[g + 1] < grpTriOff[g]) return fail(c, LF_EINVAL, "grp_tri_off not monotone");
    for (int k = 0; k < 3 * nt; ++k)
        if (tri[k] < 0 || tri[k] >= nv) return fail(c, LF_EINVAL, "triangle index out of range");
    int nref = np > 0 ? dofOff[np] : 0;
    if (np > 0 && dofOff[0] != 0) return fail(c, LF_EINVAL, "dof_off[0] must be 0");
    for (int d = 0; d < np; ++d)
        if (dofOff[d + 1] < dofOff[d]) return fail(c, LF_EINVAL, "dof_off not monotone");
    for (int r = 0; r < nref; ++r)
        if (refVertex[r] < 0 || refVertex[r] >= nv || refAxis[r] > 2 || !std::isfinite(refScale[r]))
            return fail(c, LF_EINVAL, "bad DOF ref");
    int nInterp = interpOff ? interpOff[nv] : 0;
    if (interpOff) {
        if (interpOff[0] != 0 || (nInterp > 0 && (!interpSrc || !interpW)))
            return fail(c, LF_EINVAL, "bad interpolation table");
        for (int v = 0; v < nv; ++v)
            if (interpOff[v + 1] < interpOff[v]) return fail(c, LF_EINVAL, "interp_off not monotone");
        for (int k = 0; k < nInterp; ++k)
            if (interpSrc[k] < 0 || interpSrc[k] >= nv || interpOff[interpSrc[k] + 1] != interpOff[interpSrc[k]])
                return fail(c, LF_EINVAL, "interpolation source must be a control point");
    }
    if (nSync > 0) {
        if (!syncOff || syncOff[0] != 0 || (syncOff[nSync] > 0 && !syncVertex))
            return fail(c, LF_EINVAL, "bad shared-vertex table");
        for (int s = 0; s < nSync; ++s)
            if (syncOff[s + 1] < syncOff[s]) return fail(c, LF_EINVAL, "sync_off not monotone");
        for (int k = 0; k < syncOff[nSync]; ++k)
            if (syncVertex[k] < 0 || syncVertex[k] >= nv) return fail(c, LF_EINVAL, "sync vertex out of range");
    }
    cudaSetDevice(c->device);
    c->G = G; c->V = nv; c->T = nt; c->np = np;
    c->groups.resize(G);
    for (int g = 0; g < G; ++g) {
        GroupProps& p = c->groups[g];
        p.density = density[g];
        p.chi = chi ? chi[g] : 0.0;
        p.remMag = remMag ? remMag[g] : 0.0;
        p.remInc = remInc ? remInc[g] : 0.0;
        p.remDec = remDec ? remDec[g] : 0.0;
        for (int i = 0; i < 3; ++i) p.remVec[i] = remVec ? remVec[3 * g + i] : 0.0;
    }
    c->grpTriOff.assign(grpTriOff, grpTriOff + G + 1);
    lf_status st = upload_groups(c);
    if (st != LF_OK) return st;

    // geometry + tables
    LF_TRY_CUDA(c, upload(c->d_pos, xyz, (size_t)nv * 3, c->stream));
    LF_TRY_CUDA(c, upload(c->d_pos0, xyz, (size_t)nv * 3, c->stream));
    LF_TRY_CUDA(c, upload(c->d_tri, tri, (size_t)nt * 3, c->stream));
    std::vector<int16_t> faceGroup(nt);
    for (int g = 0; g < G; ++g)
        for (int f = grpTriOff[g]; f < grpTriOff[g + 1]; ++f) faceGroup[f] = static_cast<int16_t>(g);
    LF_TRY_CUDA(c, upload(c->d_faceGroup, faceGroup.data(), faceGroup.size(), c->stream));
    std::vector<int32_t> dofOffV(np + 1, 0);
    if (np > 0) dofOffV.assign(dofOff, dofOff + np + 1);
    LF_TRY_CUDA(c, upload(c->d_dofOff, dofOffV.data(), dofOffV.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_refVertex, refVertex, (size_t)nref, c->stream));
    LF_TRY_CUDA(c, upload(c->d_refAxis, refAxis, (size_t)nref, c->stream));
    LF_TRY_CUDA(c, upload(c->d_refScale, refScale, (size_t)nref, c->stream));
    c->maxRefScale = 0.0;
    for (int r = 0; r < nref; ++r) c->maxRefScale = std::max(c->maxRefScale, std::fabs(refScale[r]));
    std::vector<int32_t> rows;
    if (interpOff) {
        for (int v = 0; v < nv; ++v)
            if (interpOff[v + 1] > interpOff[v]) rows.push_back(v);
        LF_TRY_CUDA(c, upload(c->d_interpOff, interpOff, (size_t)nv + 1, c->stream));
        LF_TRY_CUDA(c, upload(c->d_interpSrc, interpSrc, (size_t)nInterp, c->stream));
        LF_TRY_CUDA(c, upload(c->d_interpW, interpW, (size_t)nInterp, c->stream));
    }
    c->nInterpRows = static_cast<int>(rows.size());
    LF_TRY_CUDA(c, upload(c->d_interpRows, rows.data(), rows.size(), c->stream));
    c->nSync = nSync > 0 ? nSync : 0;
    if (c->nSync) {
        LF_TRY_CUDA(c, upload(c->d_syncOff, syncOff, (size_t)nSync + 1, c->stream));
        LF_TRY_CUDA(c, upload(c->d_syncVertex, syncVertex, (size_t)syncOff[nSync], c->stream));
    }
    // vertex -> (facet, corner) incidence, DOF vertices, facets needing gradients
    std::vector<int32_t> vfOff(nv + 1, 0), vf(3 * (size_t)nt);
    for (int k = 0; k < 3 * nt; ++k) vfOff[tri[k] + 1]++;
    for (int v = 0; v < nv; ++v) vfOff[v + 1] += vfOff[v];
    {
        std::vector<int32_t> fill(vfOff.begin(), vfOff.end() - 1);
        for (int k = 0; k < 3 * nt; ++k) vf[fill[tri[k]]++] = k;  // k = facet*3 + corner
    }
    LF_TRY_CUDA(c, upload(c->d_vfOff, vfOff.data(), vfOff.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_vf, vf.data(), vf.size(), c->stream));
    {
        // Reference gather: the DOF vertices.  Chain gather: every vertex whose
        // scattered position depends on the parameters -- the DOF vertices,
        // interpolation rows with such a source (a row's own DOF write is
        // overwritten), then whole averaging groups with such a member.
        std::vector<uint8_t> vref(nv, 0), vdep(nv, 0);
        for (int r = 0; r < nref; ++r) vref[refVertex[r]] = vdep[refVertex[r]] = 1;
        if (interpOff)
            for (int v = 0; v < nv; ++v) {
                if (interpOff[v + 1] == interpOff[v]) continue;
                uint8_t d = 0;
                for (int k = interpOff[v]; k < interpOff[v + 1]; ++k) d |= vref[interpSrc[k]];
                vdep[v] = d;
            }
        for (int q = 0; q < c->nSync; ++q) {
            uint8_t d = 0;
            for (int k = syncOff[q]; k < syncOff[q + 1]; ++k) d |= vdep[syncVertex[k]];
            if (d)
                for (int k = syncOff[q]; k < syncOff[q + 1]; ++k) vdep[syncVertex[k]] = 1;
        }
        auto sets = [&](const std::vector<uint8_t>& vn, std::vector<int32_t>& gv, std::vector<int32_t>& gf,
                        std::vector<uint8_t>& fn) {
            gv.clear();
            gf.clear();
            fn.assign(nt, 0);
            for (int v = 0; v < nv; ++v)
                if (vn[v]) gv.push_back(v);
            for (int f = 0; f < nt; ++f) {
                fn[f] = vn[tri[3 * f]] | vn[tri[3 * f + 1]] | vn[tri[3 * f + 2]];
                if (fn[f]) gf.push_back(f);
            }
        };
        sets(vref, c->hGvertsRef, c->hGfacetsRef, c->hFneedRef);
        sets(vdep, c->hGvertsChain, c->hGfacetsChain, c->hFneedChain);
        // interpolation transposed (CSR over sources, rows in increasing order)
        std::vector<int32_t> adjOff(nv + 1, 0), adjRow;
        std::vector<double> adjW;
        if (interpOff) {
            for (int k = 0; k < nInterp; ++k) adjOff[interpSrc[k] + 1]++;
            for (int v = 0; v < nv; ++v) adjOff[v + 1] += adjOff[v];
            adjRow.resize(nInterp);
            adjW.resize(nInterp);
            std::vector<int32_t> fill(adjOff.begin(), adjOff.end() - 1);
            for (int v = 0; v < nv; ++v)
                for (int k = interpOff[v]; k < interpOff[v + 1]; ++k) {
                    adjRow[fill[interpSrc[k]]] = v;
                    adjW[fill[interpSrc[k]]++] = interpW[k];
                }
        }
        LF_TRY_CUDA(c, upload(c->d_adjOff, adjOff.data(), adjOff.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_adjRow, adjRow.data(), adjRow.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_adjW, adjW.data(), adjW.size(), c->stream));
        LF_TRY_CUDA(c, c->d_vgrad2.reserve((size_t)nv * 3));
    }
    LF_RET_IF(apply_gather_sets(c));
    LF_TRY_CUDA(c, c->d_fc.reserve((size_t)NFC * nt));
    LF_TRY_CUDA(c, c->d_mc.reserve((size_t)NMC * nt));
    {  // facet patches of the mixed forward
        c->ptopo = build_patches(nv, xyz, nt, tri, G, grpTriOff);
        const PatchTopology& pt = c->ptopo;
        LF_TRY_CUDA(c, upload(c->d_pFacetOff, pt.facetOff.data(), pt.facetOff.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_pFacets, pt.facets.data(), pt.facets.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_pCorners, pt.facetCorners.data(), pt.facetCorners.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_pVertOff, pt.vertOff.data(), pt.vertOff.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_pVerts, pt.verts.data(), pt.verts.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_pEdgeOff, pt.edgeOff.data(), pt.edgeOff.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_pEdgeInfo, pt.edgeInfo.data(), pt.edgeInfo.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_pEdgeSlot, pt.edgeSlot.data(), pt.edgeSlot.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_pBlobOff, pt.blobOff.data(), pt.blobOff.size(), c->stream));
        std::vector<int32_t> fpatch(nt, 0), fslot(nt, 0);
        for (int q = 0; q < pt.P; ++q)
            for (int k = pt.facetOff[q]; k < pt.facetOff[q + 1]; ++k) {
                fpatch[pt.facets[k]] = q;
                fslot[pt.facets[k]] = k - pt.facetOff[q];
            }
        LF_TRY_CUDA(c, upload(c->d_pFacetPatch, fpatch.data(), fpatch.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_pFacetSlot, fslot.data(), fslot.size(), c->stream));
        LF_TRY_CUDA(c, c->d_mt2.reserve((size_t)3 * nt));
        LF_TRY_CUDA(c, c->d_blobs.reserve((size_t)std::max(pt.blobOff.back(), 16)));
        LF_TRY_CUDA(c, c->d_patchErr.reserve(1));
        LF_TRY_CUDA(c, cudaMemsetAsync(c->d_patchErr.p, 0, sizeof(unsigned int), c->stream));
        c->pchunkS = 0;
        c->pItemsEpoch = ~0ull;
    }
    LF_TRY_CUDA(c, c->d_nearPairs.reserve(1));
    LF_TRY_CUDA(c, cudaMemsetAsync(c->d_nearPairs.p, 0, sizeof(unsigned long long), c->stream));
    LF_TRY_CUDA(c, c->d_gc.reserve((size_t)NGC * nt));
    LF_TRY_CUDA(c, c->d_params.reserve(std::max(np, 1)));
    LF_TRY_CUDA(c, c->d_grad.reserve(std::max(np, 1)));
    LF_TRY_CUDA(c, c->d_vgrad.reserve((size_t)nv * 3));
    LF_TRY_CUDA(c, cudaMemsetAsync(c->d_vgrad.p, 0, (size_t)nv * 3 * sizeof(double), c->stream));
    LF_TRY_CUDA(c, c->d_out5.reserve(5));
    LF_TRY_CUDA(c, c->d_f.reserve(1));
    c->chunkCapacityS = 0;
    c->hasRef = false;
    c->smoothOn = false;
    c->vertexFreedom.clear();
    c->grpVertOff.clear();
    c->partitioned = false;
    c->planEpoch++;
    c->hasModel = true;
    c->gnReady = false;
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

extern "C" lf_status lf_set_model(lf_ctx* c, lf_model* m) {
    if (!c || !m) return LF_EINVAL;
    ModelTables t = m->host.tables();
    int G = t.nGroups;
    std::vector<double> rho(G), chi(G), rm(G), ri(G), rd(G), rv(3 * G);
    for (int g = 0; g < G; ++g) {
        const Group& gr = m->host.group(g);
        rho[g] = gr.density; chi[g] = gr.susceptibility; rm[g] = gr.remMagnitude;
        ri[g] = gr.remInclination; rd[g] = gr.remDeclination;
        rv[3 * g] = gr.remVector.x; rv[3 * g + 1] = gr.remVector.y; rv[3 * g + 2] = gr.remVector.z;
    }
    int nSync = static_cast<int>(t.syncOff.size()) - 1;
    lf_status st = lf_set_model_tables(c, G, rho.data(), chi.data(), rm.data(), ri.data(), rd.data(), rv.data(),
                                       t.nVertices, t.pos.data(), t.nTriangles, t.tri.data(), t.grpTriOff.data(),
                                       t.nDofs, t.dofOff.data(), t.refVertex.data(), t.refAxis.data(),
                                       t.refScale.data(), t.interpOff.data(), t.interpSrc.data(), t.interpW.data(),
                                       nSync, t.syncOff.data(), t.syncVertex.data());
    if (st != LF_OK) return st;
    c->grpVertOff.assign(t.vertexOffset.begin(), t.vertexOffset.end());
    // vertex freedoms in the tables' vertex order (meshes in group order)
    for (int g = 0; g < m->host.meshCount(); ++g)
        if (const Mesh* mesh = m->host.mesh(g))
            c->vertexFreedom.insert(c->vertexFreedom.end(), mesh->freedom.begin(), mesh->freedom.end());
    if ((int)c->vertexFreedom.size() != c->V) c->vertexFreedom.clear();
    return LF_OK;
}

// SurfaceSmoothness (smoothness.cpp): same-freedom neighbour lists per vertex,
// built like SurfaceMesh::buildNeighbors (surface_mesh.cpp:265-286: the other
// vertices of every triangle holding the vertex, ascending, without
// duplicates), filtered to the vertex's own freedom; FIXED vertices get none.
extern "C" lf_status lf_set_smoothness(lf_ctx* c, double weight, const uint8_t* freedom) {
    if (!c || !std::isfinite(weight) || weight < 0.0) return LF_EINVAL;
    c->epoch++;
    if (!c->hasModel) return fail(c, LF_ESTATE, "lf_set_smoothness before lf_set_model");
    if (weight == 0.0) {
        c->smoothOn = false;
        c->smoothWeight = 0.0;
        return LF_OK;
    }
    const uint8_t* fr = freedom ? freedom : (c->vertexFreedom.empty() ? nullptr : c->vertexFreedom.data());
    if (!fr) return fail(c, LF_EINVAL, "lf_set_smoothness: no vertex freedoms known (pass freedom[n_vertices])");
    const int V = c->V, T = c->T;
    for (int v = 0; v < V; ++v) {
        if (fr[v] > LF_XYZ_FREE) return fail(c, LF_EINVAL, "lf_set_smoothness: bad freedom code");
        if (fr[v] == LF_ALONG_VECTOR)
            return fail(c, LF_EINVAL, "lf_set_smoothness: ALONG_VECTOR vertices need move vectors, not supported");
    }
    std::vector<int32_t> tri((size_t)3 * T);
    LF_TRY_CUDA(c, cudaMemcpyAsync(tri.data(), c->d_tri.p, sizeof(int32_t) * tri.size(), cudaMemcpyDeviceToHost,
                                   c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    std::vector<std::vector<int32_t>> nb(V);
    for (int t = 0; t < T; ++t) {
        int a = tri[3 * t], b = tri[3 * t + 1], d = tri[3 * t + 2];
        nb[a].push_back(b); nb[a].push_back(d);
        nb[b].push_back(a); nb[b].push_back(d);
        nb[d].push_back(a); nb[d].push_back(b);
    }
    std::vector<int32_t> off(V + 1, 0), list;
    for (int v = 0; v < V; ++v) {
        std::vector<int32_t>& l = nb[v];
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
        if (fr[v] != LF_FIXED)
            for (int32_t u : l)
                if (fr[u] == fr[v]) list.push_back(u);
        off[v + 1] = static_cast<int32_t>(list.size());
    }
    LF_TRY_CUDA(c, upload(c->d_smOff, off.data(), off.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_smNbr, list.empty() ? off.data() : list.data(), std::max<size_t>(list.size(), 1),
                          c->stream));
    LF_TRY_CUDA(c, upload(c->d_freedom, fr, (size_t)V, c->stream));
    LF_TRY_CUDA(c, c->d_smDiff.reserve((size_t)3 * V));
    LF_TRY_CUDA(c, c->d_smVgrad.reserve((size_t)3 * V));
    LF_TRY_CUDA(c, c->d_blockS.reserve(cdiv(V, 256)));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    c->smoothOn = true;
    c->smoothWeight = weight;
    return LF_OK;
}

// diff and per-block penalties at the current positions.
static lf_status smooth_diff(lf_ctx* c) {
    if (!c->smoothOn) return LF_OK;
    k_smooth_diff<<<cdiv(c->V, 256), 256, 0, c->stream>>>(c->V, c->d_pos.p, c->d_freedom.p, c->d_smOff.p,
                                                          c->d_smNbr.p, c->d_smDiff.p, c->d_blockS.p);
    c->counters.launches++;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

extern "C" lf_status lf_set_field(lf_ctx* c, double inc, double dec, double field, int remMode) {
    if (!c || !std::isfinite(inc) || !std::isfinite(dec) || !std::isfinite(field) || remMode < 0 || remMode > 2)
        return LF_EINVAL;
    c->epoch++;
    c->inc = inc; c->dec = dec; c->fieldNT = field; c->remMode = remMode;
    if (c->hasModel) return upload_groups(c);
    return LF_OK;
}

static lf_status set_stations(lf_ctx* c, StationSet& s, int n, const double* xyz, const double* obs, const double* sd) {
    if (!c || n < 0 || (n > 0 && !xyz)) return LF_EINVAL;
    c->epoch++;
    if (!finite_all(xyz, (size_t)n * 3)) return fail(c, LF_EINVAL, "non-finite station position");
    if (obs && !finite_all(obs, n)) return fail(c, LF_EINVAL, "non-finite observation");
    cudaSetDevice(c->device);
    s.n = n;
    s.xyz.assign(xyz, xyz + 3 * (size_t)n);
    s.obs.assign(n, 0.0);
    s.w.assign(n, 1.0);
    for (int i = 0; i < n; ++i) {
        if (obs) s.obs[i] = obs[i];
        if (sd && sd[i] > 0) s.w[i] = 1.0 / sd[i];  // objective.cpp:26
    }
    // Segments: the whole set, or each group's stations when the stations
    // are partitioned among batched bodies (lf_set_station_groups).
    std::vector<int32_t> seg = {0, n};
    if (c->partitioned) {
        if (n != c->grpStaOff.back())
            return fail(c, LF_EINVAL, "station count differs from the sum of lf_set_station_groups counts");
        seg = c->grpStaOff;
    }
    // Morton order of (x, y) quantised to 16 bits over each segment's extent
    s.perm.resize(n);
    for (size_t g = 0; g + 1 < seg.size(); ++g) {
        const int b = seg[g], e = seg[g + 1];
        double lo[2] = {1e300, 1e300}, hi[2] = {-1e300, -1e300};
        for (int i = b; i < e; ++i)
            for (int k = 0; k < 2; ++k) {
                lo[k] = std::min(lo[k], s.xyz[3 * i + k]);
                hi[k] = std::max(hi[k], s.xyz[3 * i + k]);
            }
        std::vector<std::pair<uint32_t, int32_t>> key(e - b);
        for (int i = b; i < e; ++i) {
            uint32_t q[2];
            for (int k = 0; k < 2; ++k) {
                double span = hi[k] - lo[k];
                q[k] = span > 0 ? static_cast<uint32_t>((s.xyz[3 * i + k] - lo[k]) / span * 65535.0) : 0u;
            }
            uint32_t m = 0;
            for (int bit = 0; bit < 16; ++bit)
                m |= ((q[0] >> bit) & 1u) << (2 * bit) | ((q[1] >> bit) & 1u) << (2 * bit + 1);
            key[i - b] = {m, i};
        }
        std::stable_sort(key.begin(), key.end());
        for (int i = b; i < e; ++i) s.perm[i] = key[i - b].second;
    }
    std::vector<double> px(3 * (size_t)n), po(n), pw(n);
    for (int i = 0; i < n; ++i) {
        int j = s.perm[i];
        px[3 * i] = s.xyz[3 * j]; px[3 * i + 1] = s.xyz[3 * j + 1]; px[3 * i + 2] = s.xyz[3 * j + 2];
        po[i] = s.obs[j];
        pw[i] = s.w[j];
    }
    LF_TRY_CUDA(c, upload(s.d_xyz, px.data(), px.size(), c->stream));
    LF_TRY_CUDA(c, upload(s.d_obs, po.data(), po.size(), c->stream));
    LF_TRY_CUDA(c, upload(s.d_w, pw.data(), pw.size(), c->stream));
    LF_TRY_CUDA(c, upload(s.d_perm, s.perm.data(), s.perm.size(), c->stream));
    // bounding box of every tile of kStationTile consecutive (Morton-ordered)
    // stations; tiles never straddle segments
    {
        std::vector<double> box;
        std::vector<int32_t> tileOff(1, 0);
        for (size_t g = 0; g + 1 < seg.size(); ++g) {
            for (int t0 = seg[g]; t0 < seg[g + 1]; t0 += kStationTile) {
                double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
                for (int i = t0; i < std::min(seg[g + 1], t0 + kStationTile); ++i)
                    for (int k = 0; k < 3; ++k) {
                        lo[k] = std::min(lo[k], px[3 * i + k]);
                        hi[k] = std::max(hi[k], px[3 * i + k]);
                    }
                for (int k = 0; k < 3; ++k) box.push_back(lo[k]);
                for (int k = 0; k < 3; ++k) box.push_back(hi[k]);
            }
            tileOff.push_back(static_cast<int32_t>(box.size() / 6));
        }
        if (box.empty()) box.assign(6, 0.0);
        LF_TRY_CUDA(c, upload(s.d_tileBox, box.data(), box.size(), c->stream));
        if (c->partitioned) {
            c->grpTileOff = tileOff;
            LF_TRY_CUDA(c, upload(c->d_grpTileOff, tileOff.data(), tileOff.size(), c->stream));
        }
    }
    LF_TRY_CUDA(c, s.d_pred.reserve(std::max(n, 1)));
    LF_TRY_CUDA(c, s.d_coef.reserve(std::max(n, 1)));
    LF_TRY_CUDA(c, s.d_out.reserve(std::max(n, 1)));
    c->sameStations = c->grav.n > 0 && c->grav.n == c->mag.n && c->grav.xyz == c->mag.xyz &&
                      c->grav.perm == c->mag.perm;
    c->chunkCapacityS = 0;
    c->planEpoch++;
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

extern "C" lf_status lf_set_gravity_data(lf_ctx* c, int n, const double* xyz, const double* obs, const double* sd) {
    return c ? set_stations(c, c->grav, n, xyz, obs, sd) : LF_EINVAL;
}
extern "C" lf_status lf_set_magnetic_data(lf_ctx* c, int n, const double* xyz, const double* obs, const double* sd) {
    return c ? set_stations(c, c->mag, n, xyz, obs, sd) : LF_EINVAL;
}

extern "C" lf_status lf_set_objective(lf_ctx* c, double alpha, double refWeight, const double* refParams) {
    if (!c || !std::isfinite(alpha) || !std::isfinite(refWeight)) return LF_EINVAL;
    c->epoch++;
    if (!c->hasModel) return fail(c, LF_ESTATE, "lf_set_objective before lf_set_model");
    c->alphaMag = alpha;
    c->refWeight = refWeight;
    c->hasRef = refParams && refWeight > 0.0;
    if (c->hasRef) {
        if (!finite_all(refParams, c->np)) return fail(c, LF_EINVAL, "non-finite reference parameters");
        LF_TRY_CUDA(c, upload(c->d_refp, refParams, (size_t)c->np, c->stream));
        LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return LF_OK;
}

extern "C" lf_status lf_set_far_field_ratio(lf_ctx* c, double tau) {
    if (!c || !std::isfinite(tau)) return LF_EINVAL;
    c->epoch++;
    c->tau = tau <= 0.0 ? 3.0e38f : static_cast<float>(tau);
    c->tune.far_ratio = tau;
    return LF_OK;
}

extern "C" lf_status lf_get_near_pairs(lf_ctx* c, unsigned long long* n) {
    if (!c || !n) return LF_EINVAL;
    if (!c->hasModel) return fail(c, LF_ESTATE, "no model set");
    cudaSetDevice(c->device);
    LF_TRY_CUDA(c, cudaMemcpyAsync(n, c->d_nearPairs.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

extern "C" lf_status lf_set_precision(lf_ctx* c, int mode) {
    if (!c || (mode != LF_PREC_FP64 && mode != LF_PREC_MIXED)) return LF_EINVAL;
    c->epoch++;
    c->precision = mode;
    return LF_OK;
}

// --------------------------------------------------------------- internals --
static constexpr int kFwdThreads = 128;
static constexpr int kFwdFacetTile = 32;
static constexpr int kFacetStage = 32;  // facet records per shared-memory stage of k_forward_mixed
static constexpr int kGradThreads = 32;             // Jacobian rows: one warp of facets per CTA
static constexpr int kGradWarpsPerBlock = 4;        // objective gradient: one warp per facet

// Forward CTAs per launch of the chunked and item schedules; 0 (the mixed
// path's persistent schedule) counts as 148 x 8 there.
static int fwd_blocks(const lf_ctx* c) { return c->tune.fwd_target_blocks > 0 ? c->tune.fwd_target_blocks : 148 * 8; }

// Facet chunks for the forward: contiguous ranges inside one group, sized so
// that station tiles x chunks fill the GPU.
// With c->groupFilter >= 0 only that group's facets are planned (unit
// responses).
static void plan_chunks(lf_ctx* c, int S) {
    if (c->chunkCapacityS == S && c->chunkFilter == c->groupFilter && !c->chunksDirty && !c->chunkBegin.empty())
        return;
    const int g0 = c->groupFilter >= 0 ? c->groupFilter : 0, g1 = c->groupFilter >= 0 ? c->groupFilter + 1 : c->G;
    const int nf = c->grpTriOff[g1] - c->grpTriOff[g0];
    int sBlocks = std::max(1, cdiv(S, kFwdThreads));
    int want = std::max(1, cdiv(fwd_blocks(c), sBlocks));
    int chunkSize = std::max(64, cdiv(std::max(nf, 1), want));
    c->chunkBegin.clear(); c->chunkEnd.clear(); c->chunkGroup.clear();
    for (int g = g0; g < g1; ++g)
        for (int f = c->grpTriOff[g]; f < c->grpTriOff[g + 1]; f += chunkSize) {
            c->chunkBegin.push_back(f);
            c->chunkEnd.push_back(std::min(f + chunkSize, c->grpTriOff[g + 1]));
            c->chunkGroup.push_back(g);
        }
    c->chunkCapacityS = S;
    c->chunkFilter = c->groupFilter;
    c->chunkFacets = nf;
    c->chunksDirty = true;
    c->epoch++;
}

static lf_status upload_chunks(lf_ctx* c) {
    if (!c->chunksDirty) return LF_OK;
    if (!c->chunkBegin.empty()) {
        LF_TRY_CUDA(c, upload(c->d_chunkBegin, c->chunkBegin.data(), c->chunkBegin.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_chunkEnd, c->chunkEnd.data(), c->chunkEnd.size(), c->stream));
        LF_TRY_CUDA(c, upload(c->d_chunkGroup, c->chunkGroup.data(), c->chunkGroup.size(), c->stream));
    }
    c->chunksDirty = false;
    return LF_OK;
}

static lf_status scatter(lf_ctx* c, const double* d_params) {
    if (c->statelessScatter)
        LF_TRY_CUDA(c, cudaMemcpyAsync(c->d_pos.p, c->d_pos0.p, sizeof(double) * 3 * c->V, cudaMemcpyDeviceToDevice,
                                       c->stream));
    if (c->np > 0) {
        k_scatter_dofs<<<cdiv(c->np, 256), 256, 0, c->stream>>>(c->np, d_params, c->d_dofOff.p, c->d_refVertex.p,
                                                                  c->d_refAxis.p, c->d_refScale.p, c->d_pos.p);
        c->counters.launches++;
    }
    if (c->nInterpRows > 0) {
        k_interpolate<<<cdiv(c->nInterpRows, 256), 256, 0, c->stream>>>(c->nInterpRows, c->d_interpRows.p,
                                                                         c->d_interpOff.p, c->d_interpSrc.p,
                                                                         c->d_interpW.p, c->d_pos.p);
        c->counters.launches++;
    }
    if (c->nSync > 0) {
        k_sync_shared<<<cdiv(c->nSync, 256), 256, 0, c->stream>>>(c->nSync, c->d_syncOff.p, c->d_syncVertex.p,
                                                                   c->d_pos.p);
        c->counters.launches++;
    }
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

// Batched bodies: the stations of both data sets are the concatenation of
// per-group station lists (counts[g] stations for group g, in group order);
// each group's facets then see only their own group's stations.  Station
// data must be (re)set after this call.  counts == NULL turns it off.
extern "C" lf_status lf_set_station_groups(lf_ctx* c, int G, const int32_t* counts) {
    if (!c) return LF_EINVAL;
    if (!c->hasModel) return fail(c, LF_ESTATE, "lf_set_station_groups before lf_set_model");
    c->epoch++;
    c->planEpoch++;
    c->grav.n = c->mag.n = 0;
    c->sameStations = false;
    if (!counts) {
        c->partitioned = false;
        return LF_OK;
    }
    if (G != c->G) return fail(c, LF_EINVAL, "lf_set_station_groups: one count per group");
    std::vector<int32_t> off(G + 1, 0);
    int mx = 0;
    for (int g = 0; g < G; ++g) {
        if (counts[g] < 0) return fail(c, LF_EINVAL, "lf_set_station_groups: negative count");
        off[g + 1] = off[g] + counts[g];
        mx = std::max(mx, counts[g]);
    }
    std::vector<int32_t> sg(std::max(off[G], 1), 0);
    for (int g = 0; g < G; ++g)
        for (int i = off[g]; i < off[g + 1]; ++i) sg[i] = g;
    LF_TRY_CUDA(c, upload(c->d_grpStaOff, off.data(), off.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_staGroup, sg.data(), sg.size(), c->stream));
    LF_TRY_CUDA(c, c->d_grpF.reserve(G));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    c->grpStaOff = off;
    c->maxGroupStations = mx;
    c->partitioned = true;
    return LF_OK;
}

extern "C" lf_status lf_get_group_objectives(lf_ctx* c, double* out) {
    if (!c || !out) return LF_EINVAL;
    if (!c->partitioned) return fail(c, LF_ESTATE, "no station groups set");
    LF_TRY_CUDA(c, cudaMemcpyAsync(out, c->d_grpF.p, sizeof(double) * c->G, cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

// Item list of the batched forward: every (group, 128-station block, facet
// chunk), chunk length chosen from the total own-group pairs so that the
// list holds ~32 items per persistent CTA (no item is a large share of a
// CTA's work); ordered by cost, largest first.
static lf_status plan_items(lf_ctx* c) {
    if (c->itemsEpoch == c->planEpoch) return LF_OK;
    const int G = c->G;
    int64_t pairs = 0;
    for (int g = 0; g < G; ++g)
        pairs += (int64_t)(c->grpStaOff[g + 1] - c->grpStaOff[g]) * (c->grpTriOff[g + 1] - c->grpTriOff[g]);
    const int64_t targetItems = 32 * (int64_t)fwd_blocks(c);
    const int64_t F64 = std::max<int64_t>(kFwdFacetTile, (pairs / (128 * targetItems) + 31) / 32 * 32);
    const int F = static_cast<int>(std::min<int64_t>(F64, 1 << 30));
    std::vector<FwdItem> items;
    std::vector<int64_t> partOff(G + 1, 0);
    std::vector<int32_t> nch(G, 0);
    int64_t off = 0;
    for (int g = 0; g < G; ++g) {
        const int sb = c->grpStaOff[g], se = c->grpStaOff[g + 1], Sg = se - sb;
        const int fb = c->grpTriOff[g], Tg = c->grpTriOff[g + 1] - fb;
        partOff[g] = off;
        if (Sg == 0 || Tg == 0) continue;
        nch[g] = cdiv(Tg, F);
        for (int k = 0; k < nch[g]; ++k)
            for (int s0 = sb; s0 < se; s0 += kFwdThreads)
                items.push_back({s0, std::min(se, s0 + kFwdThreads), fb + k * F, std::min(fb + Tg, fb + (k + 1) * F),
                                 off + (int64_t)k * Sg - sb});
        off += (int64_t)nch[g] * Sg;
    }
    partOff[G] = off;
    std::stable_sort(items.begin(), items.end(), [](const FwdItem& a, const FwdItem& b) {
        return (int64_t)(a.s_end - a.s0) * (a.fe - a.fb) > (int64_t)(b.s_end - b.s0) * (b.fe - b.fb);
    });
    if (!items.empty()) LF_TRY_CUDA(c, upload(c->d_items, items.data(), items.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_grpPartOff, partOff.data(), partOff.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_grpNch, nch.data(), nch.size(), c->stream));
    c->nItems = static_cast<int>(items.size());
    c->partTotal = std::max<int64_t>(off, 1);
    c->itemPairs = pairs;
    c->itemsEpoch = c->planEpoch;
    return LF_OK;
}

// Batched forward over one station set (both data types share the groups).
template <bool GZ, bool TMI, bool MIXED>
static lf_status forward_set_items(lf_ctx* c, const StationSet& s, double* d_gz, double* d_tmi) {
    const int S = s.n;
    if (S == 0) return LF_OK;
    LF_RET_IF(plan_items(c));
    if (GZ) LF_TRY_CUDA(c, c->d_partG.reserve((size_t)c->partTotal));
    if (TMI) LF_TRY_CUDA(c, c->d_partM.reserve((size_t)c->partTotal));
    if (c->nItems > 0) {
        const int grid = std::min(c->nItems, fwd_blocks(c));
        int slot = prof_begin(c, c->evFwd, c->nFwd);
        if (MIXED)
            k_forward_mixed_items<GZ, TMI, kFacetStage><<<grid, kFwdThreads, 0, c->stream>>>(
                c->d_items.p, c->nItems, s.d_xyz.p, c->T, c->d_mc.p, c->d_mf32.p, c->tau, GZ ? c->d_partG.p : nullptr,
                TMI ? c->d_partM.p : nullptr, c->d_nearPairs.p);
        else
            k_forward_fp64_items<GZ, TMI, kFwdFacetTile><<<grid, kFwdThreads, 0, c->stream>>>(
                c->d_items.p, c->nItems, s.d_xyz.p, c->T, c->d_fc.p, GZ ? c->d_partG.p : nullptr,
                TMI ? c->d_partM.p : nullptr);
        prof_end(c, c->evFwd, slot);
    }
    k_forward_reduce_groups<<<cdiv(S, 32), 256, 0, c->stream>>>(
        S, c->d_staGroup.p, c->d_grpStaOff.p, c->d_grpPartOff.p, c->d_grpNch.p, MIXED ? nullptr : c->d_groups.p,
        GZ ? c->d_partG.p : nullptr, TMI ? c->d_partM.p : nullptr, GZ ? d_gz : nullptr, TMI ? d_tmi : nullptr);
    c->counters.launches += 2;
    c->counters.forward_pairs += (uint64_t)c->itemPairs;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

template <bool GZ, bool TMI>
static lf_status forward_set(lf_ctx* c, const StationSet& s, double* d_gz, double* d_tmi) {
    if (c->partitioned) return forward_set_items<GZ, TMI, false>(c, s, d_gz, d_tmi);
    int S = s.n;
    if (S == 0) return LF_OK;
    plan_chunks(c, S);
    lf_status st = upload_chunks(c);
    if (st != LF_OK) return st;
    int nch = static_cast<int>(c->chunkBegin.size());
    if (GZ) LF_TRY_CUDA(c, c->d_partG.reserve((size_t)nch * S));
    if (TMI) LF_TRY_CUDA(c, c->d_partM.reserve((size_t)nch * S));
    if (nch > 0) {
        dim3 grid(cdiv(S, kFwdThreads), nch);
        int slot = prof_begin(c, c->evFwd, c->nFwd);
        k_forward_fp64<GZ, TMI, kFwdFacetTile><<<grid, kFwdThreads, 0, c->stream>>>(
            S, s.d_xyz.p, c->T, c->d_fc.p, c->d_chunkBegin.p, c->d_chunkEnd.p, GZ ? c->d_partG.p : nullptr,
            TMI ? c->d_partM.p : nullptr);
        prof_end(c, c->evFwd, slot);
    }
    k_forward_reduce<<<cdiv(S, 32), 256, 0, c->stream>>>(S, nch, c->d_chunkGroup.p, c->d_groups.p,
                                                          GZ ? c->d_partG.p : nullptr, TMI ? c->d_partM.p : nullptr,
                                                          GZ ? d_gz : nullptr, TMI ? d_tmi : nullptr);
    c->counters.launches += 2;
    c->counters.forward_pairs += (uint64_t)S * (uint64_t)c->chunkFacets;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

// Patch chunks of the mixed forward: contiguous patch ranges inside one
// group (patches never cross groups), sized so that station blocks x chunks
// fill the GPU.  Honours c->groupFilter like plan_chunks.
static void plan_patch_chunks(lf_ctx* c, int S) {
    const int NT = c->patchThreads;
    if (c->pchunkS == S && c->pchunkFilter == c->groupFilter && c->pchunkThreads == NT && !c->pchunkBegin.empty())
        return;
    const PatchTopology& pt = c->ptopo;
    const int g0 = c->groupFilter >= 0 ? c->groupFilter : 0, g1 = c->groupFilter >= 0 ? c->groupFilter + 1 : c->G;
    const int np = pt.grpPatchOff[g1] - pt.grpPatchOff[g0];
    const int sBlocks = std::max(1, cdiv(S, NT));
    const int want = std::max(1, cdiv((long long)fwd_blocks(c) * 128 / NT, sBlocks));
    const int per = std::max(1, cdiv(std::max(np, 1), want));
    c->pchunkBegin.clear();
    c->pchunkEnd.clear();
    for (int g = g0; g < g1; ++g)
        for (int q = pt.grpPatchOff[g]; q < pt.grpPatchOff[g + 1]; q += per) {
            c->pchunkBegin.push_back(q);
            c->pchunkEnd.push_back(std::min(q + per, pt.grpPatchOff[g + 1]));
        }
    c->pchunkS = S;
    c->pchunkFilter = c->groupFilter;
    c->pchunkThreads = NT;
    c->pchunkFacets = c->grpTriOff[g1] - c->grpTriOff[g0];
    c->pchunksDirty = true;
    c->epoch++;
}

template <bool GZ, bool TMI, int NT>
static cudaError_t patch_kernel_attrs() {
    static const cudaError_t e = [] {
        cudaError_t a = cudaFuncSetAttribute(k_forward_patch<GZ, TMI, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(PatchSmem<NT>));
        cudaError_t b = cudaFuncSetAttribute(k_forward_patch_items<GZ, TMI, NT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(PatchSmem<NT>));
        cudaError_t d = cudaFuncSetAttribute(k_forward_patch_persistent<GZ, TMI, NT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(PatchSmem<NT>));
        return a != cudaSuccess ? a : (b != cudaSuccess ? b : d);
    }();
    return e;
}

// Per-evaluation records of the mixed forward: the per-facet FP64 / FP32
// records (near and mid facets) and the patch blobs (far facets).
static lf_status mixed_prep(lf_ctx* c) {
    if (c->tune.fwd_engine == LF_FWD_FACET) {
        LF_TRY_CUDA(c, c->d_mf32.reserve((size_t)std::max(c->T, 1)));
        k_face_prep_mixed<<<cdiv(c->T, 128), 128, 0, c->stream>>>(c->T, c->d_tri.p, c->d_pos.p, c->d_faceGroup.p,
                                                                  c->d_groups.p, c->fdir, c->d_mc.p, c->d_mf32.p,
                                                                  c->dropCollapsed);
        c->counters.launches++;
        LF_CHECK_LAUNCH(c);
        return LF_OK;
    }
    const PatchTopology& pt = c->ptopo;
    k_face_prep_patch<<<cdiv(c->T, 128), 128, 0, c->stream>>>(
        c->T, c->d_tri.p, c->d_pos.p, c->d_faceGroup.p, c->d_groups.p, c->fdir, c->d_pFacetPatch.p, c->d_pFacetSlot.p,
        c->d_pFacetOff.p, c->d_pCorners.p, c->d_pVertOff.p, c->d_pVerts.p, c->d_pEdgeOff.p, c->d_pBlobOff.p,
        c->d_mc.p, c->d_mt2.p, c->d_blobs.p, c->dropCollapsed);
    if (pt.P > 0)
        k_patch_prep<<<pt.P, 32, 0, c->stream>>>(pt.P, c->d_pos.p, c->d_pFacetOff.p, c->d_pFacets.p, c->d_pVertOff.p,
                                                  c->d_pVerts.p, c->d_pEdgeOff.p, c->d_pEdgeInfo.p, c->d_pEdgeSlot.p,
                                                  c->d_pBlobOff.p, c->T, c->d_mt2.p, c->d_blobs.p);
    c->counters.launches += pt.P > 0 ? 2 : 1;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

// Item list of the batched patch forward: (group, station block of NT,
// patch range) with about 32 items per persistent CTA, largest first.
static lf_status plan_patch_items(lf_ctx* c) {
    const int NT = c->patchThreads;
    if (c->pItemsEpoch == c->planEpoch && c->pItemsThreads == NT) return LF_OK;
    const int G = c->G;
    const PatchTopology& pt = c->ptopo;
    int64_t pairs = 0;
    for (int g = 0; g < G; ++g)
        pairs += (int64_t)(c->grpStaOff[g + 1] - c->grpStaOff[g]) * (c->grpTriOff[g + 1] - c->grpTriOff[g]);
    const int64_t targetItems = 32 * (int64_t)fwd_blocks(c) * 128 / NT;
    const double facetsPerPatch = pt.P > 0 ? (double)c->T / pt.P : 1.0;
    const int per = (int)std::max<int64_t>(1, (int64_t)((double)pairs / ((double)NT * targetItems * facetsPerPatch)));
    std::vector<FwdItem> items;
    std::vector<int64_t> partOff(G + 1, 0);
    std::vector<int32_t> nch(G, 0);
    int64_t off = 0;
    for (int g = 0; g < G; ++g) {
        const int sb = c->grpStaOff[g], se = c->grpStaOff[g + 1], Sg = se - sb;
        const int pb = pt.grpPatchOff[g], Pg = pt.grpPatchOff[g + 1] - pb;
        partOff[g] = off;
        if (Sg == 0 || Pg == 0) continue;
        nch[g] = cdiv(Pg, per);
        for (int k = 0; k < nch[g]; ++k)
            for (int s0 = sb; s0 < se; s0 += NT)
                items.push_back({s0, std::min(se, s0 + NT), pb + k * per, std::min(pb + Pg, pb + (k + 1) * per),
                                 off + (int64_t)k * Sg - sb});
        off += (int64_t)nch[g] * Sg;
    }
    partOff[G] = off;
    std::vector<int64_t> cost(items.size());
    std::vector<size_t> order(items.size());
    for (size_t i = 0; i < items.size(); ++i) {
        const FwdItem& w = items[i];
        cost[i] = (int64_t)(w.s_end - w.s0) * (pt.facetOff[w.fe] - pt.facetOff[w.fb]);
        order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
    std::vector<FwdItem> sorted(items.size());
    for (size_t i = 0; i < items.size(); ++i) sorted[i] = items[order[i]];
    if (!sorted.empty()) LF_TRY_CUDA(c, upload(c->d_pItems, sorted.data(), sorted.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_pGrpPartOff, partOff.data(), partOff.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_pGrpNch, nch.data(), nch.size(), c->stream));
    c->npItems = static_cast<int>(sorted.size());
    c->pPartTotal = std::max<int64_t>(off, 1);
    c->pItemPairs = pairs;
    c->pItemsEpoch = c->planEpoch;
    c->pItemsThreads = NT;
    c->epoch++;
    return LF_OK;
}

template <bool GZ, bool TMI, int NT>
static lf_status launch_patch_items(lf_ctx* c, const StationSet& s, int grid) {
    LF_TRY_CUDA(c, (patch_kernel_attrs<GZ, TMI, NT>()));
    k_forward_patch_items<GZ, TMI, NT><<<grid, NT, sizeof(PatchSmem<NT>), c->stream>>>(
        c->d_pItems.p, c->npItems, s.d_xyz.p, c->d_blobs.p, c->d_pBlobOff.p, c->d_mc.p, c->T, c->tau,
        GZ ? c->d_partG.p : nullptr, TMI ? c->d_partM.p : nullptr, c->d_nearPairs.p, c->d_patchErr.p);
    return LF_OK;
}

template <bool GZ, bool TMI>
static lf_status forward_set_patch_items(lf_ctx* c, const StationSet& s, double* d_gz, double* d_tmi) {
    const int S = s.n;
    if (S == 0) return LF_OK;
    LF_RET_IF(plan_patch_items(c));
    if (GZ) LF_TRY_CUDA(c, c->d_partG.reserve((size_t)c->pPartTotal));
    if (TMI) LF_TRY_CUDA(c, c->d_partM.reserve((size_t)c->pPartTotal));
    if (c->npItems > 0) {
        const int grid = std::min(c->npItems, fwd_blocks(c) * 128 / c->patchThreads);
        int slot = prof_begin(c, c->evFwd, c->nFwd);
        if (c->patchThreads == 256)
            LF_RET_IF((launch_patch_items<GZ, TMI, 256>(c, s, grid)));
        else
            LF_RET_IF((launch_patch_items<GZ, TMI, 128>(c, s, grid)));
        prof_end(c, c->evFwd, slot);
    }
    k_forward_reduce_groups<<<cdiv(S, 32), 256, 0, c->stream>>>(
        S, c->d_staGroup.p, c->d_grpStaOff.p, c->d_pGrpPartOff.p, c->d_pGrpNch.p, nullptr,
        GZ ? c->d_partG.p : nullptr, TMI ? c->d_partM.p : nullptr, GZ ? d_gz : nullptr, TMI ? d_tmi : nullptr);
    c->counters.launches += 2;
    c->counters.forward_pairs += (uint64_t)c->pItemPairs;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

template <bool GZ, bool TMI, int NT>
static lf_status launch_patch(lf_ctx* c, const StationSet& s, int nch) {
    LF_TRY_CUDA(c, (patch_kernel_attrs<GZ, TMI, NT>()));
    dim3 grid(cdiv(s.n, NT), nch);
    k_forward_patch<GZ, TMI, NT><<<grid, NT, sizeof(PatchSmem<NT>), c->stream>>>(
        s.n, s.d_xyz.p, c->d_blobs.p, c->d_pBlobOff.p, c->d_pChunkBegin.p, c->d_pChunkEnd.p, c->d_mc.p, c->T, c->tau, GZ ? c->d_partG.p : nullptr, TMI ? c->d_partM.p : nullptr, c->d_nearPairs.p, c->d_patchErr.p);
    return LF_OK;
}

// Persistent schedule: one CTA per resident slot on the device, each over a
// balanced contiguous range of (station block, patch) units.
template <bool GZ, bool TMI, int NT>
static lf_status forward_patch_persistent(lf_ctx* c, const StationSet& s, double* d_gz, double* d_tmi) {
    LF_TRY_CUDA(c, (patch_kernel_attrs<GZ, TMI, NT>()));
    static int occupancy = 0, sms = 0;
    if (!occupancy) {
        LF_TRY_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy, k_forward_patch_persistent<GZ, TMI, NT>,
                                                                     NT, sizeof(PatchSmem<NT>)));
        LF_TRY_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        occupancy = std::max(occupancy, 1);
    }
    const int S = s.n;
    const PatchTopology& pt = c->ptopo;
    const int g0 = c->groupFilter >= 0 ? c->groupFilter : 0, g1 = c->groupFilter >= 0 ? c->groupFilter + 1 : c->G;
    const int pbase = pt.grpPatchOff[g0], P = pt.grpPatchOff[g1] - pbase;
    const int NB = cdiv(S, NT);
    const long long nunits = (long long)NB * P;
    if (nunits == 0) return LF_OK;
    const int G = (int)std::min<long long>((long long)occupancy * sms, nunits);
    const long long key = ((((long long)S * 1000003 + P) * 131 + pbase) * 4099 + G) * 3 + (NT == 256);
    if (key != c->pPersistKey) {
        std::vector<int32_t> nch(NB);
        int mx = 1;
        auto owner = [&](long long u) { return static_cast<int>(((u + 1) * G - 1) / nunits); };
        for (int b = 0; b < NB; ++b) {
            nch[b] = owner((long long)b * P + P - 1) - owner((long long)b * P) + 1;
            mx = std::max(mx, nch[b]);
        }
        LF_TRY_CUDA(c, upload(c->d_pBlockNch, nch.data(), nch.size(), c->stream));
        c->pPersistKey = key;
        c->pPersistSlots = mx;
        c->pPersistGrid = G;
        c->epoch++;
    }
    if (GZ) LF_TRY_CUDA(c, c->d_partG.reserve((size_t)c->pPersistSlots * S));
    if (TMI) LF_TRY_CUDA(c, c->d_partM.reserve((size_t)c->pPersistSlots * S));
    int slot = prof_begin(c, c->evFwd, c->nFwd);
    k_forward_patch_persistent<GZ, TMI, NT><<<G, NT, sizeof(PatchSmem<NT>), c->stream>>>(
        S, s.d_xyz.p, c->d_blobs.p, c->d_pBlobOff.p, pbase, P, nunits, c->d_mc.p, c->T, c->tau,
        GZ ? c->d_partG.p : nullptr, TMI ? c->d_partM.p : nullptr, c->d_nearPairs.p, c->d_patchErr.p);
    prof_end(c, c->evFwd, slot);
    k_forward_reduce_mixed<<<cdiv(S, 32), 256, 0, c->stream>>>(S, c->pPersistSlots, GZ ? c->d_partG.p : nullptr,
                                                                TMI ? c->d_partM.p : nullptr, GZ ? d_gz : nullptr,
                                                                TMI ? d_tmi : nullptr, c->d_pBlockNch.p, NT);
    c->counters.launches += 2;
    c->counters.forward_pairs += (uint64_t)S * (uint64_t)(c->grpTriOff[g1] - c->grpTriOff[g0]);
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

template <bool GZ, bool TMI>
static lf_status forward_set_facet(lf_ctx* c, const StationSet& s, double* d_gz, double* d_tmi) {
    if (c->partitioned) return forward_set_items<GZ, TMI, true>(c, s, d_gz, d_tmi);
    int S = s.n;
    if (S == 0) return LF_OK;
    plan_chunks(c, S);
    LF_RET_IF(upload_chunks(c));
    int nch = static_cast<int>(c->chunkBegin.size());
    if (GZ) LF_TRY_CUDA(c, c->d_partG.reserve((size_t)nch * S));
    if (TMI) LF_TRY_CUDA(c, c->d_partM.reserve((size_t)nch * S));
    if (nch > 0) {
        dim3 grid(cdiv(S, kFwdThreads), nch);
        int slot = prof_begin(c, c->evFwd, c->nFwd);
        k_forward_mixed<GZ, TMI, kFacetStage><<<grid, kFwdThreads, 0, c->stream>>>(
            S, s.d_xyz.p, c->T, c->d_mc.p, c->d_mf32.p, c->d_chunkBegin.p, c->d_chunkEnd.p, c->tau,
            GZ ? c->d_partG.p : nullptr, TMI ? c->d_partM.p : nullptr, c->d_nearPairs.p);
        prof_end(c, c->evFwd, slot);
    }
    k_forward_reduce_mixed<<<cdiv(S, 32), 256, 0, c->stream>>>(S, nch, GZ ? c->d_partG.p : nullptr,
                                                                TMI ? c->d_partM.p : nullptr, GZ ? d_gz : nullptr,
                                                                TMI ? d_tmi : nullptr);
    c->counters.launches += 2;
    c->counters.forward_pairs += (uint64_t)S * (uint64_t)c->chunkFacets;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

template <bool GZ, bool TMI>
static lf_status forward_set_mixed(lf_ctx* c, const StationSet& s, double* d_gz, double* d_tmi) {
    if (c->tune.fwd_engine == LF_FWD_FACET) return forward_set_facet<GZ, TMI>(c, s, d_gz, d_tmi);
    if (c->partitioned) return forward_set_patch_items<GZ, TMI>(c, s, d_gz, d_tmi);
    int S = s.n;
    if (S == 0) return LF_OK;
    if (c->tune.fwd_target_blocks == 0)
        return c->patchThreads == 256 ? forward_patch_persistent<GZ, TMI, 256>(c, s, d_gz, d_tmi)
                                      : forward_patch_persistent<GZ, TMI, 128>(c, s, d_gz, d_tmi);
    plan_patch_chunks(c, S);
    if (c->pchunksDirty) {
        if (!c->pchunkBegin.empty()) {
            LF_TRY_CUDA(c, upload(c->d_pChunkBegin, c->pchunkBegin.data(), c->pchunkBegin.size(), c->stream));
            LF_TRY_CUDA(c, upload(c->d_pChunkEnd, c->pchunkEnd.data(), c->pchunkEnd.size(), c->stream));
        }
        c->pchunksDirty = false;
    }
    int nch = static_cast<int>(c->pchunkBegin.size());
    if (GZ) LF_TRY_CUDA(c, c->d_partG.reserve((size_t)nch * S));
    if (TMI) LF_TRY_CUDA(c, c->d_partM.reserve((size_t)nch * S));
    if (nch > 0) {
        int slot = prof_begin(c, c->evFwd, c->nFwd);
        if (c->patchThreads == 256)
            LF_RET_IF((launch_patch<GZ, TMI, 256>(c, s, nch)));
        else
            LF_RET_IF((launch_patch<GZ, TMI, 128>(c, s, nch)));
        prof_end(c, c->evFwd, slot);
    }
    k_forward_reduce_mixed<<<cdiv(S, 32), 256, 0, c->stream>>>(S, nch, GZ ? c->d_partG.p : nullptr,
                                                                TMI ? c->d_partM.p : nullptr, GZ ? d_gz : nullptr,
                                                                TMI ? d_tmi : nullptr);
    c->counters.launches += 2;
    c->counters.forward_pairs += (uint64_t)S * (uint64_t)c->pchunkFacets;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

// Positions must be current.  Writes grav.d_pred / mag.d_pred.
static lf_status forward_all(lf_ctx* c) {
    if (c->precision == LF_PREC_MIXED) {
        LF_RET_IF(mixed_prep(c));
        if (c->sameStations) return forward_set_mixed<true, true>(c, c->grav, c->grav.d_pred.p, c->mag.d_pred.p);
        lf_status st = forward_set_mixed<true, false>(c, c->grav, c->grav.d_pred.p, nullptr);
        if (st != LF_OK) return st;
        return forward_set_mixed<false, true>(c, c->mag, nullptr, c->mag.d_pred.p);
    }
    k_face_prep_fwd<<<cdiv(c->T, 128), 128, 0, c->stream>>>(c->T, c->d_tri.p, c->d_pos.p, c->d_faceGroup.p,
                                                            c->d_groups.p, c->fdir, c->d_fc.p,
                                                            c->dropCollapsed);
    c->counters.launches++;
    LF_CHECK_LAUNCH(c);
    if (c->sameStations) return forward_set<true, true>(c, c->grav, c->grav.d_pred.p, c->mag.d_pred.p);
    lf_status st = forward_set<true, false>(c, c->grav, c->grav.d_pred.p, nullptr);
    if (st != LF_OK) return st;
    return forward_set<false, true>(c, c->mag, nullptr, c->mag.d_pred.p);
}

static lf_status residuals(lf_ctx* c, bool wantCoef) {
    int nbg = cdiv(std::max(c->grav.n, 1), 256), nbm = cdiv(std::max(c->mag.n, 1), 256);
    LF_TRY_CUDA(c, c->d_blockG.reserve(nbg));
    LF_TRY_CUDA(c, c->d_blockM.reserve(nbm));
    if (c->grav.n > 0)
        k_residual<<<nbg, 256, 0, c->stream>>>(c->grav.n, c->grav.d_pred.p, c->grav.d_obs.p, c->grav.d_w.p, 1.0,
                                               wantCoef ? c->grav.d_coef.p : nullptr, c->d_blockG.p);
    else
        LF_TRY_CUDA(c, cudaMemsetAsync(c->d_blockG.p, 0, sizeof(double) * nbg, c->stream));
    bool magOn = c->mag.n > 0 && c->alphaMag > 0.0;  // joint_objective.cpp:48, :123
    if (magOn)
        k_residual<<<nbm, 256, 0, c->stream>>>(c->mag.n, c->mag.d_pred.p, c->mag.d_obs.p, c->mag.d_w.p, c->alphaMag,
                                               wantCoef ? c->mag.d_coef.p : nullptr, c->d_blockM.p);
    else
        LF_TRY_CUDA(c, cudaMemsetAsync(c->d_blockM.p, 0, sizeof(double) * nbm, c->stream));
    c->counters.launches += 2;
    if (c->partitioned) {  // per-body data misfit (lf_get_group_objectives)
        const bool g = c->grav.n > 0;
        k_group_misfit<<<c->G, 256, 0, c->stream>>>(c->G, c->d_grpStaOff.p, g ? c->grav.d_pred.p : nullptr,
                                                     g ? c->grav.d_obs.p : nullptr, g ? c->grav.d_w.p : nullptr,
                                                     magOn ? c->mag.d_pred.p : nullptr,
                                                     magOn ? c->mag.d_obs.p : nullptr,
                                                     magOn ? c->mag.d_w.p : nullptr, c->alphaMag, c->d_grpF.p);
        c->counters.launches++;
    }
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

static lf_status objective_final(lf_ctx* c, const double* d_params, double* d_f) {
    int nbg = cdiv(std::max(c->grav.n, 1), 256), nbm = cdiv(std::max(c->mag.n, 1), 256);
    k_objective_final<<<1, 256, 0, c->stream>>>(nbg, c->d_blockG.p, nbm, c->d_blockM.p, c->alphaMag, c->np, d_params,
                                                c->hasRef ? c->d_refp.p : nullptr, c->refWeight, cdiv(c->V, 256),
                                                c->smoothOn ? c->d_blockS.p : nullptr, c->smoothWeight, c->d_out5.p,
                                                d_f);
    c->counters.launches++;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

// Gradient kernels over one station set with the given adjoints; writes
// facet partial slot `slot` of d_partGrad ([slot][9][T]).  FP64 mode: one
// FP64 kernel over every (facet, station) pair.  Mixed mode: the FP64 kernel
// takes each facet's near station tiles and the FP32 far-field kernel the
// rest, writing slot + 1.  Returns the number of slots written.
// Station chunks of a gradient grid, whole tiles per chunk: enough chunks
// for tune.grad_target_warps warps (facets with a DOF vertex x chunks).  The
// mixed near-field kernel, whose work sits in few (facet, tile) places, may
// instead take tune.near_tiles_per_chunk tiles per chunk (0: as above).
static void grad_chunks(lf_ctx* c, int S, bool nearOnly, int* nchunks, int* tilesPerChunk) {
    const int ntiles = std::max(1, cdiv(S, kStationTile));
    if (c->partitioned) {  // batched bodies: one chunk covering the largest body's tiles
        *tilesPerChunk = std::max(1, cdiv(c->maxGroupStations, kStationTile));
        *nchunks = 1;
        return;
    }
    if (nearOnly && c->tune.near_tiles_per_chunk > 0) {
        *tilesPerChunk = std::min(c->tune.near_tiles_per_chunk, ntiles);
    } else {
        const int want = std::max(1, cdiv(c->tune.grad_target_warps, std::max(c->nGradFacets, 1)));
        *tilesPerChunk = cdiv(ntiles, std::min(want, ntiles));
    }
    *nchunks = cdiv(ntiles, *tilesPerChunk);
}

// Partial slots one station set takes (see gradient_set).
static int grad_slots(lf_ctx* c, int S) {
    int n1 = 1, n2 = 1, t = 1;
    if (c->precision == LF_PREC_MIXED) {
        grad_chunks(c, S, true, &n1, &t);
        grad_chunks(c, S, false, &n2, &t);
        return n1 + n2;
    }
    grad_chunks(c, S, false, &n1, &t);
    return n1;
}

// Gradient kernels over one station set with the given adjoints; writes
// facet partial slots [slot0, slot0 + returned count) of d_partGrad
// ([slot][9][T], one slot per (kernel, station chunk)).
static int gradient_set(lf_ctx* c, const StationSet& s, const double* gcoef, const double* mcoef, int slot0) {
    if (s.n == 0 || c->nGradFacets == 0) return 0;
    const bool mixed = c->precision == LF_PREC_MIXED;
    const double tau = mixed ? static_cast<double>(c->tau) : 3.0e38;
    int nch = 1, tpc = 1;
    grad_chunks(c, s.n, mixed, &nch, &tpc);
    const int32_t* grpSta = c->partitioned ? c->d_grpStaOff.p : nullptr;
    const int32_t* grpTile = c->partitioned ? c->d_grpTileOff.p : nullptr;
    const int fblocks = cdiv(c->nGradFacets, kGradWarpsPerBlock);
    // Mixed precision: the far-field kernel on the side stream, concurrent
    // with the near-field one (they write disjoint partial slots).  Serial
    // when the kernels are timed one by one (profiling).
    bool fork = mixed && c->side && !c->profiling;
    if (fork && (cudaEventRecord(c->evFork, c->stream) != cudaSuccess ||
                 cudaStreamWaitEvent(c->side, c->evFork, 0) != cudaSuccess)) {
        cudaGetLastError();
        fork = false;
    }
    int ev = prof_begin(c, c->evGrad, c->nGrad);
    k_gradient_warp_fp64<<<dim3(fblocks, nch), 32 * kGradWarpsPerBlock, 0, c->stream>>>(
        c->T, c->d_gc.p, s.n, s.d_xyz.p, gcoef, mcoef, s.d_tileBox.p, c->d_faceGroup.p, c->d_groups.p, c->fdir, tau,
        c->d_gradFacets.p, c->nGradFacets, tpc, grpSta, grpTile, c->d_partGrad.p + (size_t)slot0 * 9 * c->T);
    prof_end(c, c->evGrad, ev);
    c->counters.launches++;
    int used = nch;
    if (mixed) {
        int nch2 = 1, tpc2 = 1;
        grad_chunks(c, s.n, false, &nch2, &tpc2);
        int ev2 = prof_begin(c, c->evGrad, c->nGrad);
        k_gradient_warp_far32<<<dim3(fblocks, nch2), 32 * kGradWarpsPerBlock, 0, fork ? c->side : c->stream>>>(
            c->T, c->d_gc.p, s.n, s.d_xyz.p, gcoef, mcoef, s.d_tileBox.p, c->d_faceGroup.p, c->d_groups.p, c->fdir,
            tau, c->d_gradFacets.p, c->nGradFacets, tpc2, grpSta, grpTile,
            c->d_partGrad.p + (size_t)(slot0 + nch) * 9 * c->T);
        prof_end(c, c->evGrad, ev2);
        if (fork) {  // join: the main stream waits for the far-field kernel
            cudaEventRecord(c->evJoin, c->side);
            cudaStreamWaitEvent(c->stream, c->evJoin, 0);
        }
        c->counters.launches++;
        used += nch2;
    }
    if (c->partitioned) {
        for (int32_t f : c->hGradFacets) {
            const int g = static_cast<int>(std::upper_bound(c->grpTriOff.begin(), c->grpTriOff.end(), f) -
                                           c->grpTriOff.begin()) - 1;
            c->counters.gradient_pairs += (uint64_t)(c->grpStaOff[g + 1] - c->grpStaOff[g]);
        }
    } else {
        c->counters.gradient_pairs += (uint64_t)s.n * (uint64_t)c->nGradFacets;
    }
    return used;
}

// Finite-difference-XY partials of one station set into slots
// [slot0, slot0 + returned count): the FP64 chunking of the analytic kernels.
static int gradient_fdxy_set(lf_ctx* c, const StationSet& s, const double* gcoef, const double* mcoef, int slot0) {
    if (s.n == 0 || c->nGradFacets == 0) return 0;
    int nch = 1, tpc = 1;
    grad_chunks(c, s.n, false, &nch, &tpc);
    const int32_t* grpSta = c->partitioned ? c->d_grpStaOff.p : nullptr;
    k_gradient_fdxy<<<dim3(cdiv(c->nGradFacets, 4), nch), 128, 0, c->stream>>>(
        c->T, c->nGradFacets, c->d_gradFacets.p, c->d_fcfd.p, c->d_gc.p, s.n, s.d_xyz.p, gcoef, mcoef,
        c->d_faceGroup.p, 1.0 / c->xyStep, tpc, grpSta, c->d_partGrad.p + (size_t)slot0 * 9 * c->T);
    c->counters.launches++;
    return nch;
}

static lf_status gradient_all(lf_ctx* c, const double* d_params, double* d_grad) {
    bool gOn = c->grav.n > 0, mOn = c->mag.n > 0 && c->alphaMag > 0.0;
    k_face_prep_grad<<<cdiv(c->T, 128), 128, 0, c->stream>>>(c->T, c->d_tri.p, c->d_pos.p, c->d_faceGroup.p,
                                                             c->d_groups.p, c->d_faceNeeds.p, 1, 1, c->fdir,
                                                             c->d_gc.p);
    c->counters.launches++;
    LF_CHECK_LAUNCH(c);
    int slots = 0;
    if (c->sameStations && gOn) {
        slots = grad_slots(c, c->grav.n);
    } else {
        if (gOn) slots += grad_slots(c, c->grav.n);
        if (mOn) slots += grad_slots(c, c->mag.n);
    }
    if (c->nGradFacets == 0) slots = 0;
    const bool fdxy = c->xyMode == LF_XY_FORWARD_DIFFERENCE && slots > 0;
    if (fdxy) {  // one FP64 finite-difference slot per station chunk
        int n = 1, t = 1;
        if (c->sameStations && gOn) {
            grad_chunks(c, c->grav.n, false, &n, &t);
            slots += n;
        } else {
            if (gOn) { grad_chunks(c, c->grav.n, false, &n, &t); slots += n; }
            if (mOn) { grad_chunks(c, c->mag.n, false, &n, &t); slots += n; }
        }
    }
    if (slots == 0) {
        LF_TRY_CUDA(c, cudaMemsetAsync(c->d_vgrad.p, 0, sizeof(double) * 3 * c->V, c->stream));
    } else {
        LF_TRY_CUDA(c, c->d_partGrad.reserve((size_t)slots * 9 * c->T));
        int used = 0;
        if (c->sameStations && gOn) {
            used += gradient_set(c, c->grav, c->grav.d_coef.p, mOn ? c->mag.d_coef.p : nullptr, used);
        } else {
            if (gOn) used += gradient_set(c, c->grav, c->grav.d_coef.p, nullptr, used);
            if (mOn) used += gradient_set(c, c->mag, nullptr, c->mag.d_coef.p, used);
        }
        const int fdFrom = used;
        if (fdxy) {
            const int nf = c->nGradFacets;
            LF_TRY_CUDA(c, c->d_fcfd.reserve((size_t)7 * NFC * nf));
            k_face_prep_fdxy<<<dim3(cdiv(nf, 128), 7), 128, 0, c->stream>>>(nf, c->d_gradFacets.p, c->d_tri.p,
                                                                           c->d_pos.p, c->d_faceGroup.p,
                                                                           c->d_groups.p, c->fdir, c->xyStep,
                                                                           c->d_fcfd.p);
            c->counters.launches++;
            if (c->sameStations && gOn) {
                used += gradient_fdxy_set(c, c->grav, c->grav.d_coef.p, mOn ? c->mag.d_coef.p : nullptr, used);
            } else {
                if (gOn) used += gradient_fdxy_set(c, c->grav, c->grav.d_coef.p, nullptr, used);
                if (mOn) used += gradient_fdxy_set(c, c->mag, nullptr, c->mag.d_coef.p, used);
            }
        }
        LF_CHECK_LAUNCH(c);
        if (c->nGradVerts > 0) {
            k_vertex_reduce<<<cdiv(c->nGradVerts, 4), 128, 0, c->stream>>>(c->nGradVerts, c->d_gradVerts.p,
                                                                              c->d_vfOff.p, c->d_vf.p, c->T, used,
                                                                              fdFrom, c->d_partGrad.p, c->d_vgrad.p);
            c->counters.launches++;
        }
    }
    if (c->smoothOn) {
        k_smooth_vgrad<<<cdiv(c->V, 256), 256, 0, c->stream>>>(c->V, c->d_freedom.p, c->d_smOff.p, c->d_smNbr.p,
                                                               c->d_smDiff.p, c->d_smVgrad.p);
        c->counters.launches++;
    }
    const double* vg = c->d_vgrad.p;
    bool smoothInGather = c->smoothOn;
    if (c->gatherMode == LF_GATHER_CHAIN && c->np > 0) {
        if (c->smoothOn) {
            k_axpy<<<cdiv(3LL * c->V, 256), 256, 0, c->stream>>>((size_t)3 * c->V, c->smoothWeight, c->d_smVgrad.p,
                                                                 c->d_vgrad.p);
            c->counters.launches++;
            smoothInGather = false;
        }
        if (c->nSync > 0) {
            k_sync_shared<<<cdiv(c->nSync, 256), 256, 0, c->stream>>>(c->nSync, c->d_syncOff.p, c->d_syncVertex.p,
                                                                       c->d_vgrad.p);
            c->counters.launches++;
        }
        if (c->nInterpRows > 0) {
            k_interp_adjoint<<<cdiv(c->V, 256), 256, 0, c->stream>>>(c->V, c->d_interpOff.p, c->d_adjOff.p,
                                                                     c->d_adjRow.p, c->d_adjW.p, c->d_vgrad.p,
                                                                     c->d_vgrad2.p);
            c->counters.launches++;
            vg = c->d_vgrad2.p;
        }
    }
    if (c->np > 0) {
        k_dof_gather<<<cdiv(c->np, 256), 256, 0, c->stream>>>(c->np, c->d_dofOff.p, c->d_refVertex.p, c->d_refAxis.p,
                                                              c->d_refScale.p, vg, d_params,
                                                              c->hasRef ? c->d_refp.p : nullptr, c->refWeight,
                                                              smoothInGather ? c->d_smVgrad.p : nullptr,
                                                              c->smoothWeight, d_grad);
        c->counters.launches++;
    }
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

__global__ void k_unpermute(int n, const int32_t* __restrict__ perm, const double* __restrict__ src,
                            double* __restrict__ dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[perm[i]] = src[i];
}

// Device predictions (Morton slot order) -> caller order.
static lf_status unpermute_device(lf_ctx* c, const StationSet& s, const double* src, double* dst) {
    if (s.n == 0) return LF_OK;
    k_unpermute<<<cdiv(s.n, 256), 256, 0, c->stream>>>(s.n, s.d_perm.p, src, dst);
    c->counters.launches++;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

static lf_status check_ready(lf_ctx* c) {
    if (!c) return LF_EINVAL;
    if (!c->hasModel) return fail(c, LF_ESTATE, "no model set");
    if (c->grav.n == 0 && c->mag.n == 0) return fail(c, LF_ESTATE, "no station data set");
    cudaSetDevice(c->device);
    return LF_OK;
}

static lf_status params_to_device(lf_ctx* c, const double* params) {
    if (c->np > 0 && !params) return fail(c, LF_EINVAL, "null params");
    if (!finite_all(params, c->np)) return fail(c, LF_EINVAL, "non-finite parameter");
    if (c->np > 0)
        LF_TRY_CUDA(c, cudaMemcpyAsync(c->d_params.p, params, sizeof(double) * c->np, cudaMemcpyHostToDevice, c->stream));
    return LF_OK;
}


// ------------------------------------------------------------ public API --
extern "C" lf_status lf_forward_device(lf_ctx* c, const double* d_params, double* d_gz, double* d_tmi) {
    LF_RET_IF(check_ready(c));
    LF_RET_IF(scatter(c, d_params));
    LF_RET_IF(forward_all(c));
    if (d_gz && c->grav.n) LF_RET_IF(unpermute_device(c, c->grav, c->grav.d_pred.p, d_gz));
    if (d_tmi && c->mag.n) LF_RET_IF(unpermute_device(c, c->mag, c->mag.d_pred.p, d_tmi));
    return LF_OK;
}

extern "C" lf_status lf_forward(lf_ctx* c, const double* params, double* gz, double* tmi) {
    LF_RET_IF(check_ready(c));
    LF_RET_IF(params_to_device(c, params));
    LF_RET_IF(scatter(c, c->d_params.p));
    LF_RET_IF(forward_all(c));
    if (gz && c->grav.n) {
        LF_RET_IF(unpermute_device(c, c->grav, c->grav.d_pred.p, c->grav.d_out.p));
        LF_TRY_CUDA(c, cudaMemcpyAsync(gz, c->grav.d_out.p, sizeof(double) * c->grav.n, cudaMemcpyDeviceToHost, c->stream));
    }
    if (tmi && c->mag.n) {
        LF_RET_IF(unpermute_device(c, c->mag, c->mag.d_pred.p, c->mag.d_out.p));
        LF_TRY_CUDA(c, cudaMemcpyAsync(tmi, c->mag.d_out.p, sizeof(double) * c->mag.n, cudaMemcpyDeviceToHost, c->stream));
    }
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

// Runs `body` (a whole evaluation enqueued on c->stream) directly, or, in
// graph mode, replays a CUDA graph of it.  A cache miss runs the body eagerly
// -- which also sizes every buffer and uploads every table -- and then
// captures the same launch sequence for the next call.  A capture that fails
// is not an error (the eager run already produced the result); it is not
// retried until a setter changes the context.
template <class Body>
static lf_status run_cached(lf_ctx* c, lf_ctx::GraphSet& set, const double* p, double* f, double* grad, Body body,
                            bool always = false) {
    if ((!c->graphMode && !always) || c->profiling) return body();
    for (auto& g : set.slot)
        if (g.exec && g.epoch == c->epoch && g.reallocs == reallocAll() && g.params == p && g.f == f &&
            g.grad == grad) {
            LF_TRY_CUDA(c, cudaGraphLaunch(g.exec, c->stream));
            c->counters.forward_pairs += g.delta.forward_pairs;
            c->counters.gradient_pairs += g.delta.gradient_pairs;
            c->counters.launches += g.delta.launches;
            return LF_OK;
        }
    LF_RET_IF(body());
    if (set.failedEpoch == c->epoch) return LF_OK;
    // slots captured under an older epoch or allocation state are stale
    for (auto& g : set.slot)
        if (g.exec && (g.epoch != c->epoch || g.reallocs != reallocAll())) {
            cudaGraphExecDestroy(g.exec);
            g = lf_ctx::GraphCache{};
        }
    lf_ctx::GraphCache& g = set.slot[set.next];
    set.next = (set.next + 1) % lf_ctx::kGraphSlots;
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = lf_ctx::GraphCache{};
    const lf_counters before = c->counters;
    const uint64_t epoch0 = c->epoch, realloc0 = reallocAll();
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        set.failedEpoch = c->epoch;
        return LF_OK;
    }
    const lf_status cst = body();
    const cudaError_t ee = cudaStreamEndCapture(c->stream, &graph);
    const lf_counters after = c->counters;
    c->counters = before;  // a capture executes nothing
    bool ok = cst == LF_OK && ee == cudaSuccess && graph && c->epoch == epoch0 && reallocAll() == realloc0;
    cudaGraphExec_t exec = nullptr;
    if (ok && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) ok = false;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
        if (exec) cudaGraphExecDestroy(exec);
        cudaGetLastError();
        set.failedEpoch = c->epoch;
        return LF_OK;
    }
    g.exec = exec;
    g.epoch = c->epoch;
    g.reallocs = reallocAll();
    g.params = p;
    g.f = f;
    g.grad = grad;
    g.delta = {after.forward_pairs - before.forward_pairs, after.gradient_pairs - before.gradient_pairs,
               after.launches - before.launches};
    return LF_OK;
}

extern "C" lf_status lf_set_tuning(lf_ctx* c, const lf_tuning* t) {
    if (!c || !t || t->fwd_target_blocks < 0 || t->grad_target_warps < 1 || t->near_tiles_per_chunk < 0 ||
        (t->patch_threads != 128 && t->patch_threads != 256) || !std::isfinite(t->far_ratio) ||
        (t->fwd_engine != LF_FWD_FACET && t->fwd_engine != LF_FWD_PATCH))
        return LF_EINVAL;
    c->epoch++;
    c->tune = *t;
    c->patchThreads = t->patch_threads;
    c->tau = t->far_ratio <= 0.0 ? 3.0e38f : static_cast<float>(t->far_ratio);
    c->chunkCapacityS = 0;  // re-plan the forward chunks
    c->pchunkS = 0;
    c->planEpoch++;
    return LF_OK;
}

extern "C" lf_status lf_get_tuning(lf_ctx* c, lf_tuning* t) {
    if (!c || !t) return LF_EINVAL;
    *t = c->tune;
    return LF_OK;
}

// Max-norm relative difference of two host vectors.
static double rel_diff(const std::vector<double>& a, const std::vector<double>& b) {
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < a.size() && i < b.size(); ++i) {
        num = std::max(num, std::fabs(a[i] - b[i]));
        den = std::max(den, std::fabs(b[i]));
    }
    return den > 0.0 ? num / den : num;
}

// Coordinate search over the launch shapes, each candidate timed with device
// events over `repeats` direct (not replayed) objective+gradient evaluations
// after one untimed evaluation that sizes buffers and uploads its plan.  In
// mixed precision the far-field ratio is searched last, each candidate
// accepted only within its accuracy gate against one FP64 evaluation.
extern "C" lf_status lf_autotune(lf_ctx* c, const double* params, int repeats, lf_tuning* chosen, double* best_ms) {
    LF_RET_IF(check_ready(c));
    if (repeats <= 0) repeats = 3;
    LF_RET_IF(params_to_device(c, params));
    const bool graph = c->graphMode;
    c->graphMode = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        c->graphMode = graph;
        return fail(c, LF_ECUDA, "event creation failed");
    }
    auto timeit = [&](const lf_tuning& t, double* ms) -> lf_status {
        LF_RET_IF(lf_set_tuning(c, &t));
        LF_RET_IF(lf_objective_grad_device(c, c->d_params.p, c->d_f.p, c->d_grad.p));
        LF_TRY_CUDA(c, cudaEventRecord(e0, c->stream));
        for (int r = 0; r < repeats; ++r) LF_RET_IF(lf_objective_grad_device(c, c->d_params.p, c->d_f.p, c->d_grad.p));
        LF_TRY_CUDA(c, cudaEventRecord(e1, c->stream));
        LF_TRY_CUDA(c, cudaEventSynchronize(e1));
        float t_ms = 0.f;
        LF_TRY_CUDA(c, cudaEventElapsedTime(&t_ms, e0, e1));
        *ms = t_ms / repeats;
        return LF_OK;
    };
    // predictions (both data sets, device order) and gradient of one evaluation
    auto evaluate = [&](std::vector<double>& pg, std::vector<double>& pm, std::vector<double>& gr) -> lf_status {
        LF_RET_IF(lf_objective_grad_device(c, c->d_params.p, c->d_f.p, c->d_grad.p));
        pg.resize(c->grav.n);
        pm.resize(c->mag.n);
        gr.resize(c->np);
        if (c->grav.n)
            LF_TRY_CUDA(c, cudaMemcpyAsync(pg.data(), c->grav.d_pred.p, sizeof(double) * c->grav.n,
                                           cudaMemcpyDeviceToHost, c->stream));
        if (c->mag.n)
            LF_TRY_CUDA(c, cudaMemcpyAsync(pm.data(), c->mag.d_pred.p, sizeof(double) * c->mag.n,
                                           cudaMemcpyDeviceToHost, c->stream));
        if (c->np)
            LF_TRY_CUDA(c, cudaMemcpyAsync(gr.data(), c->d_grad.p, sizeof(double) * c->np, cudaMemcpyDeviceToHost,
                                           c->stream));
        LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
        return LF_OK;
    };
    lf_tuning best = c->tune;
    double bestMs = 0.0;
    lf_status st = timeit(best, &bestMs);
    const bool mixed = c->precision == LF_PREC_MIXED;
    const int engineC[] = {LF_FWD_FACET, LF_FWD_PATCH};
    const int fwdC[] = {0, 148 * 4, 148 * 8, 148 * 16, 148 * 32, 148 * 64, 148 * 128};
    const int gradC[] = {148 * 16, 148 * 32, 148 * 64, 148 * 128, 148 * 256};
    const int nearC[] = {0, 1, 2, 4, 8};
    const int threadsC[] = {128, 256};
    // dimensions in turn: forward engine (mixed only), forward CTAs, gradient
    // warps, near tiles (mixed), patch threads (patch engine)
    for (int dim = 0; dim < 5 && st == LF_OK; ++dim) {
        if ((dim == 0 || dim == 3) && !mixed) continue;
        if (dim == 4 && (!mixed || best.fwd_engine != LF_FWD_PATCH)) continue;
        const int* cand = dim == 0 ? engineC : dim == 1 ? fwdC : dim == 2 ? gradC : dim == 3 ? nearC : threadsC;
        const int nc = dim == 0 ? 2 : dim == 1 ? 7 : dim == 4 ? 2 : 5;
        for (int k = 0; k < nc && st == LF_OK; ++k) {
            lf_tuning t = best;
            int& field = dim == 0 ? t.fwd_engine
                                  : dim == 1 ? t.fwd_target_blocks
                                             : dim == 2 ? t.grad_target_warps
                                                        : dim == 3 ? t.near_tiles_per_chunk : t.patch_threads;
            if (field == cand[k]) continue;
            field = cand[k];
            // the persistent schedule (0 forward CTAs) exists for the patch engine only
            if (t.fwd_target_blocks == 0 && !(mixed && t.fwd_engine == LF_FWD_PATCH)) {
                if (dim == 1) continue;
                t.fwd_target_blocks = 148 * 8;
            }
            double ms = 0.0;
            st = timeit(t, &ms);
            if (st == LF_OK && ms < bestMs) {
                bestMs = ms;
                best = t;
            }
        }
    }
    // far-field ratio: accepted only within the accuracy gate against FP64
    if (st == LF_OK && mixed) {
        std::vector<double> rg, rm, rgr, g0, m0, gr0, pg, pm, gr;
        st = lf_set_tuning(c, &best);
        if (st == LF_OK) {
            c->precision = LF_PREC_FP64;
            c->epoch++;
            st = evaluate(rg, rm, rgr);
            c->precision = LF_PREC_MIXED;
            c->epoch++;
        }
        if (st == LF_OK) st = evaluate(g0, m0, gr0);  // the current ratio
        const double gradBase = st == LF_OK ? rel_diff(gr0, rgr) : 0.0;
        const double ratios[] = {2.0, 2.5, 3.0, 4.0};
        for (double tau : ratios) {
            if (st != LF_OK || tau == best.far_ratio) continue;
            lf_tuning t = best;
            t.far_ratio = tau;
            st = lf_set_tuning(c, &t);
            if (st == LF_OK) st = evaluate(pg, pm, gr);
            if (st != LF_OK) break;
            const bool okFwd = rel_diff(pg, rg) <= 0.3e-6 && rel_diff(pm, rm) <= 0.3e-6;
            const bool okGrad = rel_diff(gr, rgr) <= std::max(0.3e-5, 1.5 * gradBase);
            if (!okFwd || !okGrad) continue;
            double ms = 0.0;
            st = timeit(t, &ms);
            if (st == LF_OK && ms < bestMs) {
                bestMs = ms;
                best = t;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->graphMode = graph;
    lf_status st2 = lf_set_tuning(c, &best);
    LF_RET_IF(st);
    LF_RET_IF(st2);
    if (chosen) *chosen = best;
    if (best_ms) *best_ms = bestMs;
    return LF_OK;
}

extern "C" lf_status lf_set_collapsed_facets(lf_ctx* c, int mode) {
    if (!c) return LF_EINVAL;
    if (mode != LF_COLLAPSED_KEEP && mode != LF_COLLAPSED_DROP)
        return fail(c, LF_EINVAL, "collapsed-facet mode must be LF_COLLAPSED_KEEP or LF_COLLAPSED_DROP");
    c->dropCollapsed = mode == LF_COLLAPSED_DROP;
    c->epoch++;
    return LF_OK;
}

extern "C" lf_status lf_set_xy_derivative(lf_ctx* c, int mode, double step) {
    if (!c) return LF_EINVAL;
    if (mode != LF_XY_ANALYTIC && mode != LF_XY_FORWARD_DIFFERENCE)
        return fail(c, LF_EINVAL, "xy derivative mode must be LF_XY_ANALYTIC or LF_XY_FORWARD_DIFFERENCE");
    if (mode == LF_XY_FORWARD_DIFFERENCE && !(step > 0.0 && std::isfinite(step)))
        return fail(c, LF_EINVAL, "finite-difference step must be positive and finite");
    c->xyMode = mode;
    if (mode == LF_XY_FORWARD_DIFFERENCE) c->xyStep = step;
    c->epoch++;
    return LF_OK;
}

extern "C" lf_status lf_set_gradient_gather(lf_ctx* c, int mode) {
    if (!c) return LF_EINVAL;
    if (mode != LF_GATHER_REFERENCE && mode != LF_GATHER_CHAIN)
        return fail(c, LF_EINVAL, "gather mode must be LF_GATHER_REFERENCE or LF_GATHER_CHAIN");
    c->gatherMode = mode;
    if (!c->hasModel) return LF_OK;
    cudaSetDevice(c->device);
    return apply_gather_sets(c);
}

extern "C" lf_status lf_set_scatter_stateless(lf_ctx* c, int enabled) {
    if (!c) return LF_EINVAL;
    c->epoch++;
    c->statelessScatter = enabled != 0;
    return LF_OK;
}

extern "C" lf_status lf_set_graph_mode(lf_ctx* c, int enabled) {
    if (!c) return LF_EINVAL;
    cudaSetDevice(c->device);
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    c->graphMode = enabled != 0;
    drop_graph(c->gObjGrad);
    drop_graph(c->gObj);
    return LF_OK;
}

static lf_status objective_device(lf_ctx* c, const double* d_params) {
    LF_RET_IF(scatter(c, d_params));
    LF_RET_IF(smooth_diff(c));
    LF_RET_IF(forward_all(c));
    LF_RET_IF(residuals(c, false));
    return objective_final(c, d_params, c->d_f.p);
}

extern "C" lf_status lf_objective(lf_ctx* c, const double* params, double* out5) {
    LF_RET_IF(check_ready(c));
    if (!out5) return LF_EINVAL;
    LF_RET_IF(params_to_device(c, params));
    LF_RET_IF(run_cached(c, c->gObj, c->d_params.p, c->d_out5.p, nullptr,
                         [&] { return objective_device(c, c->d_params.p); }));
    LF_TRY_CUDA(c, cudaMemcpyAsync(out5, c->d_out5.p, sizeof(double) * 5, cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    if (!std::isfinite(out5[4])) return fail(c, LF_ENUMERIC, "non-finite objective");
    return LF_OK;
}

extern "C" lf_status lf_objective_grad_device(lf_ctx* c, const double* d_params, double* d_f, double* d_grad) {
    LF_RET_IF(check_ready(c));
    double* f = d_f ? d_f : c->d_f.p;
    double* g = d_grad ? d_grad : c->d_grad.p;
    return run_cached(c, c->gObjGrad, d_params, f, g, [&]() -> lf_status {
        LF_RET_IF(scatter(c, d_params));
        LF_RET_IF(smooth_diff(c));
        LF_RET_IF(forward_all(c));
        LF_RET_IF(residuals(c, true));
        LF_RET_IF(objective_final(c, d_params, f));
        return gradient_all(c, d_params, g);
    });
}

extern "C" lf_status lf_objective_grad(lf_ctx* c, const double* params, double* f, double* grad) {
    LF_RET_IF(check_ready(c));
    LF_RET_IF(params_to_device(c, params));
    LF_RET_IF(lf_objective_grad_device(c, c->d_params.p, c->d_f.p, c->d_grad.p));
    if (f) LF_TRY_CUDA(c, cudaMemcpyAsync(f, c->d_f.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (grad && c->np)
        LF_TRY_CUDA(c, cudaMemcpyAsync(grad, c->d_grad.p, sizeof(double) * c->np, cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    if (f && !std::isfinite(*f)) return fail(c, LF_ENUMERIC, "non-finite objective");
    return LF_OK;
}

// ---------------------------------------------------- data-weight calibration --
// Matrix-free J v and J^T w for one data set, with the Jacobian semantics of
// the reference's computeJacobian (the derivative of a DOF is its own
// vertices' positional derivative times the axis scale, gravity_forward.cpp:
// 269-289).  FP64 throughout, whatever the context's precision.
__global__ void k_pos_shift(int n, const double* __restrict__ base, const double* __restrict__ vel, double eps,
                            double* __restrict__ pos) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pos[i] = base[i] + eps * vel[i];
}

// FP64 forward of one set at the current positions into s.d_pred.
static lf_status forward_one_fp64(lf_ctx* c, StationSet& s, bool grav) {
    k_face_prep_fwd<<<cdiv(c->T, 128), 128, 0, c->stream>>>(c->T, c->d_tri.p, c->d_pos.p, c->d_faceGroup.p,
                                                            c->d_groups.p, c->fdir, c->d_fc.p,
                                                            c->dropCollapsed);
    c->counters.launches++;
    return grav ? forward_set<true, false>(c, s, s.d_pred.p, nullptr) : forward_set<false, true>(c, s, nullptr, s.d_pred.p);
}

// out[n_stations] (device order) = J v, by a central difference along the
// vertex velocity u = v scattered through the DOF refs, displacement
// max |eps u| = 1e-3 m (truncation ~1e-10 relative, rounding ~1e-12).
static lf_status jv_product(lf_ctx* c, StationSet& s, bool grav, const std::vector<double>& v, std::vector<double>& out) {
    const int n3 = 3 * c->V;
    double vmax = 0.0;
    for (double x : v) vmax = std::max(vmax, std::fabs(x));
    out.assign(s.n, 0.0);
    if (vmax == 0.0 || c->maxRefScale == 0.0) return LF_OK;
    const double eps = 1e-3 / (vmax * c->maxRefScale);
    LF_TRY_CUDA(c, c->d_vel.reserve(n3));
    LF_TRY_CUDA(c, c->d_posSave.reserve(n3));
    LF_TRY_CUDA(c, c->d_tmpS.reserve(std::max(s.n, 1)));
    LF_TRY_CUDA(c, upload(c->d_tmpP, v.data(), v.size(), c->stream));
    LF_TRY_CUDA(c, cudaMemsetAsync(c->d_vel.p, 0, sizeof(double) * n3, c->stream));
    k_scatter_dofs<<<cdiv(c->np, 256), 256, 0, c->stream>>>(c->np, c->d_tmpP.p, c->d_dofOff.p, c->d_refVertex.p,
                                                              c->d_refAxis.p, c->d_refScale.p, c->d_vel.p);
    LF_TRY_CUDA(c, cudaMemcpyAsync(c->d_posSave.p, c->d_pos.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->stream));
    std::vector<double> plus(s.n), minus(s.n);
    lf_status st = LF_OK;
    for (int sign = 1; sign >= -1 && st == LF_OK; sign -= 2) {
        k_pos_shift<<<cdiv(n3, 256), 256, 0, c->stream>>>(n3, c->d_posSave.p, c->d_vel.p, sign * eps, c->d_pos.p);
        st = forward_one_fp64(c, s, grav);
        if (st == LF_OK && cudaMemcpyAsync(sign > 0 ? plus.data() : minus.data(), s.d_pred.p, sizeof(double) * s.n,
                                           cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
            st = fail(c, LF_ECUDA, "copy failed");
    }
    // restore the positions whatever happened
    if (cudaMemcpyAsync(c->d_pos.p, c->d_posSave.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->stream) !=
            cudaSuccess && st == LF_OK)
        st = fail(c, LF_ECUDA, "position restore failed");
    LF_RET_IF(st);
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int i = 0; i < s.n; ++i) out[i] = (plus[i] - minus[i]) / (2.0 * eps);
    return LF_OK;
}

// out[np] = J^T w, w[n_stations] in device order: the gradient kernels with
// w as the station coefficients, no regularisation terms.
static lf_status jtw_product(lf_ctx* c, StationSet& s, bool grav, const std::vector<double>& w, std::vector<double>& out) {
    LF_TRY_CUDA(c, upload(c->d_tmpS, w.data(), w.size(), c->stream));
    k_face_prep_grad<<<cdiv(c->T, 128), 128, 0, c->stream>>>(c->T, c->d_tri.p, c->d_pos.p, c->d_faceGroup.p,
                                                             c->d_groups.p, c->d_faceNeeds.p, 1, 1, c->fdir,
                                                             c->d_gc.p);
    LF_TRY_CUDA(c, c->d_partGrad.reserve((size_t)std::max(grad_slots(c, s.n), 1) * 9 * c->T));
    const int used = gradient_set(c, s, grav ? c->d_tmpS.p : nullptr, grav ? nullptr : c->d_tmpS.p, 0);
    if (used > 0 && c->nGradVerts > 0)
        k_vertex_reduce<<<cdiv(c->nGradVerts, 4), 128, 0, c->stream>>>(c->nGradVerts, c->d_gradVerts.p, c->d_vfOff.p,
                                                                        c->d_vf.p, c->T, used, used, c->d_partGrad.p,
                                                                        c->d_vgrad.p);
    else
        LF_TRY_CUDA(c, cudaMemsetAsync(c->d_vgrad.p, 0, sizeof(double) * 3 * c->V, c->stream));
    LF_TRY_CUDA(c, c->d_tmpP.reserve(std::max(c->np, 1)));
    if (c->np > 0)
        k_dof_gather<<<cdiv(c->np, 256), 256, 0, c->stream>>>(c->np, c->d_dofOff.p, c->d_refVertex.p, c->d_refAxis.p,
                                                              c->d_refScale.p, c->d_vgrad.p, nullptr, nullptr, 0.0,
                                                              nullptr, 0.0, c->d_tmpP.p);
    LF_CHECK_LAUNCH(c);
    out.assign(c->np, 0.0);
    if (c->np > 0)
        LF_TRY_CUDA(c, cudaMemcpyAsync(out.data(), c->d_tmpP.p, sizeof(double) * c->np, cudaMemcpyDeviceToHost,
                                       c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

// JointObjective::calibrateDataWeights (joint_objective.cpp:281-393),
// matrix-free: power iteration (at most 50 iterations, relative tolerance
// 1e-8) for the largest eigenvalue of J^T W^2 J of each data type, W^2 =
// 1/sigma^2; alpha_mag *= clip(lambda_grav / lambda_mag, 1e-6, 1e6); when the
// ratio is not finite and positive, the gradient-norm ratio
// |J_g^T W^2 r_g| / |J_m^T W^2 r_m| instead.  The start vector is seeded
// uniform [-1, 1) (the reference draws it from Eigen's Random).
extern "C" lf_status lf_calibrate_data_weights(lf_ctx* c, const double* params, unsigned seed, double* alpha_out,
                                               double* eig_grav, double* eig_mag) {
    LF_RET_IF(check_ready(c));
    if (eig_grav) *eig_grav = 0.0;
    if (eig_mag) *eig_mag = 0.0;
    if (c->mag.n == 0 || c->grav.n == 0 || c->alphaMag <= 0.0) {
        if (alpha_out) *alpha_out = c->alphaMag;
        return LF_OK;  // joint_objective.cpp:282
    }
    if (c->partitioned) return fail(c, LF_ESTATE, "calibration is not available for batched bodies");
    LF_RET_IF(params_to_device(c, params));
    LF_RET_IF(scatter(c, c->d_params.p));
    const int prec = c->precision;
    c->precision = LF_PREC_FP64;
    auto w2_of = [&](StationSet& s, std::vector<double>& w2) -> lf_status {
        std::vector<double> w(s.n);
        LF_TRY_CUDA(c, cudaMemcpy(w.data(), s.d_w.p, sizeof(double) * s.n, cudaMemcpyDeviceToHost));
        w2.resize(s.n);
        for (int i = 0; i < s.n; ++i) w2[i] = w[i] * w[i];
        return LF_OK;
    };
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> uni(-1.0, 1.0);
    auto power = [&](StationSet& s, bool grav, double* eig) -> lf_status {
        std::vector<double> w2, v(c->np), jv, jtw;
        LF_RET_IF(w2_of(s, w2));
        for (double& x : v) x = uni(rng);
        double nv = 0.0;
        for (double x : v) nv += x * x;
        nv = std::sqrt(nv);
        for (double& x : v) x /= nv;
        double lambdaOld = 0.0;
        *eig = 0.0;
        for (int it = 0; it < 50; ++it) {
            LF_RET_IF(jv_product(c, s, grav, v, jv));
            for (int i = 0; i < s.n; ++i) jv[i] *= w2[i];
            LF_RET_IF(jtw_product(c, s, grav, jv, jtw));
            double lam = 0.0;
            for (double x : jtw) lam += x * x;
            lam = std::sqrt(lam);
            if (lam < 1e-60) return LF_OK;
            for (int d = 0; d < c->np; ++d) v[d] = jtw[d] / lam;
            if (std::fabs(lam - lambdaOld) / lam < 1e-8) break;
            lambdaOld = lam;
        }
        LF_RET_IF(jv_product(c, s, grav, v, jv));
        for (int i = 0; i < s.n; ++i) jv[i] *= w2[i];
        LF_RET_IF(jtw_product(c, s, grav, jv, jtw));
        double vh = 0.0;
        for (int d = 0; d < c->np; ++d) vh += v[d] * jtw[d];
        *eig = std::max(vh, 0.0);
        return LF_OK;
    };
    double eg = 0.0, em = 0.0;
    lf_status st = power(c->grav, true, &eg);
    if (st == LF_OK) st = power(c->mag, false, &em);
    double ratio = em > 1e-60 ? eg / em : 0.0;
    if (st == LF_OK) {
        c->epoch++;
        if (std::isfinite(ratio) && ratio > 0.0) {
            c->alphaMag *= std::max(1e-6, std::min(ratio, 1e6));
        } else {
            // gradient-norm fallback (joint_objective.cpp:357-392)
            double norms[2] = {0.0, 0.0};
            for (int k = 0; k < 2 && st == LF_OK; ++k) {
                StationSet& s = k == 0 ? c->grav : c->mag;
                std::vector<double> w2, pred(s.n), obs(s.n), coef(s.n), jtw;
                st = w2_of(s, w2);
                if (st == LF_OK) st = forward_one_fp64(c, s, k == 0);
                if (st == LF_OK && (cudaMemcpy(pred.data(), s.d_pred.p, sizeof(double) * s.n, cudaMemcpyDeviceToHost) !=
                                        cudaSuccess ||
                                    cudaMemcpy(obs.data(), s.d_obs.p, sizeof(double) * s.n, cudaMemcpyDeviceToHost) !=
                                        cudaSuccess))
                    st = fail(c, LF_ECUDA, "copy failed");
                if (st != LF_OK) break;
                for (int i = 0; i < s.n; ++i) coef[i] = w2[i] * (obs[i] - pred[i]);
                st = jtw_product(c, s, k == 0, coef, jtw);
                for (double x : jtw) norms[k] += x * x;
                norms[k] = std::sqrt(norms[k]);
            }
            if (st == LF_OK && norms[0] >= 1e-60 && norms[1] > 1e-60) c->alphaMag *= norms[0] / norms[1];
        }
    }
    c->precision = prec;
    LF_RET_IF(st);
    if (alpha_out) *alpha_out = c->alphaMag;
    if (eig_grav) *eig_grav = eg;
    if (eig_mag) *eig_mag = em;
    return LF_OK;
}

// Forward of one group alone with unit properties (GravityForward::
// computeGroupUnitResponse gravity_forward.cpp:132-146; MagneticForward::
// computeGroupUnitResponse / computeGroupUnitResponseDirection /
// computeGroupUnitRemanenceResponse magnetic_forward.cpp:148-190): the group
// table is swapped for one where every other group has zero scales, the
// chunk plan covers only the group's facets, and both are restored after.
extern "C" lf_status lf_unit_response(lf_ctx* c, const double* params, int kind, int group, const double* dir,
                                      double* out) {
    LF_RET_IF(check_ready(c));
    if (!out || kind < LF_UNIT_GRAVITY || kind > LF_UNIT_REMANENCE || group < 0 || group >= c->G ||
        (kind == LF_UNIT_DIRECTION && (!dir || !finite_all(dir, 3))))
        return fail(c, LF_EINVAL, "lf_unit_response: bad kind, group or direction");
    StationSet& s = kind == LF_UNIT_GRAVITY ? c->grav : c->mag;
    if (s.n == 0) return fail(c, LF_ESTATE, "no stations of the requested type");
    if (c->partitioned) return fail(c, LF_ESTATE, "unit responses are not available for batched bodies");
    LF_RET_IF(params_to_device(c, params));
    LF_RET_IF(scatter(c, c->d_params.p));
    std::vector<GroupConst> unit(c->gconst);
    for (GroupConst& k : unit) {
        k.gscale_fwd = k.gscale_jac = 0.0;
        k.mscale = 0.0;
        k.mag_active = 0;
    }
    GroupConst& k = unit[group];
    double m[3] = {c->fdir.x, c->fdir.y, c->fdir.z}, amp = 1.0;
    switch (kind) {
    case LF_UNIT_GRAVITY:
        k.gscale_fwd = kGSI * 1.0 * kDensityScale * kMs2ToMgal;
        k.gscale_jac = (kGSI * kDensityScale * kMs2ToMgal) * 1.0;
        break;
    case LF_UNIT_INDUCED:  // magneticClosedMesh(obs, mesh, 1.0, F_hat, F): amp = F / 100 along F_hat
        amp = 1.0 * c->fieldNT / 100.0;
        break;
    case LF_UNIT_DIRECTION:  // magneticClosedMeshVector(obs, mesh, 1.0, dir, F_hat)
        for (int i = 0; i < 3; ++i) m[i] = dir[i];
        break;
    case LF_UNIT_REMANENCE: {  // unit magnetisation along the group's remanence direction
        const GroupProps& gp = c->groups[group];
        double I = gp.remInc * kPi / 180.0, D = gp.remDec * kPi / 180.0, cI = std::cos(I);
        m[0] = cI * std::cos(D); m[1] = cI * std::sin(D); m[2] = -std::sin(I);
        break;
    }
    }
    if (kind != LF_UNIT_GRAVITY) {
        for (int i = 0; i < 3; ++i) k.mdir[i] = m[i];
        k.mscale = amp * 100.0 / (4.0 * kPi);
        k.mag_active = 1;
    }
    lf_status st = LF_OK;
    if (cudaMemcpyAsync(c->d_groups.p, unit.data(), sizeof(GroupConst) * unit.size(), cudaMemcpyHostToDevice,
                        c->stream) != cudaSuccess)
        st = fail(c, LF_ECUDA, "group table upload failed");
    double* d_g = kind == LF_UNIT_GRAVITY ? s.d_pred.p : nullptr;
    double* d_t = kind == LF_UNIT_GRAVITY ? nullptr : s.d_pred.p;
    if (st == LF_OK) {
        c->groupFilter = group;
        if (c->precision == LF_PREC_MIXED) {
            st = mixed_prep(c);
            if (st == LF_OK)
                st = kind == LF_UNIT_GRAVITY ? forward_set_mixed<true, false>(c, s, d_g, d_t)
                                         : forward_set_mixed<false, true>(c, s, d_g, d_t);
        } else {
            k_face_prep_fwd<<<cdiv(c->T, 128), 128, 0, c->stream>>>(c->T, c->d_tri.p, c->d_pos.p, c->d_faceGroup.p,
                                                                    c->d_groups.p, c->fdir, c->d_fc.p,
                                                            c->dropCollapsed);
            c->counters.launches++;
            st = kind == LF_UNIT_GRAVITY ? forward_set<true, false>(c, s, d_g, d_t)
                                         : forward_set<false, true>(c, s, d_g, d_t);
        }
        c->groupFilter = -1;
    }
    // restore the model's group table whatever happened above
    if (cudaMemcpyAsync(c->d_groups.p, c->gconst.data(), sizeof(GroupConst) * c->gconst.size(),
                        cudaMemcpyHostToDevice, c->stream) != cudaSuccess && st == LF_OK)
        st = fail(c, LF_ECUDA, "group table restore failed");
    LF_RET_IF(st);
    LF_RET_IF(unpermute_device(c, s, s.d_pred.p, s.d_out.p));
    LF_TRY_CUDA(c, cudaMemcpyAsync(out, s.d_out.p, sizeof(double) * s.n, cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

// One bounded least-squares property problem of runPropertyInversion
// (runner.cpp:737-786 / 866-913): U column-major [n x m], the reference's
// summation orders (U d by columns, U^T r by rows, squared norms in index
// order).
static std::vector<double> property_solve(const std::vector<double>& U, int n, int m, const std::vector<double>& obs,
                                          const std::vector<double>& w, const std::vector<double>& x0,
                                          const std::vector<double>& lo, const std::vector<double>& hi,
                                          const lf_property_options& o) {
    double var = 0.0;
    for (int i = 0; i < n; ++i) var += obs[i] * obs[i];
    var /= static_cast<double>(n);
    const double rms = std::sqrt(std::max(var, 1.0));
    const double lambda = o.damping;
    auto predict = [&](const std::vector<double>& d) {
        std::vector<double> y(n, 0.0);
        for (int j = 0; j < m; ++j)
            for (int i = 0; i < n; ++i) y[i] += U[(size_t)j * n + i] * d[j];
        return y;
    };
    Objective f = [&](const std::vector<double>& d) {
        const std::vector<double> pred = predict(d);
        double misfit = 0.0;
        for (int i = 0; i < n; ++i) {
            const double res = w[i] * (obs[i] - pred[i]);
            misfit += 0.5 * res * res;
        }
        misfit /= rms * rms;
        if (lambda > 0.0) {
            double sq = 0.0;
            for (int j = 0; j < m; ++j) sq += (d[j] - x0[j]) * (d[j] - x0[j]);
            misfit += 0.5 * lambda * sq;
        }
        return misfit;
    };
    Gradient g = [&](const std::vector<double>& d) {
        const std::vector<double> pred = predict(d);
        const double inv2 = 1.0 / (rms * rms);
        std::vector<double> wr(n), grad(m);
        for (int i = 0; i < n; ++i) wr[i] = inv2 * w[i] * w[i] * (obs[i] - pred[i]);
        for (int j = 0; j < m; ++j) {
            double acc = 0.0;
            for (int i = 0; i < n; ++i) acc += (-1.0 * U[(size_t)j * n + i]) * wr[i];
            grad[j] = acc;
        }
        if (lambda > 0.0)
            for (int j = 0; j < m; ++j) grad[j] = grad[j] + lambda * (d[j] - x0[j]);
        return grad;
    };
    LbfgsbOptions lo_opt;
    lo_opt.maxIterations = o.max_iterations;
    lo_opt.historySize = std::min(5, m);
    lo_opt.tolerance = o.tolerance;
    LbfgsbOptimizer opt(lo_opt);
    return opt.minimize(f, g, x0, lo, hi).params;
}

extern "C" lf_status lf_property_inversion(lf_ctx* c, const double* params, const lf_property_options* o,
                                           double* density, double* magnetic) {
    LF_RET_IF(check_ready(c));
    if (!o || o->max_iterations < 0 || !std::isfinite(o->damping) || !std::isfinite(o->tolerance))
        return fail(c, LF_EINVAL, "lf_property_inversion: bad options");
    if (c->partitioned) return fail(c, LF_ESTATE, "property inversion is not available for batched bodies");
    const int G = c->G;
    // Part A: densities from the gravity data (runner.cpp:716-798)
    if (c->grav.n > 0) {
        const int n = c->grav.n;
        std::vector<double> U((size_t)n * G), x0(G), lo(G, o->density_min), hi(G, o->density_max);
        for (int g = 0; g < G; ++g) {
            LF_RET_IF(lf_unit_response(c, params, LF_UNIT_GRAVITY, g, nullptr, U.data() + (size_t)g * n));
            x0[g] = c->groups[g].density;
        }
        const std::vector<double> d = property_solve(U, n, G, c->grav.obs, c->grav.w, x0, lo, hi, *o);
        for (int g = 0; g < G; ++g) c->groups[g].density = d[g];
    }
    // Part B: susceptibility (+ remanence) from the magnetic data (runner.cpp:803-917)
    const int ppg = c->remMode == LF_REM_FIXED_VECTOR ? 2 : (c->remMode == LF_REM_VECTOR ? 4 : 1);
    if (c->mag.n > 0) {
        const int n = c->mag.n, m = ppg * G;
        std::vector<double> U((size_t)n * m), x0(m), lo(m), hi(m);
        const double ex[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
        for (int g = 0; g < G; ++g) {
            const int col = ppg * g;
            LF_RET_IF(lf_unit_response(c, params, LF_UNIT_INDUCED, g, nullptr, U.data() + (size_t)col * n));
            x0[col] = c->groups[g].chi;
            lo[col] = o->susceptibility_min;
            hi[col] = o->susceptibility_max;
            if (ppg == 2) {
                LF_RET_IF(lf_unit_response(c, params, LF_UNIT_REMANENCE, g, nullptr, U.data() + (size_t)(col + 1) * n));
                x0[col + 1] = c->groups[g].remMag;
                lo[col + 1] = o->remanence_min;
                hi[col + 1] = o->remanence_max;
            } else if (ppg == 4) {
                for (int k = 0; k < 3; ++k) {
                    LF_RET_IF(lf_unit_response(c, params, LF_UNIT_DIRECTION, g, ex[k],
                                               U.data() + (size_t)(col + 1 + k) * n));
                    x0[col + 1 + k] = c->groups[g].remVec[k];
                    lo[col + 1 + k] = o->remanence_component_min;
                    hi[col + 1 + k] = o->remanence_component_max;
                }
            }
        }
        const std::vector<double> d = property_solve(U, n, m, c->mag.obs, c->mag.w, x0, lo, hi, *o);
        for (int g = 0; g < G; ++g) {
            const int col = ppg * g;
            c->groups[g].chi = d[col];
            if (ppg == 2) c->groups[g].remMag = d[col + 1];
            if (ppg == 4)
                for (int k = 0; k < 3; ++k) c->groups[g].remVec[k] = d[col + 1 + k];
        }
        if (magnetic)
            for (int j = 0; j < m; ++j) magnetic[j] = d[j];
    }
    if (density)
        for (int g = 0; g < G; ++g) density[g] = c->groups[g].density;
    c->epoch++;
    LF_RET_IF(upload_groups(c));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

extern "C" lf_status lf_jacobian(lf_ctx* c, const double* params, int which, double* J) {
    LF_RET_IF(check_ready(c));
    if (!J || (which != LF_GRAVITY && which != LF_MAGNETIC)) return LF_EINVAL;
    StationSet& s = which == LF_GRAVITY ? c->grav : c->mag;
    if (s.n == 0) return fail(c, LF_ESTATE, "no stations of the requested type");
    if (c->partitioned) return fail(c, LF_ESTATE, "dense Jacobian rows are not available for batched bodies");
    LF_RET_IF(params_to_device(c, params));
    LF_RET_IF(scatter(c, c->d_params.p));
    k_face_prep_grad<<<cdiv(c->T, 128), 128, 0, c->stream>>>(c->T, c->d_tri.p, c->d_pos.p, c->d_faceGroup.p,
                                                             c->d_groups.p, c->d_faceNeeds.p, which == LF_GRAVITY,
                                                             which == LF_MAGNETIC, c->fdir, c->d_gc.p);
    LF_CHECK_LAUNCH(c);
    std::vector<double> ones(s.n, 1.0);
    LF_TRY_CUDA(c, upload(c->d_ones, ones.data(), ones.size(), c->stream));
    int np = std::max(c->np, 1);
    // stations per batch so that the partial buffer stays below ~256 MB
    size_t per = (size_t)9 * c->T * sizeof(double);
    int batch = static_cast<int>(std::max<size_t>(1, std::min<size_t>({(size_t)s.n, ((size_t)256 << 20) / per, (size_t)65535})));
    LF_TRY_CUDA(c, c->d_partGrad.reserve((size_t)batch * 9 * c->T));
    LF_TRY_CUDA(c, c->d_jac.reserve((size_t)batch * np));
    std::vector<double> rows;
    for (int s0 = 0; s0 < s.n; s0 += batch) {
        int nb = std::min(batch, s.n - s0);
        dim3 grid(cdiv(c->T, kGradThreads), nb);
        const double* g1 = which == LF_GRAVITY ? c->d_ones.p : nullptr;
        const double* m1 = which == LF_MAGNETIC ? c->d_ones.p : nullptr;
        k_gradient_fp64<<<grid, kGradThreads, 0, c->stream>>>(
            c->T, c->d_gc.p, nb, s.d_xyz.p + 3 * (size_t)s0, g1, m1, 1, c->d_faceGroup.p, c->d_groups.p, c->fdir,
            c->d_partGrad.p);
        if (c->np > 0) {
            dim3 g2(cdiv(c->np, 128), nb);
            k_jacobian_gather<<<g2, 128, 0, c->stream>>>(nb, c->np, c->d_dofOff.p, c->d_refVertex.p, c->d_refAxis.p,
                                                         c->d_refScale.p, c->d_vfOff.p, c->d_vf.p, c->T,
                                                         c->d_partGrad.p, c->d_jac.p, c->np);
            rows.resize((size_t)nb * c->np);
            LF_TRY_CUDA(c, cudaMemcpyAsync(rows.data(), c->d_jac.p, sizeof(double) * (size_t)nb * c->np,
                                           cudaMemcpyDeviceToHost, c->stream));
            LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
            for (int r = 0; r < nb; ++r)
                std::copy(rows.begin() + (size_t)r * c->np, rows.begin() + (size_t)(r + 1) * c->np,
                          J + (size_t)s.perm[s0 + r] * c->np);
        }
        LF_CHECK_LAUNCH(c);
    }
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

extern "C" lf_status lf_get_positions(lf_ctx* c, double* xyz) {
    if (!c || !xyz) return LF_EINVAL;
    if (!c->hasModel) return fail(c, LF_ESTATE, "no model set");
    cudaSetDevice(c->device);
    LF_TRY_CUDA(c, cudaMemcpyAsync(xyz, c->d_pos.p, sizeof(double) * 3 * c->V, cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

extern "C" void lf_lbfgsb_default_options(lf_lbfgsb_options* o) {
    if (!o) return;
    o->max_iterations = 500;
    o->tolerance = 1e-6;
    o->history_size = 10;
    o->armijo_c1 = 1e-4;
    o->line_search_max_iter = 50;
    o->disable_line_search = 0;
    o->initial_gamma = 0.0;
    o->target_value = 0.0;
}

extern "C" lf_status lf_lbfgsb_minimize(lf_ctx* c, const double* x0, const double* lo, const double* hi,
                                        const lf_lbfgsb_options* opt, double* xOut, lf_lbfgsb_result* res) {
    LF_RET_IF(check_ready(c));
    if (!x0 || !lo || !hi || !xOut) return LF_EINVAL;
    lf_lbfgsb_options o;
    lf_lbfgsb_default_options(&o);
    if (opt) o = *opt;
    LbfgsbOptions lo2;
    lo2.maxIterations = o.max_iterations;
    lo2.tolerance = o.tolerance;
    lo2.historySize = std::max(1, o.history_size);
    lo2.armijoC1 = o.armijo_c1;
    lo2.lineSearchMaxIter = o.line_search_max_iter;
    lo2.disableLineSearch = o.disable_line_search != 0;
    lo2.initialGamma = o.initial_gamma;
    lo2.targetValue = o.target_value;
    int n = c->np;
    lf_status status = LF_OK;
    int nEval = 0, nGrad = 0;
    // Objective values of the last gradient evaluation are reused when the
    // optimizer asks for f at the same point (results are deterministic).
    std::vector<double> lastX;
    double lastF = 0.0;
    Objective f = [&](const std::vector<double>& x) -> double {
        if (status != LF_OK) return std::numeric_limits<double>::quiet_NaN();
        if (x == lastX) return lastF;
        double out5[5];
        status = lf_objective(c, x.data(), out5);
        ++nEval;
        return out5[4];
    };
    Gradient g = [&](const std::vector<double>& x) -> std::vector<double> {
        std::vector<double> gr(n, 0.0);
        if (status != LF_OK) return gr;
        double fv = 0.0;
        status = lf_objective_grad(c, x.data(), &fv, gr.data());
        ++nGrad;
        lastX = x;
        lastF = fv;
        return gr;
    };
    LbfgsbOptimizer optz(lo2);
    LbfgsbResult r = optz.minimize(f, g, std::vector<double>(x0, x0 + n), std::vector<double>(lo, lo + n),
                                   std::vector<double>(hi, hi + n));
    if (status != LF_OK) return status;
    std::copy(r.params.begin(), r.params.end(), xOut);
    if (res) {
        res->iterations = r.iterations;
        res->converged = r.converged ? 1 : 0;
        res->evaluations = nEval;
        res->gradients = nGrad;
        res->final_value = r.finalValue;
        std::snprintf(res->message, sizeof(res->message), "%s", r.message.c_str());
    }
    return LF_OK;
}

extern "C" lf_status lf_get_counters(lf_ctx* c, lf_counters* out) {
    if (!c || !out) return LF_EINVAL;
    *out = c->counters;
    return LF_OK;
}
extern "C" lf_status lf_set_profiling(lf_ctx* c, int enabled) {
    if (!c) return LF_EINVAL;
    c->epoch++;
    cudaSetDevice(c->device);
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    c->profiling = enabled != 0;
    c->nFwd = c->nGrad = 0;
    return LF_OK;
}

extern "C" lf_status lf_get_kernel_times(lf_ctx* c, double* fwdMs, int* fwdN, double* gradMs, int* gradN) {
    if (!c) return LF_EINVAL;
    cudaSetDevice(c->device);
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    auto sum = [&](std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v, size_t n, double* out) -> lf_status {
        double t = 0.0;
        for (size_t i = 0; i < n; ++i) {
            float ms = 0.f;
            LF_TRY_CUDA(c, cudaEventElapsedTime(&ms, v[i].first, v[i].second));
            t += ms;
        }
        if (out) *out = t;
        return LF_OK;
    };
    lf_status st = sum(c->evFwd, c->nFwd, fwdMs);
    if (st != LF_OK) return st;
    st = sum(c->evGrad, c->nGrad, gradMs);
    if (st != LF_OK) return st;
    if (fwdN) *fwdN = static_cast<int>(c->nFwd);
    if (gradN) *gradN = static_cast<int>(c->nGrad);
    return LF_OK;
}

extern "C" lf_status lf_reset_counters(lf_ctx* c) {
    if (!c) return LF_EINVAL;
    c->counters = {0, 0, 0};
    if (c->d_nearPairs.p) {
        cudaSetDevice(c->device);
        LF_TRY_CUDA(c, cudaMemsetAsync(c->d_nearPairs.p, 0, sizeof(unsigned long long), c->stream));
    }
    return LF_OK;
}

// ------------------------------------------- classification and constraints --
// LithologyModel::setLabelGrid / setBottomDepth / classifyPoint
// (lithology_model.cpp:89-103, 856-858, 288-363) and ConstraintHandler
// (constraint_handler.cpp:7-66) over the context's device positions.

static lf_status model_ready(lf_ctx* c) {
    if (!c) return LF_EINVAL;
    if (!c->hasModel) return fail(c, LF_ESTATE, "no model set");
    cudaSetDevice(c->device);
    return LF_OK;
}

// Classifies n device points (xyz rows) into d_out against the current
// device positions (the group triangle ranges must be on the device).
// With at most 64 groups the crossings of one point are split over several
// CTAs (parities combine by XOR); d_clsMask must hold n masks.
static lf_status classify_launch(lf_ctx* c, int n, const double* d_pts, int32_t* d_out) {
    if (n <= 0) return LF_OK;
    if (c->G > 64 || c->d_clsMask.n < (size_t)n) {
        k_classify_points<<<n, kClassifyThreads, 0, c->stream>>>(n, d_pts, c->G, c->d_grpTriOffDev.p, c->d_tri.p,
                                                                 c->d_pos.p, c->bottomDepth, c->labelGrid, d_out);
        c->counters.launches++;
        LF_CHECK_LAUNCH(c);
        return LF_OK;
    }
    const int slices = std::max(1, std::min(cdiv(c->T, 2 * kCrossThreads), cdiv(148 * 8, n)));
    const int slice = cdiv(c->T, slices);
    k_classify_prep<<<cdiv(n, 128), 128, 0, c->stream>>>(n, d_pts, c->G, c->bottomDepth, c->labelGrid, d_out,
                                                         c->d_clsMask.p);
    k_classify_cross<<<dim3(n, slices), kCrossThreads, 0, c->stream>>>(n, d_pts, c->T, slice, c->d_faceGroup.p,
                                                                        c->d_tri.p, c->d_pos.p, d_out,
                                                                        c->d_clsMask.p);
    k_classify_finish<<<cdiv(n, 128), 128, 0, c->stream>>>(n, c->d_clsMask.p, d_out);
    c->counters.launches += 3;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

static lf_status classify_dev(lf_ctx* c, int n, const double* d_pts, int32_t* d_out) {
    if (n <= 0) return LF_OK;
    LF_TRY_CUDA(c, upload(c->d_grpTriOffDev, c->grpTriOff.data(), c->grpTriOff.size(), c->stream));
    return classify_launch(c, n, d_pts, d_out);
}

// Scatter of the context's constraint parameter buffer, classification of
// the interval midpoints and the penalty into *d_out (device).
static lf_status constraint_eval_dev(lf_ctx* c, double* d_out) {
    LF_RET_IF(scatter(c, c->d_cPar.p));
    LF_RET_IF(classify_launch(c, c->nCons, c->d_cMid.p, c->d_cCls.p));
    k_constraint_penalty<<<1, kPenaltyThreads, 0, c->stream>>>(c->nCons, c->d_cCls.p, c->d_cGroup.p, c->d_cThick.p,
                                                               c->consWeight, d_out);
    c->counters.launches++;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

static lf_status constraint_params(lf_ctx* c, const double* params) {
    if (c->np > 0 && !params) return fail(c, LF_EINVAL, "null params");
    if (!finite_all(params, c->np)) return fail(c, LF_EINVAL, "non-finite parameter");
    LF_TRY_CUDA(c, upload(c->d_cPar, params, c->np, c->stream));
    return LF_OK;
}

extern "C" lf_status lf_set_label_grid(lf_ctx* c, int nx, int ny, int nz, double x0, double y0, double z0, double dx,
                                       double dy, double dz, const int32_t* labels) {
    LF_RET_IF(model_ready(c));
    c->epoch++;  // cached constraint sweeps bake the grid in
    if (nx <= 0 || ny <= 0 || nz <= 0 || !labels) {  // no grid: ray casting only
        c->labelGrid = LabelGridDev{};
        return LF_OK;
    }
    const double g[6] = {x0, y0, z0, dx, dy, dz};
    if (!finite_all(g, 6) || dx == 0.0 || dy == 0.0 || dz == 0.0 ||
        (long long)nx * ny * nz > (long long)1 << 31)
        return fail(c, LF_EINVAL, "lf_set_label_grid: bad origin, spacing or size");
    const size_t n = (size_t)nx * ny * nz;
    LF_TRY_CUDA(c, upload(c->d_labels, labels, n, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    c->labelGrid = LabelGridDev{nx, ny, nz, x0, y0, z0, dx, dy, dz, c->d_labels.p};
    return LF_OK;
}

extern "C" lf_status lf_set_bottom_depth(lf_ctx* c, double depth) {
    if (!c || std::isnan(depth)) return LF_EINVAL;
    c->epoch++;
    c->bottomDepth = depth;
    return LF_OK;
}

extern "C" lf_status lf_classify_points(lf_ctx* c, const double* params, int n, const double* xyz, int32_t* group) {
    LF_RET_IF(model_ready(c));
    if (n < 0 || (n > 0 && (!xyz || !group))) return fail(c, LF_EINVAL, "lf_classify_points: bad point arrays");
    if (params) {
        LF_RET_IF(constraint_params(c, params));
        LF_RET_IF(scatter(c, c->d_cPar.p));
    }
    if (n == 0) return LF_OK;
    if (!finite_all(xyz, 3 * (size_t)n)) return fail(c, LF_EINVAL, "lf_classify_points: non-finite point");
    LF_TRY_CUDA(c, upload(c->d_pts, xyz, 3 * (size_t)n, c->stream));
    LF_TRY_CUDA(c, c->d_ptCls.reserve(n));
    LF_TRY_CUDA(c, c->d_clsMask.reserve(std::max<size_t>(c->d_clsMask.n, n)));
    LF_RET_IF(classify_dev(c, n, c->d_pts.p, c->d_ptCls.p));
    LF_TRY_CUDA(c, cudaMemcpyAsync(group, c->d_ptCls.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

extern "C" lf_status lf_set_constraints(lf_ctx* c, int n, const double* xy, const double* z_top,
                                        const double* z_bottom, const int32_t* group, double weight) {
    LF_RET_IF(model_ready(c));
    if (n < 0 || (n > 0 && (!xy || !z_top || !z_bottom || !group)) || !std::isfinite(weight))
        return fail(c, LF_EINVAL, "lf_set_constraints: bad arrays or weight");
    if (n > 0 && (!finite_all(xy, 2 * (size_t)n) || !finite_all(z_top, n) || !finite_all(z_bottom, n)))
        return fail(c, LF_EINVAL, "lf_set_constraints: non-finite constraint");
    std::vector<double> mid(3 * (size_t)n), thick(n);
    for (int k = 0; k < n; ++k) {
        // computeViolation (constraint_handler.cpp:16-29): depth positive down
        mid[3 * k] = xy[2 * k];
        mid[3 * k + 1] = xy[2 * k + 1];
        mid[3 * k + 2] = -(z_top[k] + z_bottom[k]) / 2.0;
        thick[k] = std::abs(z_bottom[k] - z_top[k]);
    }
    LF_TRY_CUDA(c, upload(c->d_cMid, mid.data(), mid.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_cThick, thick.data(), thick.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_cGroup, group, (size_t)n, c->stream));
    LF_TRY_CUDA(c, c->d_cCls.reserve(n));
    LF_TRY_CUDA(c, c->d_cOut.reserve(1));
    LF_TRY_CUDA(c, c->d_clsMask.reserve(std::max<size_t>(c->d_clsMask.n, n)));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    c->epoch++;
    c->nCons = n;
    c->consWeight = weight;
    return LF_OK;
}

extern "C" lf_status lf_constraint_penalty(lf_ctx* c, const double* params, double* value) {
    LF_RET_IF(model_ready(c));
    if (!value) return fail(c, LF_EINVAL, "null value");
    LF_RET_IF(constraint_params(c, params));
    LF_TRY_CUDA(c, c->d_cOut.reserve(1));
    LF_TRY_CUDA(c, upload(c->d_grpTriOffDev, c->grpTriOff.data(), c->grpTriOff.size(), c->stream));
    LF_RET_IF(constraint_eval_dev(c, c->d_cOut.p));
    LF_TRY_CUDA(c, cudaMemcpyAsync(value, c->d_cOut.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

extern "C" lf_status lf_constraint_gradient(lf_ctx* c, const double* params, double* grad) {
    LF_RET_IF(model_ready(c));
    if (c->np > 0 && !grad) return fail(c, LF_EINVAL, "null grad");
    LF_RET_IF(constraint_params(c, params));
    if (c->np == 0) return LF_OK;
    LF_TRY_CUDA(c, upload(c->d_cPar0, params, c->np, c->stream));
    LF_TRY_CUDA(c, c->d_cFp.reserve(c->np));
    LF_TRY_CUDA(c, c->d_cFm.reserve(c->np));
    LF_TRY_CUDA(c, c->d_cGrad.reserve(c->np));
    LF_TRY_CUDA(c, upload(c->d_grpTriOffDev, c->grpTriOff.data(), c->grpTriOff.size(), c->stream));
    // The 2 np passes are sequential (each scatter starts from the positions
    // the previous one left, as the reference's model does) and each is a
    // handful of short launches, so the sweep is replayed as one CUDA graph
    // after its first direct run.
    auto sweep = [c]() -> lf_status {
        const double h = 1.0;  // constraint_handler.cpp:54
        for (int j = 0; j < c->np; ++j) {
            k_constraint_step<<<1, 32, 0, c->stream>>>(c->d_cPar.p, c->d_cPar0.p, j, h, 0);
            LF_RET_IF(constraint_eval_dev(c, c->d_cFp.p + j));
            k_constraint_step<<<1, 32, 0, c->stream>>>(c->d_cPar.p, c->d_cPar0.p, j, h, 1);
            LF_RET_IF(constraint_eval_dev(c, c->d_cFm.p + j));
            k_constraint_step<<<1, 32, 0, c->stream>>>(c->d_cPar.p, c->d_cPar0.p, j, h, 2);
            c->counters.launches += 3;
        }
        k_constraint_fd<<<cdiv(c->np, 256), 256, 0, c->stream>>>(c->np, c->d_cFp.p, c->d_cFm.p, h,
                                                                  c->consWeight, c->d_cGrad.p);
        c->counters.launches++;
        LF_CHECK_LAUNCH(c);
        return LF_OK;
    };
    // graph replay up to 4096 parameters (about 66k graph nodes); beyond that
    // the capture itself would cost more than the launches it saves
    if (c->np <= 4096)
        LF_RET_IF(run_cached(c, c->gCons, c->d_cPar0.p, c->d_cFp.p, c->d_cGrad.p, sweep, true));
    else
        LF_RET_IF(sweep());
    LF_TRY_CUDA(c, cudaMemcpyAsync(grad, c->d_cGrad.p, sizeof(double) * c->np, cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

// ------------------------------------------------------ gradient smoothing --
// InversionRunner::smoothGradient (runner.cpp:643-706) on device buffers.
static lf_status gsmooth_tables(lf_ctx* c) {
    if (c->gnReady) return LF_OK;
    const int V = c->V, T = c->T;
    std::vector<int32_t> tri((size_t)3 * T);
    LF_TRY_CUDA(c, cudaMemcpyAsync(tri.data(), c->d_tri.p, sizeof(int32_t) * tri.size(), cudaMemcpyDeviceToHost,
                                   c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    // SurfaceMesh::buildNeighbors (surface_mesh.cpp:265-286): sorted, unique
    std::vector<std::vector<int32_t>> nb(V);
    for (int t = 0; t < T; ++t) {
        const int a = tri[3 * t], b = tri[3 * t + 1], d = tri[3 * t + 2];
        nb[a].push_back(b); nb[a].push_back(d);
        nb[b].push_back(a); nb[b].push_back(d);
        nb[d].push_back(a); nb[d].push_back(b);
    }
    std::vector<int32_t> off(V + 1, 0), list;
    for (int v = 0; v < V; ++v) {
        std::sort(nb[v].begin(), nb[v].end());
        nb[v].erase(std::unique(nb[v].begin(), nb[v].end()), nb[v].end());
        list.insert(list.end(), nb[v].begin(), nb[v].end());
        off[v + 1] = static_cast<int32_t>(list.size());
    }
    if (list.empty()) list.push_back(0);
    LF_TRY_CUDA(c, upload(c->d_gnOff, off.data(), off.size(), c->stream));
    LF_TRY_CUDA(c, upload(c->d_gnList, list.data(), list.size(), c->stream));
    LF_TRY_CUDA(c, c->d_gsVg.reserve((size_t)3 * V));
    LF_TRY_CUDA(c, c->d_gsSg.reserve((size_t)3 * V));
    LF_TRY_CUDA(c, c->d_gsHas.reserve((size_t)3 * V));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    c->gnReady = true;
    return LF_OK;
}

extern "C" lf_status lf_smooth_gradient_device(lf_ctx* c, double weight, const double* d_in, double* d_out) {
    if (!c) return LF_EINVAL;
    if (!c->hasModel) return fail(c, LF_ESTATE, "no model set");
    if (!std::isfinite(weight)) return fail(c, LF_EINVAL, "lf_smooth_gradient: non-finite weight");
    if (c->np == 0) return LF_OK;
    if (!d_in || !d_out) return fail(c, LF_EINVAL, "lf_smooth_gradient: null gradient");
    cudaSetDevice(c->device);
    if (weight <= 0.0) {  // runner.cpp:645: the gradient unchanged
        if (d_out != d_in)
            LF_TRY_CUDA(c, cudaMemcpyAsync(d_out, d_in, sizeof(double) * c->np, cudaMemcpyDeviceToDevice, c->stream));
        return LF_OK;
    }
    LF_RET_IF(gsmooth_tables(c));
    LF_TRY_CUDA(c, cudaMemsetAsync(c->d_gsHas.p, 0, (size_t)3 * c->V, c->stream));
    k_gsmooth_scatter<<<cdiv(c->np, 256), 256, 0, c->stream>>>(c->np, c->d_dofOff.p, c->d_refVertex.p, c->d_refAxis.p,
                                                               d_in, c->d_gsVg.p, c->d_gsHas.p);
    k_gsmooth_vertex<<<cdiv(3 * (long long)c->V, 256), 256, 0, c->stream>>>(c->V, c->d_gnOff.p, c->d_gnList.p,
                                                                           c->d_gsVg.p, c->d_gsHas.p, weight,
                                                                           c->d_gsSg.p);
    k_gsmooth_gather<<<cdiv(c->np, 256), 256, 0, c->stream>>>(c->np, c->d_dofOff.p, c->d_refVertex.p, c->d_refAxis.p,
                                                              d_in, c->d_gsSg.p, d_out);
    c->counters.launches += 3;
    LF_CHECK_LAUNCH(c);
    return LF_OK;
}

extern "C" lf_status lf_smooth_gradient(lf_ctx* c, double weight, const double* grad_in, double* grad_out) {
    if (!c) return LF_EINVAL;
    if (!c->hasModel) return fail(c, LF_ESTATE, "no model set");
    if (c->np == 0) return LF_OK;
    if (!grad_in || !grad_out) return fail(c, LF_EINVAL, "lf_smooth_gradient: null gradient");
    if (!finite_all(grad_in, c->np)) return fail(c, LF_EINVAL, "lf_smooth_gradient: non-finite gradient");
    cudaSetDevice(c->device);
    LF_TRY_CUDA(c, upload(c->d_gsIn, grad_in, (size_t)c->np, c->stream));
    LF_TRY_CUDA(c, c->d_cGrad.reserve(c->np));
    LF_RET_IF(lf_smooth_gradient_device(c, weight, c->d_gsIn.p, c->d_cGrad.p));
    LF_TRY_CUDA(c, cudaMemcpyAsync(grad_out, c->d_cGrad.p, sizeof(double) * c->np, cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    return LF_OK;
}

// ------------------------------------------------------------ validation --
// LithologyModel::validate (lithology_model.cpp:624-803): the six quality
// checks in the reference's order, the first failure returned.  Vertex
// positions come from the device; the two overlap counts classify every
// vertex with the GPU ray cast (the O(V x T) part); the rest is O(V) host
// work over the downloaded positions.  Neighbour lists as
// SurfaceMesh::buildNeighbors, which the runner calls at set-up.
extern "C" lf_status lf_validate_model(lf_ctx* c, const double* params, const uint8_t* freedom,
                                       unsigned long long overlap_baseline,
                                       unsigned long long adjacent_overlap_baseline, int* passed, double* worst,
                                       char* reason, int reason_len) {
    LF_RET_IF(model_ready(c));
    if (!passed || !worst) return fail(c, LF_EINVAL, "lf_validate_model: null result");
    if (params) {
        LF_RET_IF(constraint_params(c, params));
        LF_RET_IF(scatter(c, c->d_cPar.p));
    }
    const uint8_t* fr = freedom ? freedom : (c->vertexFreedom.empty() ? nullptr : c->vertexFreedom.data());
    if (!fr) return fail(c, LF_EINVAL, "lf_validate_model: no vertex freedoms known (pass freedom[n_vertices])");
    *passed = 1;
    *worst = 0.0;
    std::string why;
    auto finish = [&](lf_status st) -> lf_status {
        if (reason && reason_len > 0) {
            std::strncpy(reason, why.c_str(), (size_t)reason_len - 1);
            reason[reason_len - 1] = '\0';
        }
        return st;
    };
    const int G = c->G, V = c->V, T = c->T;
    if (G < 2) return finish(LF_OK);
    std::vector<double> pos((size_t)3 * V);
    std::vector<int32_t> tri((size_t)3 * T);
    LF_TRY_CUDA(c, cudaMemcpyAsync(pos.data(), c->d_pos.p, sizeof(double) * pos.size(), cudaMemcpyDeviceToHost,
                                   c->stream));
    LF_TRY_CUDA(c, cudaMemcpyAsync(tri.data(), c->d_tri.p, sizeof(int32_t) * tri.size(), cudaMemcpyDeviceToHost,
                                   c->stream));
    std::vector<int32_t> syncOff, syncVertex;
    if (c->nSync > 0) {
        syncOff.resize(c->nSync + 1);
        LF_TRY_CUDA(c, cudaMemcpyAsync(syncOff.data(), c->d_syncOff.p, sizeof(int32_t) * syncOff.size(),
                                       cudaMemcpyDeviceToHost, c->stream));
        LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
        syncVertex.resize(syncOff.back());
        if (!syncVertex.empty())
            LF_TRY_CUDA(c, cudaMemcpyAsync(syncVertex.data(), c->d_syncVertex.p, sizeof(int32_t) * syncVertex.size(),
                                           cudaMemcpyDeviceToHost, c->stream));
    }
    // classification of every vertex (checks 2 and 3)
    LF_TRY_CUDA(c, c->d_ptCls.reserve(V));
    LF_TRY_CUDA(c, c->d_clsMask.reserve(std::max<size_t>(c->d_clsMask.n, V)));
    LF_RET_IF(classify_dev(c, V, c->d_pos.p, c->d_ptCls.p));
    std::vector<int32_t> cls(V);
    LF_TRY_CUDA(c, cudaMemcpyAsync(cls.data(), c->d_ptCls.p, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, c->stream));
    LF_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    // vertex range of each group mesh (meshes are stored one after another):
    // the builder's offsets, else the range the group's triangles use
    std::vector<int32_t> vlo(G, V), vhi(G, -1);
    if ((int)c->grpVertOff.size() == G + 1) {
        for (int g = 0; g < G; ++g) {
            vlo[g] = c->grpVertOff[g];
            vhi[g] = c->grpVertOff[g + 1] - 1;
        }
    } else {
        for (int g = 0; g < G; ++g)
            for (int t = c->grpTriOff[g]; t < c->grpTriOff[g + 1]; ++t)
                for (int k = 0; k < 3; ++k) {
                    vlo[g] = std::min(vlo[g], tri[3 * t + k]);
                    vhi[g] = std::max(vhi[g], tri[3 * t + k]);
                }
    }
    auto P = [&](int v, int k) { return pos[3 * (size_t)v + k]; };
    auto dist = [&](int u, int v) {
        const double dx = P(u, 0) - P(v, 0), dy = P(u, 1) - P(v, 1), dz = P(u, 2) - P(v, 2);
        return std::sqrt(dx * dx + dy * dy + dz * dz);
    };
    double xmin = 1e30, xmax = -1e30, ymin = 1e30, ymax = -1e30, zmin = 1e30, zmax = -1e30;
    for (int g = 0; g < G; ++g)
        for (int v = vlo[g]; v <= vhi[g]; ++v) {
            xmin = std::min(xmin, P(v, 0)); xmax = std::max(xmax, P(v, 0));
            ymin = std::min(ymin, P(v, 1)); ymax = std::max(ymax, P(v, 1));
            zmin = std::min(zmin, P(v, 2)); zmax = std::max(zmax, P(v, 2));
        }
    const double modelDim = std::max({xmax - xmin, ymax - ymin, zmax - zmin, 1.0});
    const double aabbMargin = modelDim * 0.02;
    // 1: shared vertex gaps
    for (int s = 0; s < c->nSync; ++s) {
        if (syncOff[s + 1] - syncOff[s] < 2) continue;
        const int r = syncVertex[syncOff[s]];
        for (int k = syncOff[s] + 1; k < syncOff[s + 1]; ++k) {
            const double gap = dist(syncVertex[k], r);
            if (gap > 0.1) {
                *passed = 0;
                *worst = std::max(*worst, gap);
                why = "Shared vertex gap: " + std::to_string(gap) + "m";
                return finish(LF_OK);
            }
        }
    }
    // 2 and 3: vertices of group g classified into another group
    unsigned long long adj = 0, nonAdj = 0;
    for (int g = 0; g < G; ++g)
        for (int v = vlo[g]; v <= vhi[g]; ++v) {
            const int k = cls[v];
            if (k < 0 || k == g) continue;
            if (std::abs(k - g) == 1) ++adj;
            else ++nonAdj;
        }
    const unsigned long long adjLimit = adjacent_overlap_baseline + 20;
    if (adj > adjLimit) {
        *passed = 0;
        *worst = static_cast<double>(adj - adjacent_overlap_baseline);
        why = "Adjacent overlap: " + std::to_string(adj) + " (baseline=" + std::to_string(adjacent_overlap_baseline) +
              ", limit=" + std::to_string(adjLimit) + ")";
        return finish(LF_OK);
    }
    const unsigned long long overlapLimit = overlap_baseline + 120;
    if (nonAdj > overlapLimit) {
        *passed = 0;
        *worst = static_cast<double>(nonAdj - overlap_baseline);
        why = "Non-adjacent overlap: " + std::to_string(nonAdj) + " (baseline=" + std::to_string(overlap_baseline) +
              ", limit=" + std::to_string(overlapLimit) + ")";
        return finish(LF_OK);
    }
    // 4: boundary vertices (not XYZ-free) quantised to 0.1 mm must stay together
    std::map<std::array<int64_t, 3>, std::vector<int>> boundary;
    for (int g = 0; g < G; ++g)
        for (int v = vlo[g]; v <= vhi[g]; ++v) {
            if (fr[v] == LF_XYZ_FREE) continue;
            const std::array<int64_t, 3> key = {static_cast<int64_t>(std::round(P(v, 0) * 1e4)),
                                                static_cast<int64_t>(std::round(P(v, 1) * 1e4)),
                                                static_cast<int64_t>(std::round(P(v, 2) * 1e4))};
            boundary[key].push_back(v);
        }
    for (const auto& kv : boundary) {
        const std::vector<int>& vs = kv.second;
        for (size_t i = 1; i < vs.size(); ++i) {
            const double gap = dist(vs[i], vs[0]);
            if (gap > 0.1) {
                *passed = 0;
                *worst = std::max(*worst, gap);
                why = "Edge tearing: boundary vertices diverged by " + std::to_string(gap) + "m";
                return finish(LF_OK);
            }
        }
    }
    // 5: containment in the model's (own) bounding box with a 2 % margin
    for (int g = 0; g < G; ++g)
        for (int v = vlo[g]; v <= vhi[g]; ++v) {
            const double x = P(v, 0), y = P(v, 1), z = P(v, 2);
            if (x < xmin - aabbMargin || x > xmax + aabbMargin || y < ymin - aabbMargin || y > ymax + aabbMargin ||
                z < zmin - aabbMargin || z > zmax + aabbMargin) {
                *passed = 0;
                *worst = std::max({xmin - aabbMargin - x, x - xmax - aabbMargin, ymin - aabbMargin - y,
                                   y - ymax - aabbMargin, zmin - aabbMargin - z, z - zmax - aabbMargin, 0.0});
                why = "AABB containment: vertex in group " + std::to_string(g) + " outside model envelope";
                return finish(LF_OK);
            }
        }
    // 6: spikes -- |vertex - mean of its mesh neighbours| above modelDim / 5
    const double spikeThreshold = modelDim / 5.0;
    std::vector<std::vector<int32_t>> nb(V);
    for (int t = 0; t < T; ++t) {
        const int a = tri[3 * t], b = tri[3 * t + 1], d = tri[3 * t + 2];
        nb[a].push_back(b); nb[a].push_back(d);
        nb[b].push_back(a); nb[b].push_back(d);
        nb[d].push_back(a); nb[d].push_back(b);
    }
    for (int g = 0; g < G; ++g)
        for (int v = vlo[g]; v <= vhi[g]; ++v) {
            std::vector<int32_t>& l = nb[v];
            std::sort(l.begin(), l.end());
            l.erase(std::unique(l.begin(), l.end()), l.end());
            if (l.empty()) continue;
            double ax = 0.0, ay = 0.0, az = 0.0;
            for (int32_t u : l) {
                ax += P(u, 0);
                ay += P(u, 1);
                az += P(u, 2);
            }
            const double n = static_cast<double>(l.size());
            ax /= n; ay /= n; az /= n;
            const double lx = P(v, 0) - ax, ly = P(v, 1) - ay, lz = P(v, 2) - az;
            const double mag = std::sqrt(lx * lx + ly * ly + lz * lz);
            if (mag > spikeThreshold) {
                *passed = 0;
                *worst = mag;
                why = "Spike detected: vertex in group " + std::to_string(g) + " vi=" + std::to_string(v - vlo[g]) +
                      " Laplacian=" + std::to_string(mag) + "m (threshold=" + std::to_string(spikeThreshold) + "m)";
                return finish(LF_OK);
            }
        }
    return finish(LF_OK);
}
