// ref_wrap.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A thin extern "C" harness around the reference's own, unmodified C++
// classes (LithologyModel, SurfaceMesh, GravityForward, MagneticForward,
// ObjectiveFunction, JointObjective, ReferenceModelRegularization,
// LBFGSBOptimizer).  oracle/Makefile compiles it together with the
// reference's sources into oracle/_ref/libref_litho.so.  It is used to pin
// the C restatement (oracle/litho_oracle.c) and the product's DOF builder,
// and, as `kind: "reference"`, as the timed CPU baseline.  Nothing in the
// product library links or loads it.
#include <litho_invert/forward/gravity_forward.h>
#include <litho_invert/forward/magnetic_forward.h>
#include <litho_invert/inversion/constraint_handler.h>
#include <litho_invert/io/exporters.h>
#include <litho_invert/io/surface_loader.h>
#include <litho_invert/inversion/joint_objective.h>
#include <litho_invert/inversion/lbfgsb_optimizer.h>
#include <litho_invert/inversion/objective.h>
#include <litho_invert/litho/lithology_model.h>
#include <litho_invert/regularization/reference_model.h>
#include <litho_invert/regularization/smoothness.h>
#include <litho_invert/core/geometry.h>

#include "gpu_dropin.hpp"

#include <array>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace litho_invert;

namespace {
struct RefCtx {
    std::shared_ptr<LithologyModel> model = std::make_shared<LithologyModel>();
    GravityData grav;
    MagneticData mag;
    double inc = 90.0, dec = 0.0, field = 50000.0;
    int remMode = 0;
    std::shared_ptr<GravityForward> gf;
    std::shared_ptr<MagneticForward> mf;
    std::shared_ptr<ObjectiveFunction> gobj;
    std::shared_ptr<JointObjective> jobj;
    std::shared_ptr<ReferenceModelRegularization> refReg;
    double alphaMag = 1.0;
    double refWeight = 0.0;
    double smoothWeight = 0.0;
    std::shared_ptr<SurfaceSmoothness> smooth;
    VectorXd refParams;
    std::shared_ptr<ConstraintHandler> cons;
    bool built = false;
    // the operators the objective runs on: the reference's own forwards, or
    // the GPU drop-ins after ref_use_gpu
    std::shared_ptr<litho_dropin::GpuSession> gpu;
    std::shared_ptr<ForwardModel> gfwd;
    std::shared_ptr<MagneticForward> mfwd;

    void build() {
        gf = std::make_shared<GravityForward>(model, grav);
        mf = std::make_shared<MagneticForward>(model, mag, inc, dec, field);
        mf->setRemanenceMode(static_cast<RemanentMagnetizationMode>(remMode));
        gfwd = gf;
        mfwd = mf;
        if (gpu) {
            gfwd = std::make_shared<litho_dropin::GpuGravityForward>(gpu);
            mfwd = std::make_shared<litho_dropin::GpuMagneticForward>(gpu, model, mag, inc, dec, field);
        }
        gobj = std::make_shared<ObjectiveFunction>(gfwd, grav);
        // the runner registers the smoothness first, then the reference model
        // (runner.cpp:164-179)
        smooth = std::make_shared<SurfaceSmoothness>(model);
        smooth->setWeight(smoothWeight);
        if (smoothWeight > 0.0) gobj->addRegularization(smooth);
        if (refWeight > 0.0 && refParams.size() > 0) {
            refReg = std::make_shared<ReferenceModelRegularization>(model);
            refReg->setWeight(refWeight);
            refReg->captureReference(refParams);
            gobj->addRegularization(refReg);
        }
        jobj = std::make_shared<JointObjective>(gobj, mag.empty() ? nullptr : mfwd, mag, alphaMag);
        built = true;
    }
    void ensure() { if (!built) build(); }
};
VectorXd toVec(int n, const double* p) {
    VectorXd v(n);
    for (int i = 0; i < n; ++i) v[i] = p[i];
    return v;
}
void fromVec(const VectorXd& v, double* p) {
    for (Eigen::Index i = 0; i < v.size(); ++i) p[i] = v[i];
}
void fromMat(const MatrixXd& J, double* p) {  // row-major out
    for (Eigen::Index i = 0; i < J.rows(); ++i)
        for (Eigen::Index j = 0; j < J.cols(); ++j) p[i * J.cols() + j] = J(i, j);
}
}  // namespace

extern "C" {

void* ref_new() { return new RefCtx(); }
void ref_free(void* h) { delete static_cast<RefCtx*>(h); }

// Adds a group (LithoGroup, litho_group.h:13-34).  LithoGroup::isValid rejects
// density <= 0, so the density is written after addGroup, as a caller must.
int ref_add_group(void* h, int id, double density, double susceptibility, double rem_mag,
                  double rem_inc, double rem_dec, const double* rem_vec) {
    auto* c = static_cast<RefCtx*>(h);
    LithoGroup g(id, "group" + std::to_string(id), 1.0, susceptibility);
    g.remanence_magnitude = rem_mag;
    g.remanence_inclination = rem_inc;
    g.remanence_declination = rem_dec;
    if (rem_vec) g.magnetization = Vector3d(rem_vec[0], rem_vec[1], rem_vec[2]);
    int idx = c->model->addGroup(g);
    if (idx >= 0) c->model->group(idx).density = density;
    c->built = false;
    return idx;
}

// freedom[v] uses the VertexFreedom numbering (surface_mesh.h:9-19).
int ref_set_mesh(void* h, int group, int nv, const double* xyz, const uint8_t* freedom, int nt,
                 const int32_t* tri, const double* axis_scale3, double min_z, double max_z) {
    auto* c = static_cast<RefCtx*>(h);
    auto mesh = std::make_shared<SurfaceMesh>();
    for (int v = 0; v < nv; ++v)
        mesh->addVertex(Vector3d(xyz[3 * v], xyz[3 * v + 1], xyz[3 * v + 2]),
                        static_cast<VertexFreedom>(freedom[v]));
    for (int t = 0; t < nt; ++t) mesh->addTriangle(tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]);
    for (int a = 0; a < 3; ++a) mesh->setAxisScale(a, axis_scale3[a]);
    mesh->setBounds(min_z, max_z);
    c->model->setGroupMesh(group, mesh);
    c->built = false;
    return 0;
}

int ref_set_control_point_stride(void* h, int stride) {
    auto* c = static_cast<RefCtx*>(h);
    return static_cast<int>(c->model->setControlPointStride(stride));
}
void ref_build_shared_sync(void* h) { static_cast<RefCtx*>(h)->model->buildSharedVertexSync(); }
void ref_apply_model_bounds(void* h, double margin) {
    static_cast<RefCtx*>(h)->model->applyModelBounds(margin);
}

int ref_dof_count(void* h) { return static_cast<int>(static_cast<RefCtx*>(h)->model->totalDofCount()); }

int ref_vertex_count(void* h) {
    auto* c = static_cast<RefCtx*>(h);
    int n = 0;
    for (int m = 0; m < c->model->groupMeshCount(); ++m)
        if (c->model->groupMesh(m)) n += static_cast<int>(c->model->groupMesh(m)->vertexCount());
    return n;
}

// Global DOF tables: for each global DOF, its (global vertex, axis, axis
// scale) refs in (mesh, local DOF) order.  Returns the number of refs.
int ref_dof_tables(void* h, int32_t* dof_off, int32_t* ref_vertex, uint8_t* ref_axis,
                   double* ref_scale) {
    auto* c = static_cast<RefCtx*>(h);
    auto& M = *c->model;
    int np = static_cast<int>(M.totalDofCount());
    std::vector<std::vector<std::array<double, 3>>> refs(np);
    int vbase = 0;
    for (int m = 0; m < M.groupMeshCount(); ++m) {
        const SurfaceMesh* mesh = M.groupMesh(m);
        if (!mesh) continue;
        const auto& maps = mesh->dofMappings();
        for (int l = 0; l < static_cast<int>(maps.size()); ++l) {
            int g = M.globalDofIndex(m, l);
            if (g < 0) continue;
            refs[g].push_back({double(vbase + maps[l].vertexIndex), double(maps[l].axis),
                               mesh->axisScale(maps[l].axis)});
        }
        vbase += static_cast<int>(mesh->vertexCount());
    }
    int k = 0;
    dof_off[0] = 0;
    for (int g = 0; g < np; ++g) {
        for (auto& r : refs[g]) {
            ref_vertex[k] = static_cast<int32_t>(r[0]);
            ref_axis[k] = static_cast<uint8_t>(r[1]);
            ref_scale[k] = r[2];
            ++k;
        }
        dof_off[g + 1] = k;
    }
    return k;
}

void ref_is_control_point(void* h, uint8_t* out) {
    auto* c = static_cast<RefCtx*>(h);
    int k = 0;
    for (int m = 0; m < c->model->groupMeshCount(); ++m) {
        const SurfaceMesh* mesh = c->model->groupMesh(m);
        if (!mesh) continue;
        for (uint32_t v = 0; v < mesh->vertexCount(); ++v) out[k++] = mesh->isControlPoint(v) ? 1 : 0;
    }
}

void ref_assemble(void* h, double* params) { fromVec(static_cast<RefCtx*>(h)->model->assembleParameterVector(), params); }

void ref_bounds(void* h, double* lo, double* hi) {
    VectorXd l, u;
    static_cast<RefCtx*>(h)->model->getBounds(l, u);
    fromVec(l, lo);
    fromVec(u, hi);
}

void ref_apply(void* h, const double* params) {
    auto* c = static_cast<RefCtx*>(h);
    c->model->applyParameterVector(toVec(static_cast<int>(c->model->totalDofCount()), params));
}

void ref_positions(void* h, double* out) {
    auto* c = static_cast<RefCtx*>(h);
    int k = 0;
    for (int m = 0; m < c->model->groupMeshCount(); ++m) {
        const SurfaceMesh* mesh = c->model->groupMesh(m);
        if (!mesh) continue;
        for (uint32_t v = 0; v < mesh->vertexCount(); ++v) {
            const auto& p = mesh->vertex(v).position;
            out[k++] = p.x(); out[k++] = p.y(); out[k++] = p.z();
        }
    }
}

void ref_set_gravity(void* h, int n, const double* xyz, const double* obs, const double* std) {
    auto* c = static_cast<RefCtx*>(h);
    c->grav.clear();
    for (int i = 0; i < n; ++i)
        c->grav.emplace_back(Vector3d(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]), obs ? obs[i] : 0.0,
                             std ? std[i] : 0.0);
    c->built = false;
}

void ref_set_magnetic(void* h, int n, const double* xyz, const double* obs, const double* std,
                      double inc, double dec, double field, int rem_mode) {
    auto* c = static_cast<RefCtx*>(h);
    c->mag.clear();
    for (int i = 0; i < n; ++i)
        c->mag.emplace_back(Vector3d(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]), obs ? obs[i] : 0.0,
                            std ? std[i] : 0.0);
    c->inc = inc; c->dec = dec; c->field = field; c->remMode = rem_mode;
    c->built = false;
}

void ref_set_objective(void* h, double alpha_mag, double ref_weight, const double* ref_params) {
    auto* c = static_cast<RefCtx*>(h);
    c->alphaMag = alpha_mag;
    c->refWeight = ref_weight;
    if (ref_params) c->refParams = toVec(static_cast<int>(c->model->totalDofCount()), ref_params);
    c->built = false;
}

// LithologyModel::setLabelGrid / setBottomDepth / classifyPoint
// (lithology_model.cpp:89-103, 856-858, 288-363) on the current positions.
void ref_set_label_grid(void* h, int nx, int ny, int nz, double x0, double y0, double z0, double dx, double dy,
                        double dz, const int32_t* labels) {
    std::vector<int> lab(labels ? static_cast<size_t>(nx) * ny * nz : 0);
    for (size_t i = 0; i < lab.size(); ++i) lab[i] = labels[i];
    static_cast<RefCtx*>(h)->model->setLabelGrid(lab, nx, ny, nz, x0, y0, z0, dx, dy, dz);
}
void ref_set_bottom_depth(void* h, double depth) { static_cast<RefCtx*>(h)->model->setBottomDepth(depth); }
void ref_classify(void* h, int n, const double* xyz, int32_t* out) {
    auto* c = static_cast<RefCtx*>(h);
    for (int i = 0; i < n; ++i) out[i] = c->model->classifyPoint(Vector3d(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
}

// ConstraintHandler (constraint_handler.cpp:7-66).
void ref_set_constraints(void* h, int n, const double* xy, const double* z_top, const double* z_bottom,
                         const int32_t* group, double weight) {
    auto* c = static_cast<RefCtx*>(h);
    std::vector<Constraint> cs(n);
    for (int k = 0; k < n; ++k) {
        cs[k].position = Vector3d(xy[2 * k], xy[2 * k + 1], 0.0);
        cs[k].z_top = z_top[k];
        cs[k].z_bottom = z_bottom[k];
        cs[k].litho_group_id = group[k];
    }
    c->cons = std::make_shared<ConstraintHandler>(c->model, cs);
    c->cons->setWeight(weight);
}
double ref_constraint_value(void* h, const double* params) {
    auto* c = static_cast<RefCtx*>(h);
    return c->cons->evaluate(toVec(static_cast<int>(c->model->totalDofCount()), params));
}
void ref_constraint_gradient(void* h, const double* params, double* grad) {
    auto* c = static_cast<RefCtx*>(h);
    fromVec(c->cons->gradient(toVec(static_cast<int>(c->model->totalDofCount()), params)), grad);
}

// JointObjective::calibrateDataWeights (joint_objective.cpp:281-393) at
// params; returns the new magnetic weight.
double ref_calibrate(void* h, const double* params) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    c->jobj->calibrateDataWeights(toVec(static_cast<int>(c->jobj->parameterCount()), params));
    return c->jobj->magneticWeight();
}

void ref_set_smoothness(void* h, double weight) {
    auto* c = static_cast<RefCtx*>(h);
    c->smoothWeight = weight;
    c->built = false;
}

// SurfaceSmoothness::evaluate / gradient (smoothness.cpp:20-390) with the
// weight set by ref_set_smoothness.
double ref_smoothness_value(void* h, const double* params) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    return c->smooth->evaluate(toVec(static_cast<int>(c->model->totalDofCount()), params));
}
void ref_smoothness_gradient(void* h, const double* params, double* grad) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    fromVec(c->smooth->gradient(toVec(static_cast<int>(c->model->totalDofCount()), params)), grad);
}

void ref_group_magnetization(void* h, int g, double* amp, double* dir3) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    Vector3d d;
    c->mf->buildGroupMagnetization(g, *amp, d);
    dir3[0] = d.x(); dir3[1] = d.y(); dir3[2] = d.z();
}

void ref_forward_gz(void* h, const double* params, double* out) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    fromVec(c->gfwd->compute(toVec(static_cast<int>(c->gfwd->parameterCount()), params)), out);
}

void ref_forward_tmi(void* h, const double* params, double* out) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    fromVec(c->mfwd->compute(toVec(static_cast<int>(c->mfwd->parameterCount()), params)), out);
}

// Unit responses at params (kind 0 gravity, 1 induced, 2 direction, 3 remanence).
void ref_unit_response(void* h, const double* params, int kind, int group, const double* dir, double* out) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    c->model->applyParameterVector(toVec(static_cast<int>(c->gf->parameterCount()), params));
    VectorXd r;
    if (kind == 0) r = c->gf->computeGroupUnitResponse(group);
    else if (kind == 1) r = c->mf->computeGroupUnitResponse(group);
    else if (kind == 2) r = c->mf->computeGroupUnitResponseDirection(group, Vector3d(dir[0], dir[1], dir[2]));
    else r = c->mf->computeGroupUnitRemanenceResponse(group);
    fromVec(r, out);
}

// loadSurfaceMesh (surface_loader.cpp:163-181): counts, and with non-null
// buffers the vertices and 0-based triangles; 0 when the loader returns null.
int ref_load_surface(const char* path, int* nv, int* nt, double* xyz, int32_t* tri) {
    auto mesh = loadSurfaceMesh(path);
    if (!mesh) return 0;
    *nv = static_cast<int>(mesh->vertexCount());
    *nt = static_cast<int>(mesh->triangleCount());
    if (xyz)
        for (uint32_t i = 0; i < mesh->vertexCount(); ++i)
            for (int k = 0; k < 3; ++k) xyz[3 * i + k] = mesh->vertex(i).position[k];
    if (tri)
        for (uint32_t i = 0; i < mesh->triangleCount(); ++i) {
            const Triangle& t = mesh->triangle(i);
            tri[3 * i] = static_cast<int32_t>(t.v0);
            tri[3 * i + 1] = static_cast<int32_t>(t.v1);
            tri[3 * i + 2] = static_cast<int32_t>(t.v2);
        }
    return 1;
}

// InversionExporter(dir, base).exportTS(mesh, suffix) of the given surface.
void ref_export_ts(const char* dir, const char* base, const char* suffix, int nv, const double* xyz, int nt,
                   const int32_t* tri) {
    SurfaceMesh mesh;
    for (int i = 0; i < nv; ++i) mesh.addVertex(Vector3d(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
    for (int i = 0; i < nt; ++i)
        mesh.addTriangle(static_cast<uint32_t>(tri[3 * i]), static_cast<uint32_t>(tri[3 * i + 1]),
                         static_cast<uint32_t>(tri[3 * i + 2]));
    InversionExporter(dir, base).exportTS(mesh, suffix);
}

// LithologyModel::validate (lithology_model.cpp:624-803) on the current
// positions, neighbours built as the runner builds them (runner.cpp:59).
int ref_validate(void* h, unsigned long long overlap_baseline, unsigned long long adjacent_baseline, double* worst,
                 char* reason, int reason_len) {
    auto* c = static_cast<RefCtx*>(h);
    for (int i = 0; i < c->model->groupMeshCount(); ++i)
        if (c->model->groupMesh(i)) c->model->groupMesh(i)->buildNeighbors();
    const ValidationResult r = c->model->validate(overlap_baseline, adjacent_baseline);
    *worst = r.worstViolation;
    std::strncpy(reason, r.failureReason.c_str(), (size_t)reason_len - 1);
    reason[reason_len - 1] = '\0';
    return r.passed ? 1 : 0;
}

// InversionRunner::smoothGradient (runner.cpp:643-706), restated with the
// reference model's public API (runner.cpp is not compiled here).
void ref_smooth_gradient(void* h, double w, const double* g_in, double* g_out) {
    auto* c = static_cast<RefCtx*>(h);
    for (int i = 0; i < c->model->groupMeshCount(); ++i)  // as the runner does at set-up (runner.cpp:59)
        if (c->model->groupMesh(i)) c->model->groupMesh(i)->buildNeighbors();
    const LithologyModel* model = c->model.get();
    const Index np = static_cast<Index>(model->totalDofCount());
    VectorXd g = toVec(static_cast<int>(np), g_in);
    VectorXd smoothed = g;
    if (w > 0.0) {
        const int nM = model->groupMeshCount();
        for (int mi = 0; mi < nM; ++mi) {
            const auto* mesh = model->groupMesh(mi);
            if (!mesh || mesh->vertexCount() == 0) continue;
            const auto& mappings = mesh->dofMappings();
            const uint32_t nVerts = mesh->vertexCount();
            std::vector<double> vertGrad(nVerts * 3, 0.0);
            std::vector<int> vertHasAxis(nVerts * 3, 0);
            for (uint32_t li = 0; li < mappings.size(); ++li) {
                const auto& dm = mappings[li];
                const int gi = model->globalDofIndex(mi, static_cast<int>(li));
                if (gi < 0 || gi >= g.size()) continue;
                const uint32_t idx = dm.vertexIndex * 3 + dm.axis;
                vertGrad[idx] = g[gi];
                vertHasAxis[idx] = 1;
            }
            std::vector<double> smoothGrad(nVerts * 3, 0.0);
            for (uint32_t vi = 0; vi < nVerts; ++vi) {
                const auto& neighbors = mesh->neighborVertices(vi);
                for (int a = 0; a < 3; ++a) {
                    const uint32_t idx = vi * 3 + a;
                    if (!vertHasAxis[idx]) continue;
                    double neighborSum = 0.0;
                    int nNbr = 0;
                    for (uint32_t ni : neighbors) {
                        const uint32_t nidx = ni * 3 + a;
                        if (vertHasAxis[nidx]) {
                            neighborSum += vertGrad[nidx];
                            ++nNbr;
                        }
                    }
                    if (nNbr > 0) {
                        const double neighborMean = neighborSum / nNbr;
                        smoothGrad[idx] = (1.0 - w) * vertGrad[idx] + w * neighborMean;
                    } else {
                        smoothGrad[idx] = vertGrad[idx];
                    }
                }
            }
            for (uint32_t li = 0; li < mappings.size(); ++li) {
                const auto& dm = mappings[li];
                const int gi = model->globalDofIndex(mi, static_cast<int>(li));
                if (gi < 0 || gi >= g.size()) continue;
                smoothed[gi] = smoothGrad[dm.vertexIndex * 3 + dm.axis];
            }
        }
    }
    fromVec(smoothed, g_out);
}

// InversionRunner::runPropertyInversion parts A and B (runner.cpp:708-917),
// restated with the reference's own classes (GravityForward /
// MagneticForward unit responses, LBFGSBOptimizer): runner.cpp itself needs
// the IO and EM modules and is not compiled here.  opt = {density min, max,
// chi min, max, remanence min, max, remanence component min, max, damping,
// tolerance}.  Returns the new properties and writes them into the groups.
void ref_property_inversion(void* h, const double* params, const double* opt, int max_iter, double* density,
                            double* magnetic) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    c->model->applyParameterVector(toVec(static_cast<int>(c->gf->parameterCount()), params));
    const int nGroups = c->model->groupCount();
    const double lambda = opt[8], tol = opt[9];
    auto solve = [&](const MatrixXd& U, const std::vector<double>& obsv, const std::vector<double>& sdv,
                     VectorXd x0, const VectorXd& lo, const VectorXd& hi) {
        const size_t n = obsv.size();
        double var = 0.0;
        for (size_t i = 0; i < n; ++i) var += obsv[i] * obsv[i];
        var /= static_cast<double>(n);
        const double rms = std::sqrt(std::max(var, 1.0));
        const VectorXd ref = x0;
        auto obj = [&](const VectorXd& d) -> double {
            VectorXd pred = U * d;
            double misfit = 0.0;
            for (size_t i = 0; i < n; ++i) {
                double w = (sdv[i] > 0) ? (1.0 / sdv[i]) : 1.0;
                double res = w * (obsv[i] - pred[static_cast<Index>(i)]);
                misfit += 0.5 * res * res;
            }
            misfit /= rms * rms;
            if (lambda > 0.0) {
                VectorXd diff = d - ref;
                misfit += 0.5 * lambda * diff.squaredNorm();
            }
            return misfit;
        };
        auto grad = [&](const VectorXd& d) -> VectorXd {
            VectorXd pred = U * d;
            VectorXd Wr(static_cast<Index>(n));
            double invScale2 = 1.0 / (rms * rms);
            for (size_t i = 0; i < n; ++i) {
                double w = (sdv[i] > 0) ? (1.0 / sdv[i]) : 1.0;
                Wr[static_cast<Index>(i)] = invScale2 * w * w * (obsv[i] - pred[static_cast<Index>(i)]);
            }
            VectorXd g = -U.transpose() * Wr;
            if (lambda > 0.0) g += lambda * (d - ref);
            return g;
        };
        LBFGSBOptimizer o;
        o.setMaxIterations(max_iter);
        o.setHistorySize(std::min(5, static_cast<int>(x0.size())));
        o.setTolerance(tol);
        return o.minimize(obj, grad, x0, lo, hi).params;
    };
    {  // part A
        const size_t n = c->grav.size();
        MatrixXd U(static_cast<Index>(n), nGroups);
        VectorXd x0(nGroups), lo(nGroups), hi(nGroups);
        std::vector<double> obsv(n), sdv(n);
        for (size_t i = 0; i < n; ++i) { obsv[i] = c->grav[i].g_obs; sdv[i] = c->grav[i].g_std; }
        for (int g = 0; g < nGroups; ++g) {
            U.col(g) = c->gf->computeGroupUnitResponse(g);
            x0[g] = c->model->group(g).density;
            lo[g] = opt[0];
            hi[g] = opt[1];
        }
        VectorXd d = solve(U, obsv, sdv, x0, lo, hi);
        for (int g = 0; g < nGroups; ++g) c->model->group(g).density = d[g];
    }
    if (!c->mag.empty()) {  // part B
        const int ppg = c->remMode == 1 ? 2 : (c->remMode == 2 ? 4 : 1);
        const size_t n = c->mag.size();
        const int m = ppg * nGroups;
        MatrixXd U(static_cast<Index>(n), m);
        VectorXd x0(m), lo(m), hi(m);
        std::vector<double> obsv(n), sdv(n);
        for (size_t i = 0; i < n; ++i) { obsv[i] = c->mag[i].t_obs; sdv[i] = c->mag[i].t_std; }
        for (int g = 0; g < nGroups; ++g) {
            const int col = ppg * g;
            U.col(col) = c->mf->computeGroupUnitResponse(g);
            x0[col] = c->model->group(g).susceptibility;
            lo[col] = opt[2];
            hi[col] = opt[3];
            if (ppg == 2) {
                U.col(col + 1) = c->mf->computeGroupUnitRemanenceResponse(g);
                x0[col + 1] = c->model->group(g).remanence_magnitude;
                lo[col + 1] = opt[4];
                hi[col + 1] = opt[5];
            } else if (ppg == 4) {
                const Vector3d e[3] = {Vector3d(1.0, 0.0, 0.0), Vector3d(0.0, 1.0, 0.0), Vector3d(0.0, 0.0, 1.0)};
                for (int k = 0; k < 3; ++k) {
                    U.col(col + 1 + k) = c->mf->computeGroupUnitResponseDirection(g, e[k]);
                    x0[col + 1 + k] = c->model->group(g).magnetization[k];
                    lo[col + 1 + k] = opt[6];
                    hi[col + 1 + k] = opt[7];
                }
            }
        }
        VectorXd d = solve(U, obsv, sdv, x0, lo, hi);
        for (int j = 0; j < m; ++j) magnetic[j] = d[j];
        for (int g = 0; g < nGroups; ++g) {
            const int col = ppg * g;
            c->model->group(g).susceptibility = d[col];
            if (ppg == 2) c->model->group(g).remanence_magnitude = d[col + 1];
            if (ppg == 4) c->model->group(g).magnetization = Vector3d(d[col + 1], d[col + 2], d[col + 3]);
        }
    }
    for (int g = 0; g < nGroups; ++g) density[g] = c->model->group(g).density;
}

void ref_jacobian_gz(void* h, const double* params, double* J) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    fromMat(c->gfwd->computeJacobian(toVec(static_cast<int>(c->gfwd->parameterCount()), params)), J);
}

void ref_jacobian_tmi(void* h, const double* params, double* J) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    fromMat(c->mfwd->computeJacobian(toVec(static_cast<int>(c->mfwd->parameterCount()), params)), J);
}

// Switches this model's objective to the GPU drop-in operators
// (gpu_dropin.hpp): opens liblitho_gpu.so at `lib_path`, creates a context on
// `device` and uploads the reference model's groups, meshes and DOF tables
// (built here from the reference's own dofMappings / globalDofIndex, as
// ref_dof_tables does), the inducing field and both station sets.  The
// control-point interpolation rows and shared-vertex groups are private in
// the reference; a model that has them passes them in (interp_* / sync_*,
// NULL otherwise).  Call after the model and the data are set.  Returns 0 on
// success, -1 if the library cannot be opened, else the lf_status.
int ref_use_gpu(void* h, const char* lib_path, int device, int precision, const int32_t* interp_off,
                const int32_t* interp_src, const double* interp_w, int n_sync, const int32_t* sync_off,
                const int32_t* sync_vertex) {
    auto* c = static_cast<RefCtx*>(h);
    auto s = std::make_shared<litho_dropin::GpuSession>();
    if (!s->api.open(lib_path)) return -1;
    lf_status st = s->api.create(&s->ctx, device);
    if (st != LF_OK) return st;
    auto& M = *c->model;
    const int G = M.groupCount();
    std::vector<double> rho(G), chi(G), rm(G), ri(G), rd(G), rv(3 * G);
    for (int g = 0; g < G; ++g) {
        const LithoGroup& gr = M.group(g);
        rho[g] = gr.density; chi[g] = gr.susceptibility; rm[g] = gr.remanence_magnitude;
        ri[g] = gr.remanence_inclination; rd[g] = gr.remanence_declination;
        rv[3 * g] = gr.magnetization.x(); rv[3 * g + 1] = gr.magnetization.y(); rv[3 * g + 2] = gr.magnetization.z();
    }
    std::vector<double> xyz;
    std::vector<int32_t> tri, grpTriOff(1, 0);
    int vbase = 0;
    for (int g = 0; g < G; ++g) {
        const SurfaceMesh* mesh = g < M.groupMeshCount() ? M.groupMesh(g) : nullptr;
        if (mesh) {
            for (uint32_t v = 0; v < mesh->vertexCount(); ++v) {
                const auto& p = mesh->vertex(v).position;
                xyz.push_back(p.x()); xyz.push_back(p.y()); xyz.push_back(p.z());
            }
            for (uint32_t t = 0; t < mesh->triangleCount(); ++t) {
                const auto& tr = mesh->triangle(t);
                tri.push_back(vbase + static_cast<int32_t>(tr.v0));
                tri.push_back(vbase + static_cast<int32_t>(tr.v1));
                tri.push_back(vbase + static_cast<int32_t>(tr.v2));
            }
            vbase += static_cast<int>(mesh->vertexCount());
        }
        grpTriOff.push_back(static_cast<int32_t>(tri.size() / 3));
    }
    const int np = static_cast<int>(M.totalDofCount());
    std::vector<int32_t> dofOff(np + 1), refVertex(3 * (size_t)vbase + 8);
    std::vector<uint8_t> refAxis(3 * (size_t)vbase + 8);
    std::vector<double> refScale(3 * (size_t)vbase + 8);
    ref_dof_tables(h, dofOff.data(), refVertex.data(), refAxis.data(), refScale.data());
    st = s->api.set_model_tables(s->ctx, G, rho.data(), chi.data(), rm.data(), ri.data(), rd.data(), rv.data(), vbase,
                                 xyz.data(), static_cast<int>(tri.size() / 3), tri.data(), grpTriOff.data(), np,
                                 dofOff.data(), refVertex.data(), refAxis.data(), refScale.data(), interp_off,
                                 interp_src, interp_w, n_sync, sync_off, sync_vertex);
    if (st == LF_OK) st = s->api.set_field(s->ctx, c->inc, c->dec, c->field, c->remMode);
    auto upload = [&](auto& data, auto fn, auto value, auto sigma) {
        std::vector<double> p, o, sd;
        for (const auto& d : data) {
            p.push_back(d.position.x()); p.push_back(d.position.y()); p.push_back(d.position.z());
            o.push_back(value(d)); sd.push_back(sigma(d));
        }
        return fn(s->ctx, static_cast<int>(data.size()), p.data(), o.data(), sd.data());
    };
    if (st == LF_OK)
        st = upload(c->grav, s->api.set_gravity_data, [](const GravityPoint& d) { return d.g_obs; },
                    [](const GravityPoint& d) { return d.g_std; });
    if (st == LF_OK)
        st = upload(c->mag, s->api.set_magnetic_data, [](const MagneticPoint& d) { return d.t_obs; },
                    [](const MagneticPoint& d) { return d.t_std; });
    if (st == LF_OK) st = s->api.set_precision(s->ctx, precision);
    if (st != LF_OK) return st;
    s->ng = static_cast<int>(c->grav.size());
    s->nm = static_cast<int>(c->mag.size());
    s->np = np;
    c->gpu = s;
    c->built = false;
    return 0;
}

// JointObjective::evaluateComponents (joint_objective.cpp:113-173):
// out5 = {gravityMisfit, magneticMisfit, regularization, constraint, total}.
void ref_objective(void* h, const double* params, double* out5) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    auto r = c->jobj->evaluateComponents(toVec(static_cast<int>(c->jobj->parameterCount()), params));
    out5[0] = r.gravityMisfit; out5[1] = r.magneticMisfit; out5[2] = r.regularization;
    out5[3] = r.constraintPenalty; out5[4] = r.total;
}

// JointObjective::gradient (joint_objective.cpp:42-111).
void ref_gradient(void* h, const double* params, double* grad) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    fromVec(c->jobj->gradient(toVec(static_cast<int>(c->jobj->parameterCount()), params)), grad);
}

// LBFGSBOptimizer::minimize (lbfgsb_optimizer.cpp:162-263) on the joint
// objective, with the reference's defaults unless overridden.
int ref_lbfgsb(void* h, const double* x0, const double* lo, const double* hi, int max_iter,
               double ftol, int history, double* x_out, double* f_out) {
    auto* c = static_cast<RefCtx*>(h);
    c->ensure();
    int np = static_cast<int>(c->jobj->parameterCount());
    LBFGSBOptimizer opt;
    opt.setMaxIterations(max_iter);
    opt.setTolerance(ftol);
    opt.setHistorySize(history);
    auto f = [c](const VectorXd& x) { return c->jobj->evaluate(x); };
    auto g = [c](const VectorXd& x) { return c->jobj->gradient(x); };
    auto res = opt.minimize(f, g, toVec(np, x0), toVec(np, lo), toVec(np, hi));
    fromVec(res.params, x_out);
    *f_out = res.finalValue;
    return res.iterations;
}

}  // extern "C"

// Geometry primitives and static facet functions of the reference
// (core/geometry.cpp:10-52, GravityForward::gravityFacet gravity_forward.cpp:153-158,
// MagneticForward::magneticFacet magnetic_forward.cpp:312-347) for golden vectors.
extern "C" {
double ref_solid_angle(const double* a, const double* b, const double* c, const double* o) {
    return solidAngle(Vector3d(a[0], a[1], a[2]), Vector3d(b[0], b[1], b[2]), Vector3d(c[0], c[1], c[2]),
                      Vector3d(o[0], o[1], o[2]));
}
double ref_line_integral_term(const double* a, const double* b, const double* o) {
    return lineIntegralTerm(Vector3d(a[0], a[1], a[2]), Vector3d(b[0], b[1], b[2]), Vector3d(o[0], o[1], o[2]));
}
double ref_gravity_facet(const double* o, const double* a, const double* b, const double* c) {
    return GravityForward::gravityFacet(Vector3d(o[0], o[1], o[2]), Vector3d(a[0], a[1], a[2]),
                                        Vector3d(b[0], b[1], b[2]), Vector3d(c[0], c[1], c[2]));
}
double ref_magnetic_facet(const double* o, const double* a, const double* b, const double* c, const double* m,
                          const double* f) {
    return MagneticForward::magneticFacet(Vector3d(o[0], o[1], o[2]), Vector3d(a[0], a[1], a[2]),
                                          Vector3d(b[0], b[1], b[2]), Vector3d(c[0], c[1], c[2]),
                                          Vector3d(m[0], m[1], m[2]), Vector3d(f[0], f[1], f[2]));
}
}  // extern "C"
