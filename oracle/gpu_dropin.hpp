// gpu_dropin.hpp -- TEST INFRASTRUCTURE ONLY (compiled into oracle/_ref by
// oracle/Makefile, together with the reference's own sources).
//
// The drop-in a maintainer of the reference would add: GPU operators behind
// the reference's own ForwardModel interface
// (modules/litho-forward/include/litho_invert/forward/forward_model.h:6-33),
// so that the reference's ObjectiveFunction (objective.cpp:22-105),
// JointObjective (joint_objective.cpp:42-173) and LBFGSBOptimizer
// (lbfgsb_optimizer.cpp:162-263) run unchanged on top of liblitho_gpu.so.
//
//  * GpuGravityForward : ForwardModel replaces GravityForward
//    (gravity_forward.h:10-11): compute = lf_forward (gz), computeJacobian =
//    lf_jacobian(LF_GRAVITY) (the reference's CP-only DOF gather, analytic
//    derivatives instead of its per-facet forward differences).
//  * GpuMagneticForward : MagneticForward replaces MagneticForward
//    (magnetic_forward.h:10-12).  JointObjective holds a
//    shared_ptr<MagneticForward>, so the GPU operator derives from the
//    concrete class and overrides compute / computeJacobian.
//
// The library is opened with dlopen when a caller asks for the drop-in, so a
// process that never does (the CPU baseline) never loads it.  The reference
// model's positions are not updated by these operators (the context keeps the
// positions on the device, as the reference keeps them in its mutable model);
// the reference's regularisations that read mesh positions are not combined
// with them here.
#pragma once
#include <dlfcn.h>

#include <litho_invert/forward/forward_model.h>
#include <litho_invert/forward/magnetic_forward.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../include/litho_gpu.h"

namespace litho_dropin {

using namespace litho_invert;

// Entry points of liblitho_gpu.so used by the drop-in.
struct GpuApi {
    void* handle = nullptr;
    decltype(&lf_create) create = nullptr;
    decltype(&lf_destroy) destroy = nullptr;
    decltype(&lf_last_error) last_error = nullptr;
    decltype(&lf_set_model_tables) set_model_tables = nullptr;
    decltype(&lf_set_field) set_field = nullptr;
    decltype(&lf_set_gravity_data) set_gravity_data = nullptr;
    decltype(&lf_set_magnetic_data) set_magnetic_data = nullptr;
    decltype(&lf_set_precision) set_precision = nullptr;
    decltype(&lf_forward) forward = nullptr;
    decltype(&lf_jacobian) jacobian = nullptr;

    bool open(const char* path) {
        handle = dlopen(path, RTLD_NOW | RTLD_LOCAL);
        if (!handle) return false;
        auto get = [this](auto& fn, const char* name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(handle, name));
            return fn != nullptr;
        };
        return get(create, "lf_create") && get(destroy, "lf_destroy") && get(last_error, "lf_last_error") &&
               get(set_model_tables, "lf_set_model_tables") && get(set_field, "lf_set_field") &&
               get(set_gravity_data, "lf_set_gravity_data") && get(set_magnetic_data, "lf_set_magnetic_data") &&
               get(set_precision, "lf_set_precision") && get(forward, "lf_forward") && get(jacobian, "lf_jacobian");
    }
};

// One device context shared by the two operators (as the reference's
// forwards share one LithologyModel).
struct GpuSession {
    GpuApi api;
    lf_ctx* ctx = nullptr;
    int ng = 0, nm = 0, np = 0;
    ~GpuSession() {
        if (ctx && api.destroy) api.destroy(ctx);
    }
    void check(lf_status s) const {
        if (s != LF_OK) throw std::runtime_error(std::string("liblitho_gpu: ") + api.last_error(ctx));
    }
};

inline VectorXd to_vector(const std::vector<double>& v) {
    VectorXd out(static_cast<Eigen::Index>(v.size()));
    for (size_t i = 0; i < v.size(); ++i) out[static_cast<Eigen::Index>(i)] = v[i];
    return out;
}

inline std::vector<double> to_std(const VectorXd& v) {
    std::vector<double> out(static_cast<size_t>(v.size()));
    for (Eigen::Index i = 0; i < v.size(); ++i) out[static_cast<size_t>(i)] = v[i];
    return out;
}

inline MatrixXd rows_to_matrix(const std::vector<double>& rm, int rows, int cols) {
    MatrixXd J(rows, cols);
    for (int i = 0; i < rows; ++i)
        for (int j = 0; j < cols; ++j) J(i, j) = rm[(size_t)i * cols + j];
    return J;
}

class GpuGravityForward : public ForwardModel {
public:
    explicit GpuGravityForward(std::shared_ptr<GpuSession> s) : s_(std::move(s)) {}
    VectorXd compute(const VectorXd& params) override {
        std::vector<double> p = to_std(params), gz(s_->ng);
        s_->check(s_->api.forward(s_->ctx, p.data(), gz.data(), nullptr));
        return to_vector(gz);
    }
    MatrixXd computeJacobian(const VectorXd& params) override {
        std::vector<double> p = to_std(params), J((size_t)s_->ng * s_->np);
        s_->check(s_->api.jacobian(s_->ctx, p.data(), LF_GRAVITY, J.data()));
        return rows_to_matrix(J, s_->ng, s_->np);
    }
    size_t dataCount() const override { return static_cast<size_t>(s_->ng); }
    size_t parameterCount() const override { return static_cast<size_t>(s_->np); }

private:
    std::shared_ptr<GpuSession> s_;
};

class GpuMagneticForward : public MagneticForward {
public:
    GpuMagneticForward(std::shared_ptr<GpuSession> s, std::shared_ptr<LithologyModel> model,
                       const MagneticData& data, double inc, double dec, double field)
        : MagneticForward(std::move(model), data, inc, dec, field), s_(std::move(s)) {}
    VectorXd compute(const VectorXd& params) override {
        std::vector<double> p = to_std(params), tmi(s_->nm);
        s_->check(s_->api.forward(s_->ctx, p.data(), nullptr, tmi.data()));
        return to_vector(tmi);
    }
    MatrixXd computeJacobian(const VectorXd& params) override {
        std::vector<double> p = to_std(params), J((size_t)s_->nm * s_->np);
        s_->check(s_->api.jacobian(s_->ctx, p.data(), LF_MAGNETIC, J.data()));
        return rows_to_matrix(J, s_->nm, s_->np);
    }

private:
    std::shared_ptr<GpuSession> s_;
};

}  // namespace litho_dropin
