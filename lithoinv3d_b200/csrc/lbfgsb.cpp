#include "lbfgsb.hpp"

#include <algorithm>
#include <cmath>
#include <limits>

namespace litho_b200 {

namespace {
double dotv(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}
}  // namespace

// LBFGSBOptimizer::project / projectInPlace, lbfgsb_optimizer.cpp:13-31.
void LbfgsbOptimizer::project(std::vector<double>& x) const {
    for (size_t i = 0; i < x.size(); ++i) x[i] = std::max(lb_[i], std::min(ub_[i], x[i]));
}

// Two-loop recursion, lbfgsb_optimizer.cpp:33-72.  With an empty history the
// reference takes steepest descent; initialGamma > 0 replaces that first step
// by -gamma * g (the warm-start hook; the reference has no such setter).
std::vector<double> LbfgsbOptimizer::direction(const std::vector<double>& g) const {
    std::vector<double> r(g.size());
    if (s_.empty()) {
        double gam = opt_.initialGamma > 0.0 ? opt_.initialGamma : 1.0;
        for (size_t i = 0; i < g.size(); ++i) r[i] = -gam * g[i];
        return r;
    }
    const auto& sl = s_.back();
    const auto& yl = y_.back();
    double sy = dotv(sl, yl), yy = dotv(yl, yl);
    double gamma = (yy > std::numeric_limits<double>::epsilon()) ? (sy / yy) : 1.0;
    int m = static_cast<int>(s_.size());
    std::vector<double> alpha(m);
    std::vector<double> q = g;
    for (int i = m - 1; i >= 0; --i) {
        alpha[i] = rho_[i] * dotv(s_[i], q);
        for (size_t k = 0; k < q.size(); ++k) q[k] -= alpha[i] * y_[i][k];
    }
    for (size_t k = 0; k < q.size(); ++k) r[k] = gamma * q[k];
    for (int i = 0; i < m; ++i) {
        double beta = rho_[i] * dotv(y_[i], r);
        for (size_t k = 0; k < r.size(); ++k) r[k] += s_[i][k] * (alpha[i] - beta);
    }
    for (auto& v : r) v = -v;
    return r;
}

// Projected Armijo backtracking, lbfgsb_optimizer.cpp:85-144.
double LbfgsbOptimizer::lineSearch(const Objective& f, const Gradient& grad, const std::vector<double>& d,
                                   std::vector<double>& xNew, std::vector<double>& gNew) {
    size_t n = x_.size();
    if (opt_.disableLineSearch) {
        xNew.resize(n);
        for (size_t i = 0; i < n; ++i) xNew[i] = x_[i] + d[i];
        project(xNew);
        gNew = grad(xNew);
        return 1.0;
    }
    double alpha = 1.0;
    double f0 = f(x_);
    double gd = dotv(g_, d);
    if (gd >= 0.0) {
        xNew = x_;
        gNew = g_;
        return 0.0;
    }
    const double minAlpha = 1e-16;
    std::vector<double> xTry(n);
    for (int it = 0; it < opt_.lineSearchMaxIter; ++it) {
        if (alpha < minAlpha) break;
        for (size_t i = 0; i < n; ++i) xTry[i] = x_[i] + alpha * d[i];
        project(xTry);
        double fTry = f(xTry);
        double dec = 0.0;
        for (size_t i = 0; i < n; ++i) dec += g_[i] * (xTry[i] - x_[i]);
        if (dec >= 0.0) {
            alpha *= 0.5;
            continue;
        }
        if (fTry <= f0 + opt_.armijoC1 * dec) {
            xNew = xTry;
            gNew = grad(xNew);
            return alpha;
        }
        alpha *= 0.5;
    }
    alpha = minAlpha;
    xNew.resize(n);
    for (size_t i = 0; i < n; ++i) xNew[i] = x_[i] + alpha * d[i];
    project(xNew);
    gNew = grad(xNew);
    return alpha;
}

// LBFGSBOptimizer::minimize, lbfgsb_optimizer.cpp:162-263.
LbfgsbResult LbfgsbOptimizer::minimize(const Objective& f, const Gradient& grad, const std::vector<double>& x0,
                                       const std::vector<double>& lb, const std::vector<double>& ub) {
    LbfgsbResult res;
    lb_ = lb;
    ub_ = ub;
    x_ = x0;
    project(x_);
    g_ = grad(x_);
    s_.clear();
    y_.clear();
    rho_.clear();
    double pg0 = 0.0;
    int stall = 0, iters = 0;
    size_t n = x_.size();
    for (int k = 0; k < opt_.maxIterations; ++k) {
        iters = k + 1;
        double pg = 0.0;
        for (size_t i = 0; i < n; ++i) {
            double p = std::max(lb_[i], std::min(ub_[i], x_[i] - g_[i]));
            pg += (x_[i] - p) * (x_[i] - p);
        }
        pg = std::sqrt(pg);
        if (k == 0) pg0 = pg;
        if (opt_.targetValue > 0.0 && f(x_) <= opt_.targetValue) {
            res.converged = true;
            res.message = "Reached the target objective value";
            break;
        }
        if (k > 0 && pg < opt_.tolerance * std::max(1.0, pg0)) {
            res.converged = true;
            res.message = "Converged: projected gradient below tolerance";
            break;
        }
        std::vector<double> d = direction(g_);
        std::vector<double> xNew, gNew;
        double alpha = lineSearch(f, grad, d, xNew, gNew);
        if (alpha == 0.0) {
            res.converged = true;
            res.message = "Converged: no step taken";
            break;
        }
        if (alpha < 1e-8) {
            if (++stall >= 3) {
                res.converged = true;
                res.message = "Converged: line search stalled";
                break;
            }
        } else {
            stall = 0;
        }
        std::vector<double> s(n), y(n);
        for (size_t i = 0; i < n; ++i) { s[i] = xNew[i] - x_[i]; y[i] = gNew[i] - g_[i]; }
        double sy = dotv(s, y);
        if (sy > 1e-16) {
            if (static_cast<int>(s_.size()) >= opt_.historySize) {
                s_.erase(s_.begin());
                y_.erase(y_.begin());
                rho_.erase(rho_.begin());
            }
            s_.push_back(s);
            y_.push_back(y);
            rho_.push_back(1.0 / dotv(y, s));
        }
        x_ = xNew;
        g_ = gNew;
    }
    res.params = x_;
    res.finalValue = f(x_);
    res.iterations = iters;
    if (!res.converged && iters >= opt_.maxIterations) res.message = "Maximum iterations reached";
    return res;
}

}  // namespace litho_b200
