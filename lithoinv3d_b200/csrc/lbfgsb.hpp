// Projected L-BFGS ("L-BFGS-B" in the reference) on the host.  The device
// evaluates the objective and its gradient; only the O(np * m) two-loop
// recursion, projection and Armijo backtracking run here.
// Semantics: LBFGSBOptimizer, modules/litho-inversion/src/inversion/lbfgsb_optimizer.cpp:33-263.
#pragma once
#include <functional>
#include <string>
#include <vector>

namespace litho_b200 {

struct LbfgsbOptions {
    int maxIterations = 500;
    double tolerance = 1e-6;
    int historySize = 10;
    double armijoC1 = 1e-4;
    int lineSearchMaxIter = 50;
    bool disableLineSearch = false;
    double initialGamma = 0.0;  // > 0: H0 = gamma * I when the history is empty
    double targetValue = 0.0;   // > 0: stop once f <= targetValue (e.g. chi^2 = N)
};

struct LbfgsbResult {
    std::vector<double> params;
    double finalValue = 0.0;
    int iterations = 0;
    bool converged = false;
    std::string message;
};

using Objective = std::function<double(const std::vector<double>&)>;
using Gradient = std::function<std::vector<double>(const std::vector<double>&)>;

class LbfgsbOptimizer {
public:
    explicit LbfgsbOptimizer(const LbfgsbOptions& o) : opt_(o) {}
    LbfgsbResult minimize(const Objective& f, const Gradient& g, const std::vector<double>& x0,
                          const std::vector<double>& lb, const std::vector<double>& ub);

private:
    LbfgsbOptions opt_;
    std::vector<std::vector<double>> s_, y_;
    std::vector<double> rho_;
    std::vector<double> x_, g_, lb_, ub_;
    std::vector<double> direction(const std::vector<double>& g) const;
    double lineSearch(const Objective& f, const Gradient& g, const std::vector<double>& d,
                      std::vector<double>& xNew, std::vector<double>& gNew);
    void project(std::vector<double>& x) const;
};

}  // namespace litho_b200
