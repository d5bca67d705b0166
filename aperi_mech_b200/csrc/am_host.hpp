// am_host.hpp -- host-side mirror of the aperi-mech objects that feed the hot path:
// material property completion (Materials/Base.h), boundary-condition time
// functions (src/BoundaryCondition.cpp + MathUtils.h interpolations) and the
// direct time stepper (include/TimeStepper.h). Plain C++; no device code.
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace am {
namespace host {

// LinearElasticProperties::CompleteProperties (Materials/Base.h:47-129): exactly two
// of {E, nu, mu, lambda, K} given (NaN = missing); fills the rest and checks bounds.
struct LinearElasticProperties {
    double youngs_modulus = std::numeric_limits<double>::quiet_NaN();
    double poisson_ratio = std::numeric_limits<double>::quiet_NaN();
    double shear_modulus = std::numeric_limits<double>::quiet_NaN();
    double lambda = std::numeric_limits<double>::quiet_NaN();
    double bulk_modulus = std::numeric_limits<double>::quiet_NaN();

    void CompleteProperties() {
        double& E = youngs_modulus;
        double& nu = poisson_ratio;
        double& G = shear_modulus;
        double& L = lambda;
        double& K = bulk_modulus;
        auto has = [](double x) { return !std::isnan(x); };
        const int n = has(E) + has(nu) + has(G) + has(L) + has(K);
        if (n != 2) throw std::runtime_error("Exactly two properties must be defined. Defined: " + std::to_string(n));
        if (has(K) && has(E)) {
            nu = (3 * K - E) / (6 * K);
            G = E / (2 * (1 + nu));
            L = (E * nu) / ((1 + nu) * (1 - 2 * nu));
        } else if (has(K) && has(L)) {
            G = (3 * (K - L)) / 2;
            nu = L / (2 * (L + G));
            E = 2 * G * (1 + nu);
        } else if (has(K) && has(G)) {
            L = K - (2.0 / 3.0) * G;
            nu = L / (2 * (L + G));
            E = 2 * G * (1 + nu);
        } else if (has(K) && has(nu)) {
            E = 3 * K * (1 - 2 * nu);
            G = E / (2 * (1 + nu));
            L = (E * nu) / ((1 + nu) * (1 - 2 * nu));
        } else if (has(E) && has(L)) {
            const double a = 2 * L, b = L + E, c = -L;
            nu = (-b + std::sqrt(b * b - 4 * a * c)) / (2 * a);
            G = E / (2 * (1 + nu));
            K = L + (2.0 / 3.0) * G;
        } else if (has(E) && has(G)) {
            nu = (E / (2 * G)) - 1;
            L = (E * nu) / ((1 + nu) * (1 - 2 * nu));
            K = L + (2.0 / 3.0) * G;
        } else if (has(E) && has(nu)) {
            G = E / (2 * (1 + nu));
            L = (E * nu) / ((1 + nu) * (1 - 2 * nu));
            K = E / (3 * (1 - 2 * nu));
        } else if (has(L) && has(G)) {
            K = L + (2.0 / 3.0) * G;
            nu = L / (2 * (L + G));
            E = 2 * G * (1 + nu);
        } else if (has(L) && has(nu)) {
            E = (L * (1 + nu) * (1 - 2 * nu)) / nu;
            G = E / (2 * (1 + nu));
            K = L + (2.0 / 3.0) * G;
        } else if (has(G) && has(nu)) {
            E = 2 * G * (1 + nu);
            L = (2 * G * nu) / (1 - 2 * nu);
            K = (2 * G * (1 + nu)) / (3 * (1 - 2 * nu));
        } else {
            throw std::runtime_error("Unsupported property pair combination");
        }
        if (nu < -1.0 || nu >= 0.5)
            throw std::runtime_error("Poisson's ratio violation: " + std::to_string(nu) + " must be in [-1, 0.5)");
        if (E <= 0.0) throw std::runtime_error("Young's modulus must be positive: " + std::to_string(E));
        if (G <= 0.0) throw std::runtime_error("Shear modulus must be positive: " + std::to_string(G));
        if (K <= 0.0) throw std::runtime_error("Bulk modulus must be positive: " + std::to_string(K));
        if (L <= -(2.0 / 3.0) * G) throw std::runtime_error("Lame's parameter violation: lambda must be > -2G/3");
    }
};

// ---- interpolations (MathUtils.h) ----
inline double ConstantInterpolation(double x, const std::vector<double>& ab, const std::vector<double>& ord) {
    const size_t n = ab.size();
    if (n == 1) return ord[0];
    if (x < ab[0]) return 0.0;
    if (x > ab[n - 1]) return ord[n - 1];
    for (size_t i = 0; i + 1 < n; ++i)
        if (x >= ab[i] && x <= ab[i + 1]) return ord[i];
    throw std::runtime_error("Constant interpolation failed.");
}
inline double LinearInterpolation(double x, const std::vector<double>& ab, const std::vector<double>& ord) {
    const size_t n = ab.size();
    if (n == 1) return ord[0];
    if (x < ab[0]) return ord[0];
    if (x > ab[n - 1]) return ord[n - 1];
    for (size_t i = 0; i + 1 < n; ++i)
        if (x >= ab[i] && x <= ab[i + 1]) {
            const double slope = (ord[i + 1] - ord[i]) / (ab[i + 1] - ab[i]);
            return ord[i] + slope * (x - ab[i]);
        }
    throw std::runtime_error("Linear interpolation failed.");
}
inline double SmoothStep(double x, const std::vector<double>& ab, const std::vector<double>& ord) {
    const size_t n = ab.size();
    if (n == 1 || x < ab[0]) return ord[0];
    if (x > ab[n - 1]) return ord[n - 1];
    for (size_t i = 0; i + 1 < n; ++i)
        if (x >= ab[i] && x <= ab[i + 1]) {
            const double t = (x - ab[i]) / (ab[i + 1] - ab[i]);
            return ord[i] + (ord[i + 1] - ord[i]) * t * t * t * (10.0 - 15.0 * t + 6.0 * t * t);
        }
    throw std::runtime_error("Smooth step interpolation failed.");
}
inline double SmoothStepD1(double x, const std::vector<double>& ab, const std::vector<double>& ord) {
    const size_t n = ab.size();
    if (n == 1 || x < ab[0] || x > ab[n - 1]) return 0.0;
    for (size_t i = 0; i + 1 < n; ++i)
        if (x >= ab[i] && x <= ab[i + 1]) {
            const double t = (x - ab[i]) / (ab[i + 1] - ab[i]);
            return (ord[i + 1] - ord[i]) * (30.0 * t * t - 60.0 * t * t * t + 30.0 * t * t * t * t) / (ab[i + 1] - ab[i]);
        }
    throw std::runtime_error("Smooth step interpolation derivative failed.");
}
inline double SmoothStepD2(double x, const std::vector<double>& ab, const std::vector<double>& ord) {
    const size_t n = ab.size();
    if (n == 1 || x < ab[0] || x > ab[n - 1]) return 0.0;
    for (size_t i = 0; i + 1 < n; ++i)
        if (x >= ab[i] && x <= ab[i + 1]) {
            const double t = (x - ab[i]) / (ab[i + 1] - ab[i]);
            return (ord[i + 1] - ord[i]) * (60.0 * t - 180.0 * t * t + 120.0 * t * t * t) / ((ab[i + 1] - ab[i]) * (ab[i + 1] - ab[i]));
        }
    throw std::runtime_error("Smooth step interpolation second derivative failed.");
}

// BoundaryCondition (src/BoundaryCondition.cpp): values per component, the velocity and
// acceleration time functions derived from a displacement or velocity time function,
// and the active time range.
struct BoundaryCondition {
    std::vector<int32_t> nodes;
    int32_t component_mask = 0;
    int32_t kind = 0;           // 0 displacement, 1 velocity
    int32_t time_function = 0;  // 0 ramp, 1 smooth step
    double values[3] = {0, 0, 0};
    std::vector<double> abscissa, ordinate, ordinate_derivative;
    double active_start = 0.0, active_end = std::numeric_limits<double>::max();

    void Finish() {
        if (abscissa.size() != ordinate.size()) throw std::runtime_error("Abscissa and ordinate vectors must be the same size.");
        if (abscissa.empty()) throw std::runtime_error("Abscissa and ordinate vectors must have at least one value.");
        ordinate_derivative.assign(ordinate.size(), 0.0);
        for (size_t i = 0; i + 1 < ordinate.size(); ++i)
            ordinate_derivative[i] = (ordinate[i + 1] - ordinate[i]) / (abscissa[i + 1] - abscissa[i]);
    }
    bool Active(double t) const { return !(t < active_start || t > active_end); }
    double VelocityScale(double t) const {
        if (time_function == 0)
            return kind == 0 ? ConstantInterpolation(t, abscissa, ordinate_derivative) : LinearInterpolation(t, abscissa, ordinate);
        return kind == 0 ? SmoothStepD1(t, abscissa, ordinate) : SmoothStep(t, abscissa, ordinate);
    }
    double AccelerationScale(double t) const {
        if (time_function == 0) return kind == 0 ? 0.0 : ConstantInterpolation(t, abscissa, ordinate_derivative);
        return kind == 0 ? SmoothStepD2(t, abscissa, ordinate) : SmoothStepD1(t, abscissa, ordinate);
    }
};

// DirectTimeStepper::GetTimeIncrement (include/TimeStepper.h:97-128) under the
// ExplicitSolver::Solve loop `while (!AtEnd(time)) { ...; time += dt; }`.
inline std::vector<double> DirectTimeSchedule(double dt, double t_end, int64_t max_steps) {
    std::vector<double> dts;
    double time = 0.0;
    while (!(time >= t_end) && static_cast<int64_t>(dts.size()) < max_steps) {
        double d;
        if (time + dt <= t_end)
            d = dt;
        else if (time > t_end)
            d = 0.0;
        else
            d = t_end - time;
        dts.push_back(d);
        time += d;
    }
    return dts;
}

}  // namespace host
}  // namespace am
