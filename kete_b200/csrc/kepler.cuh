// kepler.cuh -- universal-variable two-body propagation on the device.
//
// Restates kete_core/propagation/kepler.rs:119-297 (g_1, g_2, solve_kepler_universal,
// analytic_2_body) and kete_core/fitting/newton.rs:18-65 (newton_raphson).  The
// reference's recursive interval halving (depth <= 10) becomes an explicit stack of
// pending half-intervals, processed in the same order.
#pragma once
#include "common.cuh"

namespace kb {

constexpr double PARABOLIC_BETA = 1e-10;

__device__ __forceinline__ double g_1(double s, double beta) {
    if (fabs(beta) < PARABOLIC_BETA) return s;
    const double bs = sqrt(fabs(beta));
    if (beta >= 0.0) return sin(bs * s) / bs;
    return sinh(bs * s) / bs;
}

__device__ __forceinline__ double g_2(double s, double beta) {
    if (fabs(beta) < PARABOLIC_BETA) return powi<2>(s) / 2.0;
    const double bs = sqrt(fabs(beta)) * s;
    if (beta >= 0.0) {
        const double sn = sin(bs / 2.0);
        return 2.0 * (sn * sn) / beta;
    }
    return (1.0 - cosh(bs)) / beta;
}

// f(x) and f'(x) of the universal Kepler equation (kepler.rs:189-199, 217-227)
struct KepEq {
    double r0, rv0, beta, b_sqrt, dt;
    bool hyperbolic;
    double mu;  // GM of the central body (GMS in kete)
    __device__ __forceinline__ double f(double x) const {
        double g1, g2;
        if (!hyperbolic) {
            g1 = sin(b_sqrt * x) / b_sqrt;
            const double sn = sin(b_sqrt * x / 2.0);
            g2 = 2.0 * (sn * sn) / beta;
        } else {
            g1 = sinh(b_sqrt * x) / b_sqrt;
            g2 = (1.0 - cosh(b_sqrt * x)) / beta;
        }
        const double g3 = (x - g1) / beta;
        return r0 * g1 + rv0 * g2 + mu * g3 - dt;
    }
    __device__ __forceinline__ double d(double x) const {
        double g2d, g1d;
        if (!hyperbolic) {
            sincos(b_sqrt * x, &g2d, &g1d);
        } else {
            g2d = sinh(b_sqrt * x);
            g1d = cosh(b_sqrt * x);
        }
        const double g3d = (1.0 - g1d) / beta;
        return r0 * g1d + rv0 * g2d + mu * g3d;
    }
};

// newton_raphson (fitting/newton.rs:18-65): two damped half steps per iteration,
// the second reusing f unless |f'| < 1e-3.  At most 100 iterations.
__device__ __forceinline__ int newton(const KepEq& q, double start, double atol, double& out) {
    double x = start;
    if (fabs(q.d(x)) < 1e-12) x += 0.1;
    for (int it = 0; it < 100; ++it) {
        double f_eval = q.f(x);
        if (fabs(f_eval) < atol) {
            out = x;
            return ST_OK;
        }
        double d_eval = q.d(x);
        if (fabs(d_eval) < 1e-12) return ST_CONVERGENCE;
        if (!isfinite(d_eval) || !isfinite(f_eval)) return ST_CONVERGENCE;
        x -= 0.5 * f_eval / d_eval;
        d_eval = q.d(x);
        if (fabs(d_eval) < 1e-3) f_eval = q.f(x);
        x -= 0.5 * f_eval / d_eval;
    }
    return ST_CONVERGENCE;
}

__device__ __forceinline__ int solve_kepler_universal(double dt, double r0, double v0, double rv0,
                                                      double& s_out, double& beta_out,
                                                      double mu = GMS) {
    const double beta = 2.0 * mu / r0 - powi<2>(v0);
    const double b_sqrt = sqrt(fabs(beta));
    double res = 0.0;
    int rc;
    if (beta >= PARABOLIC_BETA) {
        const double period = mu * powi<-3>(b_sqrt);
        const double dtm = fmod(dt, period * TAU);
        KepEq q{r0, rv0, beta, b_sqrt, dtm, false, mu};
        const double guess = (1.0 / b_sqrt) * dtm / period;
        rc = newton(q, guess, 1e-11, res);
    } else if (fabs(beta) < PARABOLIC_BETA) {
        const double a0 = -6.0 * dt / mu;
        const double a1 = 6.0 * r0 / mu;
        const double a2 = 3.0 * rv0 / mu;
        const double p = (3.0 * a1 - powi<2>(a2)) / 3.0;
        const double qq = (9.0 * a1 * a2 - 27.0 * a0 - 2.0 * powi<3>(a2)) / 27.0;
        const double w = pow(qq / 2.0 + sqrt(powi<2>(qq) / 4.0 + powi<3>(p) / 27.0), 1.0 / 3.0);
        res = w - p / (3.0 * w) - a2 / 3.0;
        rc = ST_OK;
    } else {
        KepEq q{r0, rv0, beta, b_sqrt, dt, true, mu};
        // kete's starting point uses its GMS_SQRT literal (kepler.rs:228)
        const double mu_sqrt = mu == GMS ? GMS_SQRT : sqrt(mu);
        rc = newton(q, mu_sqrt * fabs(beta) * dt, 1e-11, res);
    }
    if (rc != ST_OK) return ST_CONVERGENCE;
    s_out = res;
    beta_out = beta;
    return ST_OK;
}

// The f and g update of one closed-form step from the solved anomaly s (kepler.rs:270-288).
__device__ __forceinline__ void two_body_apply(double s, double beta, double r0, double rv0,
                                               double p[3], double v[3], double mu = GMS) {
    const double g1 = g_1(s, beta), g2 = g_2(s, beta);
    const double f = 1.0 - mu / r0 * g2;
    const double g = r0 * g1 + rv0 * g2;
    double np[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) np[i] = p[i] * f + v[i] * g;
    const double nr0 = norm3(np[0], np[1], np[2]);
    const double f_dot = -mu / (nr0 * r0) * g1;
    const double g_dot = 1.0 - (mu / nr0) * g2;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        v[i] = p[i] * f_dot + v[i] * g_dot;
        p[i] = np[i];
    }
}

// One closed-form step; returns ST_CONVERGENCE when the solver fails.
__device__ __forceinline__ int two_body_leaf(double time, double p[3], double v[3]) {
    const double r0 = norm3(p[0], p[1], p[2]);
    const double v0 = norm3(v[0], v[1], v[2]);
    const double rv0 = p[0] * v[0] + p[1] * v[1] + p[2] * v[2];
    double s, beta;
    if (solve_kepler_universal(time, r0, v0, rv0, s, beta) != ST_OK) return ST_CONVERGENCE;
    two_body_apply(s, beta, r0, rv0, p, v);
    return ST_OK;
}

// analytic_2_body (kepler.rs:254-297), in place.  Stack entries hold the remaining
// half-intervals and the depth value their recursive call would receive.
static __device__ __noinline__ int analytic_2_body(double time, double p[3], double v[3]) {
    double st_dt[12];
    int st_depth[12];
    int top = 0;
    st_dt[0] = time;
    st_depth[0] = 0;
    top = 1;
    int guard = 0;
    while (top > 0) {
        if (++guard > 4096) return ST_TIMEOUT;
        --top;
        const double dt = st_dt[top];
        int depth = st_depth[top];
        if (depth >= 10) return ST_CONVERGENCE;
        depth += 1;
        if (fabs(dt) < 1e-10) continue;
        if (isnan(p[0] * v[0] + p[1] * v[1] + p[2] * v[2]) ||
            isinf(p[0] * v[0] + p[1] * v[1] + p[2] * v[2]))
            return ST_CONVERGENCE;
        if (two_body_leaf(dt, p, v) == ST_OK) continue;
        if (top + 2 > 12) return ST_CONVERGENCE;
        // second half pushed first so the first half runs first
        st_dt[top] = dt * 0.5;
        st_depth[top] = depth;
        st_dt[top + 1] = 0.5 * dt;
        st_depth[top + 1] = depth;
        top += 2;
    }
    return ST_OK;
}

}  // namespace kb
