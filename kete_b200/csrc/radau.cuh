// radau.cuh -- Gauss-Radau 15th-order class-II integrator, one object per thread.
//
// Restates RadauIntegrator::integrate / step (kete_core/propagation/radau.rs:160-346):
// up to 10 predictor-corrector iterations over the 7 Gauss-Radau nodes, convergence when
// max|b6_new - b6_old| / (|a| + 1e-6) < 1e-14, next step h * (1e-6 max(|a|+1e-6) /
// max|b6|)^(1/7) clamped to [0.25, 4]; failures shrink h by 0.7 (at most 10 in a row);
// |h| >= 0.005 days.
//
// The corrector's starting b for a new step: the reference carries b over unscaled.  Here
// the previous step's acceleration polynomial is re-expanded about its end for the new
// step's length (predict_b_row, Everhart's predictor).  The corrector converges to the
// same fixed point (to its 1e-14 test; in practice to the same bits) in about a quarter
// fewer iterations.  After a failed attempt b is kept as it is, as in the reference.
//
// Divisions by node spacings are multiplications by reciprocals tabulated on the host.
#pragma once
#include "common.cuh"
#include "forces.cuh"

namespace kb {

struct RadauCounters {
    int32_t steps = 0;       // accepted steps
    int32_t iterations = 0;  // corrector iterations (each = 7 force evaluations)
    int32_t exact = 0;       // exact evaluations (1 initial + 1 per accepted step)
};

// a(tau) = a0 + sum_k b_k tau^(k+1) over the step just taken, re-expanded about its end for
// a step q times as long: b'_m = q^(m+1) sum_{k>=m} C(k+1, m+1) b_k (one component).
__device__ __forceinline__ void predict_b_row(double* row, double q) {
    double b[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) b[k] = row[k];
    double qp = q;
#pragma unroll
    for (int m = 0; m < 7; ++m) {
        double s2 = 0.0;
#pragma unroll
        for (int k = m; k < 7; ++k) s2 += c_tab.shift_c[m][k] * b[k];
        row[m] = qp * s2;
        qp *= q;
    }
}

// The transpose: the adjoint of the previous step's b from the adjoint of the predicted b.
__device__ __forceinline__ void predict_b_row_transposed(double* row, double q) {
    double l[7], qp[7];
    double p = q;
#pragma unroll
    for (int m = 0; m < 7; ++m) {
        l[m] = row[m];
        qp[m] = p;
        p *= q;
    }
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        double s2 = 0.0;
#pragma unroll
        for (int m = 0; m <= k; ++m) s2 += c_tab.shift_c[m][k] * qp[m] * l[m];
        row[k] = s2;
    }
}

struct RadauObj {
    double t;
    double x[3], v[3], a[3];
    double b[3][7];
};

template <class Force>
__device__ __forceinline__ int radau_step(RadauObj& s, Force& F, double h, double& next_h,
                                          RadauCounters& cnt) {
    double g[3][7];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 7; ++k) g[c][k] = 0.0;
    double ev[3] = {s.a[0], s.a[1], s.a[2]};
    const double h2 = h * h;
    for (int iter = 0; iter < 10; ++iter) {
        cnt.iterations++;
        const double b6_old[3] = {s.b[0][6], s.b[1][6], s.b[2][6]};
#pragma unroll 1
        for (int j = 1; j < 8; ++j) {
            const double f = c_tab.spacing[j];
            double xs[3], vs[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double bw = 0.0, bu = 0.0;
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    bw += c_tab.w_pow[j][k] * s.b[c][k];
                    bu += c_tab.u_pow[j][k] * s.b[c][k];
                }
                xs[c] = s.x[c] + f * s.v[c] * h + c_tab.frac2[j] * h2 * (s.a[c] / 2.0 + bw);
                vs[c] = s.v[c] + f * h * (s.a[c] + bu);
            }
            const int rc = F.eval(false, s.t + f * h, xs, vs, ev);
            if (rc != ST_OK) return rc;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double gk = (ev[c] - s.a[c]) * c_tab.inv_frac[j];
#pragma unroll
                for (int z = 1; z < 7; ++z)
                    if (z < j) gk = (gk - g[c][z - 1]) * c_tab.inv_diff[j][z];
#pragma unroll
                for (int k = 0; k < 7; ++k)
                    if (k == j - 1) g[c][k] = gk;
            }
        }
        // b = g * C (radau.rs:313); C is lower triangular
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int jj = 0; jj < 7; ++jj) {
                double acc = c_tab.c[jj][jj] * g[c][jj];
#pragma unroll
                for (int k = jj + 1; k < 7; ++k) acc += c_tab.c[k][jj] * g[c][k];
                s.b[c][jj] = acc;
            }
        double fem[3], ratio[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            fem[c] = fabs(ev[c]) + 1e-6;
            ratio[c] = fabs(s.b[c][6] - b6_old[c]) / fem[c];
        }
        if (fmax(fmax(ratio[0], ratio[1]), ratio[2]) < 1e-14) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double dw = 0.0, du = 0.0;
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    dw += s.b[c][k] * c_tab.w[k];
                    du += s.b[c][k] * c_tab.u[k];
                }
                s.x[c] += s.v[c] * h + h2 * (s.a[c] * 0.5 + dw);
                s.v[c] += h * (s.a[c] + du);
            }
            s.t += h;
            cnt.exact++;
            const int rc = F.eval(true, s.t, s.x, s.v, s.a);
            if (rc != ST_OK) return rc;
            cnt.steps++;
            const double mb6 = fmax(fmax(fabs(s.b[0][6]), fabs(s.b[1][6])), fabs(s.b[2][6]));
            const double r = pow(1e-6 * fmax(fmax(fem[0], fem[1]), fem[2]) / mb6, 1.0 / 7.0);
            next_h = h * clampd(r, 0.25, 4.0);
            return ST_OK;
        }
    }
    return ST_CONVERGENCE;
}

// Integrate s from s.t to tf.  max_loops bounds the step loop (ST_TIMEOUT when hit).
template <class Force>
__device__ int radau_integrate(RadauObj& s, double tf, Force& F, RadauCounters& cnt,
                               int max_loops) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 7; ++k) s.b[c][k] = 0.0;
    cnt.exact++;
    int rc = F.eval(true, s.t, s.x, s.v, s.a);
    if (rc != ST_OK) return rc;
    if (fabs(tf - s.t) < 1e-10) return ST_OK;
    double h = copysign(0.1, tf - s.t);
    double h_prev = 0.0;
    bool predict = false;
    int failures = 0;
    for (int loop = 0; loop < max_loops; ++loop) {
        if (fabs(s.t - tf) <= fabs(h)) h = tf - s.t;
        if (predict) {
#pragma unroll
            for (int c = 0; c < 3; ++c) predict_b_row(s.b[c], h / h_prev);
        }
        double nh = h;
        rc = radau_step(s, F, h, nh, cnt);
        if (rc == ST_OK) {
            h_prev = h;
            predict = true;
            h = nh;
            if (fabs(s.t - tf) < 1e-12) return ST_OK;
            failures = 0;
        } else if (rc == ST_IMPACT || rc == ST_DAF_LIMITS) {
            return rc;
        } else {
            predict = false;
            failures += 1;
            h *= 0.7;
            if (failures > 10) return ST_CONVERGENCE;
        }
        if (fabs(h) < 0.005) h = copysign(0.005, h);
    }
    return ST_TIMEOUT;
}

}  // namespace kb
