// kepler_stm.cuh -- two-body state-transition matrices and covariance propagation.
//
// kete's compute_stm / propagate_covariance (src/kete/state_transition.py:8-59,
// kete_core/propagation/state_transition.rs:52-122) integrate the variational equations
// with RK4(5) and carry three defects: the acceleration Jacobian is off by a factor -1/2
// (acceleration.rs:267-290), the scaled-time equations use the unscaled GM
// (state_transition.rs:6-47 with acceleration.rs:66-80), and the matrix comes back
// transposed (state_transition.rs:86-121).  Here the matrix is d(p1, v1)/d(p0, v0) of the
// closed-form two-body solution itself: the final state is analytic_2_body's (kepler.rs:
// 254-297, the same interval halving), and each closed-form step is differentiated with
// dual numbers.  The universal anomaly's derivative comes from the implicit function
// theorem on the Kepler equation, ds = -dF / F'(s), at the anomaly of the unreduced
// equation (the elliptic solve reduces time modulo the period, which moves with the
// state).  Leaf Jacobians chain in the order the steps run.
#pragma once
#include "common.cuh"
#include "kepler.cuh"
#include "tangent.cuh"

namespace kb {

__device__ __forceinline__ D6 dsqrt(const D6& a) {
    const double r = sqrt(a.v);
    const double k = 0.5 / r;
    D6 o;
    o.v = r;
#pragma unroll
    for (int i = 0; i < 6; ++i) o.d[i] = a.d[i] * k;
    return o;
}

// sin and cos, or sinh and cosh, of a dual argument
__device__ __forceinline__ void dsincos(const D6& x, bool hyperbolic, D6& sn, D6& cs) {
    double s, c;
    if (hyperbolic) {
        s = sinh(x.v);
        c = cosh(x.v);
    } else {
        sincos(x.v, &s, &c);
    }
    sn.v = s;
    cs.v = c;
    const double dc = hyperbolic ? s : -s;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        sn.d[i] = x.d[i] * c;
        cs.d[i] = x.d[i] * dc;
    }
}

// Universal functions g1 = s c1(z), g2 = s^2 c2(z), g3 = s^3 c3(z) with z = beta s^2
// (Stumpff functions).  For |z| < 0.1 the alternating series, which stays accurate where
// (s - g1) / beta cancels; otherwise the circular or hyperbolic closed forms.
__device__ __forceinline__ void universal_dual(const D6& s, const D6& beta, D6& g1, D6& g2, D6& g3) {
    const D6 z = beta * s * s;
    if (fabs(z.v) < 0.1) {
        // c_k(z) = sum_j (-z)^j / (2j + k)!, eight terms (next term below 1e-23)
        D6 c1 = dconst(0.0), c2 = dconst(0.0), c3 = dconst(0.0);
        double f1 = 1.0, f2 = 2.0, f3 = 6.0;  // 1!, 2!, 3!
        D6 zp = dconst(1.0);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c1 = c1 + zp * (1.0 / f1);
            c2 = c2 + zp * (1.0 / f2);
            c3 = c3 + zp * (1.0 / f3);
            zp = zp * (-1.0) * z;
            f1 *= (double)((2 * j + 2) * (2 * j + 3));
            f2 *= (double)((2 * j + 3) * (2 * j + 4));
            f3 *= (double)((2 * j + 4) * (2 * j + 5));
        }
        g1 = s * c1;
        g2 = s * s * c2;
        g3 = s * s * s * c3;
        return;
    }
    const bool hyp = beta.v < 0.0;
    const D6 bs = hyp ? dsqrt(-beta) : dsqrt(beta);
    D6 sn, cs;
    dsincos(bs * s, hyp, sn, cs);
    g1 = sn / bs;
    g2 = (1.0 - cs) / beta;  // 2 sin^2(x/2) / beta, and (1 - cosh x) / beta
    g3 = (s - g1) / beta;
}

// One closed-form step of dt from (p, v), in place, with its 6x6 Jacobian J (row-major,
// rows d(p1, v1), columns d(p0, v0)).  Values follow two_body_leaf exactly.
__device__ __forceinline__ int two_body_leaf_stm(double dt, double p[3], double v[3], double mu,
                                                 double J[36]) {
    const double r0 = norm3(p[0], p[1], p[2]);
    const double v0 = norm3(v[0], v[1], v[2]);
    const double rv0 = p[0] * v[0] + p[1] * v[1] + p[2] * v[2];
    double s, beta;
    if (solve_kepler_universal(dt, r0, v0, rv0, s, beta, mu) != ST_OK) return ST_CONVERGENCE;
    // the anomaly of the unreduced equation: whole revolutions added back
    double s_full = s;
    if (beta >= PARABOLIC_BETA) {
        const double b_sqrt = sqrt(beta);
        const double period = mu * powi<-3>(b_sqrt) * TAU;
        const double revs = rint((dt - fmod(dt, period)) / period);
        s_full = s + revs * TAU / b_sqrt;
    }
    D6 P[3], V[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        P[i] = dconst(p[i]);
        V[i] = dconst(v[i]);
        P[i].d[i] = 1.0;
        V[i].d[3 + i] = 1.0;
    }
    const D6 R0 = dsqrt(ddot(P, P));
    const D6 RV0 = ddot(P, V);
    const D6 B = 2.0 * mu * drecip(R0) - ddot(V, V);
    // dF at fixed s, and dF/ds = r0 g0 + rv0 g1 + mu g2 with g0 = 1 - beta g2
    D6 g1, g2, g3;
    universal_dual(dconst(s_full), B, g1, g2, g3);
    const D6 F = R0 * g1 + RV0 * g2 + mu * g3;
    const double Fs = r0 * (1.0 - B.v * g2.v) + rv0 * g1.v + mu * g2.v;
    D6 S = dconst(s_full);
#pragma unroll
    for (int i = 0; i < 6; ++i) S.d[i] = -F.d[i] / Fs;
    universal_dual(S, B, g1, g2, g3);
    const D6 f = 1.0 - mu * drecip(R0) * g2;
    const D6 g = R0 * g1 + RV0 * g2;
    D6 NP[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) NP[i] = P[i] * f + V[i] * g;
    const D6 NR = dsqrt(ddot(NP, NP));
    const D6 f_dot = -mu * drecip(NR * R0) * g1;
    const D6 g_dot = 1.0 - mu * drecip(NR) * g2;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const D6 NV = P[i] * f_dot + V[i] * g_dot;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            J[i * 6 + c] = NP[i].d[c];
            J[(3 + i) * 6 + c] = NV.d[c];
        }
    }
    two_body_apply(s, beta, r0, rv0, p, v, mu);
    return ST_OK;
}

// analytic_2_body with the state-transition matrix Phi (row-major 6x6) chained through the
// leaves; Phi starts as the identity.
static __device__ __noinline__ int analytic_2_body_stm(double time, double p[3], double v[3], double mu,
                                                double Phi[36]) {
#pragma unroll
    for (int k = 0; k < 36; ++k) Phi[k] = (k % 7 == 0) ? 1.0 : 0.0;
    double st_dt[12];
    int st_depth[12];
    st_dt[0] = time;
    st_depth[0] = 0;
    int top = 1;
    int guard = 0;
    double J[36];
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
        if (two_body_leaf_stm(dt, p, v, mu, J) == ST_OK) {
            double tmp[36];
            for (int r = 0; r < 6; ++r)
                for (int c = 0; c < 6; ++c) {
                    double acc = 0.0;
#pragma unroll
                    for (int k = 0; k < 6; ++k) acc += J[r * 6 + k] * Phi[k * 6 + c];
                    tmp[r * 6 + c] = acc;
                }
#pragma unroll
            for (int k = 0; k < 36; ++k) Phi[k] = tmp[k];
            continue;
        }
        if (top + 2 > 12) return ST_CONVERGENCE;
        st_dt[top] = dt * 0.5;
        st_depth[top] = depth;
        st_dt[top + 1] = 0.5 * dt;
        st_depth[top + 1] = depth;
        top += 2;
    }
    return ST_OK;
}

}  // namespace kb
