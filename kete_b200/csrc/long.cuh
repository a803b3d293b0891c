// long.cuh -- system integration without SPK perturbers: propagate_n_body_vec
// (kete_core/propagation/mod.rs:142-237) with vec_accel (acceleration.rs:197-249).
//
// The nine massive bodies of SIMPLE_PLANETS (Sun, Mercury, Venus, Earth-Moon barycentre,
// Mars to Neptune; gravity.rs:137-153) are integrated together with a batch of test
// particles by ONE Radau integration over all their coordinates: the step size and the
// convergence test take the maximum over the whole system (radau.rs:317-346 on a DVector).
// A thread block integrates one batch, one thread per body; each force evaluation is
// block-collective (the massive bodies' predicted states go through shared memory), and the
// convergence and step-size maxima are block reductions, so every thread takes the same
// decisions.  Every body feels every massive body but itself; the comet / dust model acts
// relative to the Sun on the batch's test particles after the first, as the reference's
// `idx > n_massive` (acceleration.rs:239-240) has it.  Each corrector starts from the
// predicted b (predict_b_row) and the integration runs in the frame the massive states are
// given in (heliocentric at the start epoch); results are relative to the Sun's final state.
#pragma once
#include "common.cuh"
#include "forces.cuh"
#include "internal.h"
#include "radau.cuh"

namespace kb {

constexpr int LONG_MASSIVE = 9;

__device__ __forceinline__ double long_block_max(double v, double* s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x >> 5;
    __syncthreads();  // s_red free from the previous reduction
    if ((threadIdx.x & 31) == 0) s_red[warp] = v;
    __syncthreads();
    double m = s_red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, s_red[w]);
    return m;
}

// GravParams::add_acceleration (gravity.rs:171-216) of massive body k on a body at relative
// position rp / velocity rv, into w.
__device__ __forceinline__ void long_pair(int k, const double rp[3], const double rv[3], double w[3]) {
    const double mass = c_tab.simple_mass[k];
    const int kind = c_tab.simple_kind[k];
    const double r2 = rp[0] * rp[0] + rp[1] * rp[1] + rp[2] * rp[2];
    const double ir = rsqrt(r2);
    const double ir3 = ir * ir * ir;
    const double kk = mass * ir3;
    w[0] -= rp[0] * kk;
    w[1] -= rp[1] * kk;
    w[2] -= rp[2] * kk;
    if (kind == FK_SUN || kind == FK_JUPITER) {
        const double r_v = 4.0 * (rp[0] * rv[0] + rp[1] * rv[1] + rp[2] * rv[2]);
        const double rel_v2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
        const double gr_const = mass * C_AU_PER_DAY_INV_SQUARED * ir3;
        const double c = 4. * mass * ir - rel_v2;
#pragma unroll
        for (int i = 0; i < 3; ++i) w[i] += gr_const * (c * rp[i] + r_v * rv[i]);
        const double rc = c_tab.rot_c, rs = c_tab.rot_s;
        const double ez = -rs * rp[1] + rc * rp[2];
        const double zr = ez * ir;
        const double z_squared = 5.0 * (zr * zr);
        const double rr = c_tab.simple_radius[k] * ir;
        const double coef = 1.5 * (kind == FK_JUPITER ? JUPITER_J2 : SUN_J2) * mass * (rr * rr) * ir3;
        const double ey = rc * rp[1] + rs * rp[2];
        const double jx = rp[0] * coef * (z_squared - 1.0);
        const double jy = ey * coef * (z_squared - 1.0);
        const double jz = ez * coef * (z_squared - 3.0);
        w[0] += jx;
        w[1] += rc * jy - rs * jz;
        w[2] += rs * jy + rc * jz;
    }
}

// Block-collective vec_accel at one evaluation point: every thread passes its body's
// point; the acceleration of active bodies lands in out.  Returns ST_IMPACT for the whole
// block when an exact evaluation finds a body within a massive body's radius.
__device__ __forceinline__ int long_eval(bool exact, int body, int m, const double xe[3],
                                         const double ve[3], const NonGrav& ng, double* s_m,
                                         double out[3]) {
    __syncthreads();  // the previous evaluation's reads of s_m are done
    if (body < LONG_MASSIVE) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            s_m[6 * body + c] = xe[c];
            s_m[6 * body + 3 + c] = ve[c];
        }
    }
    __syncthreads();
    int hit = 0;
    double acc[3] = {0.0, 0.0, 0.0};
    if (body < m) {
        for (int k = 0; k < LONG_MASSIVE; ++k) {
            if (k == body) continue;
            const double rp[3] = {xe[0] - s_m[6 * k], xe[1] - s_m[6 * k + 1], xe[2] - s_m[6 * k + 2]};
            const double rv[3] = {ve[0] - s_m[6 * k + 3], ve[1] - s_m[6 * k + 4], ve[2] - s_m[6 * k + 5]};
            if (exact && norm3(rp[0], rp[1], rp[2]) <= c_tab.simple_radius[k]) hit = 1;
            double w[3] = {0.0, 0.0, 0.0};
            long_pair(k, rp, rv, w);
            if (c_tab.simple_naif[k] == 10 && body > LONG_MASSIVE && ng.kind != 0) {
                const double3 na = nongrav_accel(ng, make_double3(rp[0], rp[1], rp[2]),
                                                 make_double3(rv[0], rv[1], rv[2]));
                w[0] += na.x;
                w[1] += na.y;
                w[2] += na.z;
            }
            acc[0] += w[0];
            acc[1] += w[1];
            acc[2] += w[2];
        }
    }
    out[0] = acc[0];
    out[1] = acc[1];
    out[2] = acc[2];
    return __syncthreads_or(hit) ? ST_IMPACT : ST_OK;
}

__global__ void __launch_bounds__(64) nbody_long_kernel(LongArgs a) {
    __shared__ double s_m[6 * LONG_MASSIVE];
    __shared__ double s_red[2];
    const int body = threadIdx.x;
    const int64_t i0 = (int64_t)blockIdx.x * a.batch;
    const int64_t rem = a.n - i0;
    const int nb = (int)(rem < a.batch ? rem : a.batch);
    const int m = LONG_MASSIVE + nb;
    const bool active = body < m;
    const int64_t obj = body >= LONG_MASSIVE ? i0 + (body - LONG_MASSIVE) : -1;
    const int64_t n = a.n;

    double x[3] = {0, 0, 0}, v[3] = {0, 0, 0}, acc[3] = {0, 0, 0};
    NonGrav ng;
    ng.base = nullptr;
    ng.stride = n;
    ng.kind = 0;
    if (body < LONG_MASSIVE) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            x[c] = a.planets[6 * body + c];
            v[c] = a.planets[6 * body + 3 + c];
        }
    } else if (active) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            x[c] = a.pos[c * n + obj];
            v[c] = a.vel[c * n + obj];
        }
        if (a.nongrav) {
            ng.base = a.nongrav + obj;
            ng.kind = (int)a.nongrav[obj];
        }
    }
    double b[3][7], g[3][7];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 7; ++k) b[c][k] = g[c][k] = 0.0;

    int rc = ST_OK;
    if (a.planet_status) {  // massive states read from the SPK on the device
        int bad = 0;
        if (body < LONG_MASSIVE && a.planet_status[body] != ST_OK) bad = 1;
        if (__syncthreads_or(bad)) rc = ST_DAF_LIMITS;
    }
    const double tf = a.jd1;
    double t = a.jd0;
    if (rc == ST_OK) rc = long_eval(true, body, m, x, v, ng, s_m, acc);
    if (rc == ST_OK && !(fabs(tf - t) < 1e-10)) {
        double h = copysign(0.1, tf - t), h_prev = 0.0;
        bool predict = false;
        int failures = 0;
        rc = ST_TIMEOUT;
        for (int loop = 0; loop < a.max_loops; ++loop) {
            if (fabs(t - tf) <= fabs(h)) h = tf - t;
            if (predict) {
#pragma unroll
                for (int c = 0; c < 3; ++c) predict_b_row(b[c], h / h_prev);
            }
            bool converged = false;
            int erc = ST_OK;
            double next_h = h;
            const double h2 = h * h;
            for (int iter = 0; iter < 10 && !converged; ++iter) {
                double b6_old[3] = {b[0][6], b[1][6], b[2][6]};
                double ev[3] = {acc[0], acc[1], acc[2]};
#pragma unroll
                for (int j = 1; j < 8; ++j) {
                    const double f = c_tab.spacing[j];
                    double xs[3], vs[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double bw = 0.0, bu = 0.0;
#pragma unroll
                        for (int k = 0; k < 7; ++k) {
                            bw += c_tab.w_pow[j][k] * b[c][k];
                            bu += c_tab.u_pow[j][k] * b[c][k];
                        }
                        xs[c] = x[c] + f * v[c] * h + c_tab.frac2[j] * h2 * (acc[c] / 2.0 + bw);
                        vs[c] = v[c] + f * h * (acc[c] + bu);
                    }
                    long_eval(false, body, m, xs, vs, ng, s_m, ev);
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double gk = (ev[c] - acc[c]) * c_tab.inv_frac[j];
#pragma unroll
                        for (int z = 1; z < 7; ++z)
                            if (z < j) gk = (gk - g[c][z - 1]) * c_tab.inv_diff[j][z];
#pragma unroll
                        for (int k = 0; k < 7; ++k)
                            if (k == j - 1) g[c][k] = gk;
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int jj = 0; jj < 7; ++jj) {
                        double s2 = g[c][jj];
#pragma unroll
                        for (int k = jj + 1; k < 7; ++k) s2 += c_tab.c[k][jj] * g[c][k];
                        b[c][jj] = s2;
                    }
                double ratio = 0.0, fem = 0.0, mb6 = 0.0;
                if (active) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const double fe = fabs(ev[c]) + 1e-6;
                        ratio = fmax(ratio, fabs(b[c][6] - b6_old[c]) / fe);
                        fem = fmax(fem, fe);
                        mb6 = fmax(mb6, fabs(b[c][6]));
                    }
                }
                if (long_block_max(ratio, s_red) < 1e-14) {
                    const double fem_max = long_block_max(fem, s_red);
                    const double b6_max = long_block_max(mb6, s_red);
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double dw = 0.0, du = 0.0;
#pragma unroll
                        for (int k = 0; k < 7; ++k) {
                            dw += b[c][k] * c_tab.w[k];
                            du += b[c][k] * c_tab.u[k];
                        }
                        x[c] += v[c] * h + h2 * (acc[c] * 0.5 + dw);
                        v[c] += h * (acc[c] + du);
                    }
                    t += h;
                    erc = long_eval(true, body, m, x, v, ng, s_m, acc);
                    next_h = h * clampd(pow(1e-6 * fem_max / b6_max, 1.0 / 7.0), 0.25, 4.0);
                    converged = true;
                }
            }
            if (erc != ST_OK) {
                rc = erc;
                break;
            }
            if (converged) {
                h_prev = h;
                predict = true;
                h = next_h;
                if (fabs(t - tf) < 1e-12) {
                    rc = ST_OK;
                    break;
                }
                failures = 0;
            } else {
                predict = false;
                failures += 1;
                h *= 0.7;
                if (failures > 10) {
                    rc = ST_CONVERGENCE;
                    break;
                }
            }
            if (fabs(h) < 0.005) h = copysign(0.005, h);
        }
    }
    // results relative to the Sun's final state
    __syncthreads();
    if (body == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            s_m[c] = x[c];
            s_m[3 + c] = v[c];
        }
    }
    __syncthreads();
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (obj >= 0 && active) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a.out_pos[c * n + obj] = rc == ST_OK ? x[c] - s_m[c] : nan;
            a.out_vel[c * n + obj] = rc == ST_OK ? v[c] - s_m[3 + c] : nan;
        }
        a.status[obj] = rc;
    }
    if (a.out_planets && blockIdx.x == gridDim.x - 1 && body < LONG_MASSIVE) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a.out_planets[6 * body + c] = rc == ST_OK ? x[c] - s_m[c] : nan;
            a.out_planets[6 * body + 3 + c] = rc == ST_OK ? v[c] - s_m[3 + c] : nan;
        }
    }
}

// -------------------------------------------------------------------------------------------
// The same integration with the seven corrector nodes in parallel (batches of up to 23 test
// particles, 32 bodies with the massive ones): warp w evaluates node w + 1 of every body of
// the batch (lane = body), as the node evaluations of one corrector iteration only use the
// previous iteration's b.  The state, b and the node evaluations live in shared memory; the
// divided differences, b and the state update are then formed by one thread per (body,
// coordinate), in the same order as nbody_long_kernel, and the step-end evaluation by warp
// 0.  An iteration then costs one evaluation's latency instead of seven.
// -------------------------------------------------------------------------------------------
constexpr int LN_WARPS = 7;
constexpr int LN_BODIES = 32;

__device__ __forceinline__ double ln_block_max(double v, double* s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();  // s_red free from the previous reduction
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = s_red[0];
#pragma unroll
    for (int w = 1; w < LN_WARPS; ++w) m = fmax(m, s_red[w]);
    return m;
}

// Warp-collective vec_accel at one evaluation point per lane (lane = body); ms holds the
// massive bodies' states of this warp's point.  Returns ST_IMPACT for the warp when an exact
// evaluation finds a body within a massive body's radius.
__device__ __forceinline__ int ln_eval(bool exact, int body, int m, const double xe[3],
                                       const double ve[3], const NonGrav& ng, double* ms,
                                       double out[3]) {
    __syncwarp();  // the previous evaluation's reads of ms are done
    if (body < LONG_MASSIVE) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ms[6 * body + c] = xe[c];
            ms[6 * body + 3 + c] = ve[c];
        }
    }
    __syncwarp();
    int hit = 0;
    double acc[3] = {0.0, 0.0, 0.0};
    if (body < m) {
        for (int k = 0; k < LONG_MASSIVE; ++k) {
            if (k == body) continue;
            const double rp[3] = {xe[0] - ms[6 * k], xe[1] - ms[6 * k + 1], xe[2] - ms[6 * k + 2]};
            const double rv[3] = {ve[0] - ms[6 * k + 3], ve[1] - ms[6 * k + 4], ve[2] - ms[6 * k + 5]};
            if (exact && norm3(rp[0], rp[1], rp[2]) <= c_tab.simple_radius[k]) hit = 1;
            double w[3] = {0.0, 0.0, 0.0};
            long_pair(k, rp, rv, w);
            if (c_tab.simple_naif[k] == 10 && body > LONG_MASSIVE && ng.kind != 0) {
                const double3 na = nongrav_accel(ng, make_double3(rp[0], rp[1], rp[2]),
                                                 make_double3(rv[0], rv[1], rv[2]));
                w[0] += na.x;
                w[1] += na.y;
                w[2] += na.z;
            }
            acc[0] += w[0];
            acc[1] += w[1];
            acc[2] += w[2];
        }
    }
    out[0] = acc[0];
    out[1] = acc[1];
    out[2] = acc[2];
    return __any_sync(0xffffffffu, hit) ? ST_IMPACT : ST_OK;
}

__global__ void __launch_bounds__(32 * LN_WARPS) nbody_long_nodes_kernel(LongArgs a) {
    __shared__ double s_x[LN_BODIES][3], s_v[LN_BODIES][3], s_acc[LN_BODIES][3];
    __shared__ double s_b[LN_BODIES][3][7];
    __shared__ double s_ev[LN_WARPS][LN_BODIES][3];
    __shared__ double s_ms[LN_WARPS][6 * LONG_MASSIVE];
    __shared__ double s_red[LN_WARPS];
    __shared__ int s_rc;
    const int body = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int64_t i0 = (int64_t)blockIdx.x * a.batch;
    const int64_t rem = a.n - i0;
    const int nb = (int)(rem < a.batch ? rem : a.batch);
    const int m = LONG_MASSIVE + nb;
    const bool active = body < m;
    const int64_t obj = body >= LONG_MASSIVE ? i0 + (body - LONG_MASSIVE) : -1;
    const int64_t n = a.n;
    // the (body, coordinate) this thread forms g, b and the state update for
    const int tb = threadIdx.x / 3, tc = threadIdx.x % 3;
    const bool task = threadIdx.x < 3 * LN_BODIES && tb < m;

    NonGrav ng;
    ng.base = nullptr;
    ng.stride = n;
    ng.kind = 0;
    if (active && body >= LONG_MASSIVE && a.nongrav) {
        ng.base = a.nongrav + obj;
        ng.kind = (int)a.nongrav[obj];
    }
    if (warp == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double xv = 0.0, vv = 0.0;
            if (body < LONG_MASSIVE) {
                xv = a.planets[6 * body + c];
                vv = a.planets[6 * body + 3 + c];
            } else if (active) {
                xv = a.pos[c * n + obj];
                vv = a.vel[c * n + obj];
            }
            s_x[body][c] = xv;
            s_v[body][c] = vv;
            s_acc[body][c] = 0.0;
        }
    }
    for (int k = threadIdx.x; k < LN_BODIES * 21; k += blockDim.x) (&s_b[0][0][0])[k] = 0.0;
    if (threadIdx.x == 0) s_rc = ST_OK;
    __syncthreads();

    int rc = ST_OK;
    if (a.planet_status) {  // massive states read from the SPK on the device
        int bad = 0;
        if (warp == 0 && body < LONG_MASSIVE && a.planet_status[body] != ST_OK) bad = 1;
        if (__syncthreads_or(bad)) rc = ST_DAF_LIMITS;
    }
    // exact evaluation of the current state by warp 0 into s_acc; block-uniform status
    auto exact_eval = [&]() -> int {
        __syncthreads();  // the state is complete
        if (warp == 0) {
            double xe[3], ve[3], ev[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                xe[c] = s_x[body][c];
                ve[c] = s_v[body][c];
            }
            const int erc = ln_eval(true, body, m, xe, ve, ng, s_ms[0], ev);
#pragma unroll
            for (int c = 0; c < 3; ++c) s_acc[body][c] = ev[c];
            if (body == 0) s_rc = erc;
        }
        __syncthreads();
        return s_rc;
    };
    const double tf = a.jd1;
    double t = a.jd0;
    if (rc == ST_OK) rc = exact_eval();
    if (rc == ST_OK && !(fabs(tf - t) < 1e-10)) {
        double h = copysign(0.1, tf - t), h_prev = 0.0;
        bool predict = false;
        int failures = 0;
        rc = ST_TIMEOUT;
        const int j = warp + 1;  // this warp's node
        const double f = c_tab.spacing[j], fr2 = c_tab.frac2[j];
        for (int loop = 0; loop < a.max_loops; ++loop) {
            if (fabs(t - tf) <= fabs(h)) h = tf - t;
            if (predict && task) predict_b_row(s_b[tb][tc], h / h_prev);
            __syncthreads();
            bool converged = false;
            int erc = ST_OK;
            double next_h = h;
            const double h2 = h * h;
            for (int iter = 0; iter < 10 && !converged; ++iter) {
                // node j of every body
                double xs[3], vs[3], ev[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    double bw = 0.0, bu = 0.0;
#pragma unroll
                    for (int k = 0; k < 7; ++k) {
                        bw += c_tab.w_pow[j][k] * s_b[body][c][k];
                        bu += c_tab.u_pow[j][k] * s_b[body][c][k];
                    }
                    xs[c] = s_x[body][c] + f * s_v[body][c] * h + fr2 * h2 * (s_acc[body][c] / 2.0 + bw);
                    vs[c] = s_v[body][c] + f * h * (s_acc[body][c] + bu);
                }
                ln_eval(false, body, m, xs, vs, ng, s_ms[warp], ev);
#pragma unroll
                for (int c = 0; c < 3; ++c) s_ev[warp][body][c] = ev[c];
                __syncthreads();  // every node evaluated; b still the previous iteration's
                double ratio = 0.0, fem = 0.0, mb6 = 0.0;
                if (task) {
                    const double ac = s_acc[tb][tc];
                    const double b6_old = s_b[tb][tc][6];
                    double g[7];
#pragma unroll
                    for (int jj = 1; jj < 8; ++jj) {
                        double gk = (s_ev[jj - 1][tb][tc] - ac) * c_tab.inv_frac[jj];
#pragma unroll
                        for (int z = 1; z < 7; ++z)
                            if (z < jj) gk = (gk - g[z - 1]) * c_tab.inv_diff[jj][z];
                        g[jj - 1] = gk;
                    }
                    double bn[7];
#pragma unroll
                    for (int jj = 0; jj < 7; ++jj) {
                        double s2 = g[jj];
#pragma unroll
                        for (int k = jj + 1; k < 7; ++k) s2 += c_tab.c[k][jj] * g[k];
                        bn[jj] = s2;
                    }
#pragma unroll
                    for (int jj = 0; jj < 7; ++jj) s_b[tb][tc][jj] = bn[jj];
                    // the convergence test reads the last node's evaluation (node 7)
                    const double fe = fabs(s_ev[LN_WARPS - 1][tb][tc]) + 1e-6;
                    ratio = fabs(bn[6] - b6_old) / fe;
                    fem = fe;
                    mb6 = fabs(bn[6]);
                }
                if (ln_block_max(ratio, s_red) < 1e-14) {
                    const double fem_max = ln_block_max(fem, s_red);
                    const double b6_max = ln_block_max(mb6, s_red);
                    if (task) {
                        double dw = 0.0, du = 0.0;
#pragma unroll
                        for (int k = 0; k < 7; ++k) {
                            dw += s_b[tb][tc][k] * c_tab.w[k];
                            du += s_b[tb][tc][k] * c_tab.u[k];
                        }
                        const double xo = s_x[tb][tc], vo = s_v[tb][tc], ao = s_acc[tb][tc];
                        s_x[tb][tc] = xo + (vo * h + h2 * (ao * 0.5 + dw));
                        s_v[tb][tc] = vo + h * (ao + du);
                    }
                    t += h;
                    erc = exact_eval();
                    next_h = h * clampd(pow(1e-6 * fem_max / b6_max, 1.0 / 7.0), 0.25, 4.0);
                    converged = true;
                }
            }
            if (erc != ST_OK) {
                rc = erc;
                break;
            }
            if (converged) {
                h_prev = h;
                predict = true;
                h = next_h;
                if (fabs(t - tf) < 1e-12) {
                    rc = ST_OK;
                    break;
                }
                failures = 0;
            } else {
                predict = false;
                failures += 1;
                h *= 0.7;
                if (failures > 10) {
                    rc = ST_CONVERGENCE;
                    break;
                }
            }
            if (fabs(h) < 0.005) h = copysign(0.005, h);
        }
    }
    // results relative to the Sun's final state
    __syncthreads();
    if (warp == 0) {
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        if (obj >= 0 && active) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                a.out_pos[c * n + obj] = rc == ST_OK ? s_x[body][c] - s_x[0][c] : nan;
                a.out_vel[c * n + obj] = rc == ST_OK ? s_v[body][c] - s_v[0][c] : nan;
            }
            a.status[obj] = rc;
        }
        if (a.out_planets && blockIdx.x == gridDim.x - 1 && body < LONG_MASSIVE) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                a.out_planets[6 * body + c] = rc == ST_OK ? s_x[body][c] - s_x[0][c] : nan;
                a.out_planets[6 * body + 3 + c] = rc == ST_OK ? s_v[body][c] - s_v[0][c] : nan;
            }
        }
    }
}

}  // namespace kb
