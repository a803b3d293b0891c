// sens.cu -- N-body forward sensitivities: the node-parallel form (nbody_stm_nodes_kernel,
// stm_nodes.cuh) and the one-object-per-thread form (nbody_stm_kernel, every force term in
// dual numbers from tangent.cuh, the Jacobian of every corrector iteration at its own
// points), with their host launcher.
// every object of the differentiation workloads carries the comet model: inline it
#define KB_FORCE_NG_INLINE 1
#include "common.cuh"
#include "forces.cuh"
#include "internal.h"
#include "radau.cuh"
#include "stm_nodes.cuh"
#include "tangent.cuh"

namespace kb {
KB_CONSTANT_UPLOADER(sens)
}  // namespace kb

namespace kb {

// -------------------------------------------------------------------------------------------
// N-body propagation with forward sensitivities: the state at each of n_epochs epochs and
// its 6 x 8 derivative with respect to the initial position, initial velocity, A1 and A2.
// One object per thread; every epoch starts a fresh integration from the previous one, as
// consecutive propagate_n_body calls do (kete_core/propagation/mod.rs:70-118).
// -------------------------------------------------------------------------------------------
__device__ void radau_tangent_segment(TangentForce& F, double& t, double tf, double x[3],
                                      double v[3], double dx[3][TAN_DIRS], double dv[3][TAN_DIRS],
                                      int max_loops, int& rc_out) {
    double a[3], da[3][TAN_DIRS], J[3][6], jp[3][2];
    double b[3][7], db[3][7][TAN_DIRS];
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 7; ++k) {
            b[c][k] = 0.0;
            for (int p = 0; p < TAN_DIRS; ++p) db[c][k][p] = 0.0;
        }
    auto tangent_of = [&](double out[3][TAN_DIRS], const double X[3][TAN_DIRS],
                          const double V[3][TAN_DIRS]) {
        for (int c = 0; c < 3; ++c)
            for (int p = 0; p < TAN_DIRS; ++p) {
                double s = 0.0;
                for (int i = 0; i < 3; ++i) s += J[c][i] * X[i][p] + J[c][3 + i] * V[i][p];
                if (p == 6) s += jp[c][0];
                if (p == 7) s += jp[c][1];
                out[c][p] = s;
            }
    };
    int rc = F.eval(true, t, x, v, a, J, jp);
    if (rc != ST_OK) {
        rc_out = rc;
        return;
    }
    tangent_of(da, dx, dv);
    if (fabs(tf - t) < 1e-10) {
        rc_out = ST_OK;
        return;
    }
    double h = copysign(0.1, tf - t);
    double h_prev = 0.0;
    bool predict = false;
    int failures = 0;
    for (int loop = 0; loop < max_loops; ++loop) {
        if (fabs(t - tf) <= fabs(h)) h = tf - t;
        if (predict) {  // the predicted b (predict_b_row) and its tangent
            const double q = h / h_prev;
            for (int c = 0; c < 3; ++c) {
                predict_b_row(b[c], q);
                for (int p = 0; p < TAN_DIRS; ++p) {
                    double row[7];
                    for (int k = 0; k < 7; ++k) row[k] = db[c][k][p];
                    predict_b_row(row, q);
                    for (int k = 0; k < 7; ++k) db[c][k][p] = row[k];
                }
            }
        }
        // ---- one step (radau.rs:225-346) with its tangent ----
        double g[3][7], dg[3][7][TAN_DIRS];
        double ev[3] = {a[0], a[1], a[2]};
        const double h2 = h * h;
        bool converged = false;
        double next_h = h;
        for (int iter = 0; iter < 10 && rc == ST_OK && !converged; ++iter) {
            const double b6_old[3] = {b[0][6], b[1][6], b[2][6]};
            for (int j = 1; j < 8; ++j) {
                const double f = c_tab.spacing[j];
                double xs[3], vs[3], dX[3][TAN_DIRS], dV[3][TAN_DIRS], dE[3][TAN_DIRS];
                for (int c = 0; c < 3; ++c) {
                    double bw = 0.0, bu = 0.0;
                    for (int k = 0; k < 7; ++k) {
                        bw += c_tab.w_pow[j][k] * b[c][k];
                        bu += c_tab.u_pow[j][k] * b[c][k];
                    }
                    xs[c] = x[c] + f * v[c] * h + c_tab.frac2[j] * h2 * (a[c] / 2.0 + bw);
                    vs[c] = v[c] + f * h * (a[c] + bu);
                    for (int p = 0; p < TAN_DIRS; ++p) {
                        double dbw = 0.0, dbu = 0.0;
                        for (int k = 0; k < 7; ++k) {
                            dbw += c_tab.w_pow[j][k] * db[c][k][p];
                            dbu += c_tab.u_pow[j][k] * db[c][k][p];
                        }
                        dX[c][p] = dx[c][p] + f * dv[c][p] * h + c_tab.frac2[j] * h2 * (da[c][p] / 2.0 + dbw);
                        dV[c][p] = dv[c][p] + f * h * (da[c][p] + dbu);
                    }
                }
                rc = F.eval(false, t + f * h, xs, vs, ev, J, jp);
                if (rc != ST_OK) break;
                tangent_of(dE, dX, dV);
                for (int c = 0; c < 3; ++c) {
                    double gk = (ev[c] - a[c]) * c_tab.inv_frac[j];
                    for (int z = 1; z < j; ++z) gk = (gk - g[c][z - 1]) * c_tab.inv_diff[j][z];
                    g[c][j - 1] = gk;
                    for (int p = 0; p < TAN_DIRS; ++p) {
                        double dgk = (dE[c][p] - da[c][p]) * c_tab.inv_frac[j];
                        for (int z = 1; z < j; ++z) dgk = (dgk - dg[c][z - 1][p]) * c_tab.inv_diff[j][z];
                        dg[c][j - 1][p] = dgk;
                    }
                }
            }
            if (rc != ST_OK) break;
            for (int c = 0; c < 3; ++c)
                for (int jj = 0; jj < 7; ++jj) {
                    double s2 = g[c][jj];
                    for (int k = jj + 1; k < 7; ++k) s2 += c_tab.c[k][jj] * g[c][k];
                    b[c][jj] = s2;
                    for (int p = 0; p < TAN_DIRS; ++p) {
                        double d2 = dg[c][jj][p];
                        for (int k = jj + 1; k < 7; ++k) d2 += c_tab.c[k][jj] * dg[c][k][p];
                        db[c][jj][p] = d2;
                    }
                }
            double fem[3], ratio[3];
            for (int c = 0; c < 3; ++c) {
                fem[c] = fabs(ev[c]) + 1e-6;
                ratio[c] = fabs(b[c][6] - b6_old[c]) / fem[c];
            }
            if (fmax(fmax(ratio[0], ratio[1]), ratio[2]) < 1e-14) {
                for (int c = 0; c < 3; ++c) {
                    double dw = 0.0, du = 0.0;
                    for (int k = 0; k < 7; ++k) {
                        dw += b[c][k] * c_tab.w[k];
                        du += b[c][k] * c_tab.u[k];
                    }
                    for (int p = 0; p < TAN_DIRS; ++p) {
                        double ddw = 0.0, ddu = 0.0;
                        for (int k = 0; k < 7; ++k) {
                            ddw += db[c][k][p] * c_tab.w[k];
                            ddu += db[c][k][p] * c_tab.u[k];
                        }
                        dx[c][p] += dv[c][p] * h + h2 * (da[c][p] * 0.5 + ddw);
                        dv[c][p] += h * (da[c][p] + ddu);
                    }
                    x[c] += v[c] * h + h2 * (a[c] * 0.5 + dw);
                    v[c] += h * (a[c] + du);
                }
                t += h;
                rc = F.eval(true, t, x, v, a, J, jp);
                if (rc != ST_OK) break;
                tangent_of(da, dx, dv);
                const double mb6 = fmax(fmax(fabs(b[0][6]), fabs(b[1][6])), fabs(b[2][6]));
                const double r = pow(1e-6 * fmax(fmax(fem[0], fem[1]), fem[2]) / mb6, 1.0 / 7.0);
                next_h = h * clampd(r, 0.25, 4.0);
                converged = true;
            }
        }
        if (rc == ST_IMPACT || rc == ST_DAF_LIMITS) {
            rc_out = rc;
            return;
        }
        if (converged) {
            h_prev = h;
            predict = true;
            h = next_h;
            if (fabs(t - tf) < 1e-12) {
                rc_out = ST_OK;
                return;
            }
            failures = 0;
        } else {
            rc = ST_OK;
            predict = false;
            failures += 1;
            h *= 0.7;
            if (failures > 10) {
                rc_out = ST_CONVERGENCE;
                return;
            }
        }
        if (fabs(h) < 0.005) h = copysign(0.005, h);
    }
    rc_out = ST_TIMEOUT;
}

__global__ void __launch_bounds__(64) nbody_stm_kernel(StmArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t n = a.n;
    double t = a.jd0[i];
    double x[3] = {a.pos[i], a.pos[n + i], a.pos[2 * n + i]};
    double v[3] = {a.vel[i], a.vel[n + i], a.vel[2 * n + i]};
    // d(state in the integration frame)/d(initial state in the caller's frame)
    double R[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    if (a.frame == FRAME_ECLIPTIC) {
        const double c = c_tab.rot_c, s = c_tab.rot_s;
        R[1][1] = c; R[1][2] = -s; R[2][1] = s; R[2][2] = c;
    }
    double dx[3][TAN_DIRS], dv[3][TAN_DIRS];
    for (int c = 0; c < 3; ++c)
        for (int p = 0; p < TAN_DIRS; ++p) {
            dx[c][p] = p < 3 ? R[c][p] : 0.0;
            dv[c][p] = (p >= 3 && p < 6) ? R[c][p - 3] : 0.0;
        }
    TangentForce F;
    F.n_force = a.n_force;
    F.ng.base = a.nongrav ? a.nongrav + i : nullptr;
    F.ng.stride = n;
    F.ng.kind = a.nongrav ? (int)a.nongrav[i] : 0;
    F.impact_id = 0;
    F.min_dist = 1e300;
    int rc = ST_OK;
    if (!(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]) && isfinite(v[0]) && isfinite(v[1]) &&
          isfinite(v[2]) && isfinite(t)))
        rc = ST_VALUE_ERROR;
    // the derivative of the comet model is taken with its time delay dt = 0
    if (F.ng.kind == 1 && F.ng.p(9) != 0.0) rc = ST_VALUE_ERROR;
    if (rc == ST_OK) rc = to_ssb_equatorial(t, a.frame, a.chain, x, v);
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int k = 0; k < a.n_epochs; ++k) {
        if (rc == ST_OK) radau_tangent_segment(F, t, a.epochs[k], x, v, dx, dv, a.max_loops, rc);
        double px[3] = {x[0], x[1], x[2]}, pv[3] = {v[0], v[1], v[2]};
        int orc = rc;
        if (orc == ST_OK) orc = from_ssb_equatorial(a.epochs[k], a.frame, a.chain, px, pv);
        double* st = a.out_state + (int64_t)k * 6 * n;
        double* phi = a.out_stm + (int64_t)k * 48 * n;
        for (int c = 0; c < 3; ++c) {
            st[c * n + i] = orc == ST_OK ? px[c] : nan;
            st[(3 + c) * n + i] = orc == ST_OK ? pv[c] : nan;
            for (int p = 0; p < TAN_DIRS; ++p) {
                // back to the caller's frame: R^T d(state)
                double sx = 0.0, sv = 0.0;
                for (int q = 0; q < 3; ++q) {
                    sx += R[q][c] * dx[q][p];
                    sv += R[q][c] * dv[q][p];
                }
                phi[(c * TAN_DIRS + p) * n + i] = orc == ST_OK ? sx : nan;
                phi[((3 + c) * TAN_DIRS + p) * n + i] = orc == ST_OK ? sv : nan;
            }
        }
        if (orc != ST_OK) rc = orc;
    }
    a.status[i] = rc;
}

int launch_nbody_stm(const StmArgs& a, int form, cudaStream_t stream) {
    if (a.n <= 0) return 0;
    if (form == 1) {  // one object per thread
        nbody_stm_kernel<<<(unsigned)((a.n + 63) / 64), 64, 0, stream>>>(a);
        return launched(1, "nbody_stm_kernel launch");
    }
    // node-parallel: tangents in dynamic shared memory above the 48 KB static limit (a
    // function attribute, set on every launch: it is not a stream operation)
    int rc = cuda_check(cudaFuncSetAttribute(nbody_stm_nodes_kernel<1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             STM_DYN_SMEM),
                        "sensitivity kernel shared memory");
    if (rc) return rc;
    const int64_t grid = (a.n * SG + STM_BLOCK - 1) / STM_BLOCK;
    nbody_stm_nodes_kernel<1><<<(unsigned)grid, STM_BLOCK, STM_DYN_SMEM, stream>>>(a);
    return launched(1, "nbody_stm_nodes_kernel launch");
}

}  // namespace kb
