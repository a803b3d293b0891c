// stm_nodes.cuh -- forward sensitivities of the N-body propagation on the node-parallel
// layout: the state and its 6 x 8 derivative with respect to the initial position, initial
// velocity, A1 and A2 at each of n epochs, for 8 lanes per object.
//
// The step loop is the one of the checkpointed forward pass (sens_rounds, adjoint.cuh): every
// object is integrated by a group of 8 lanes with the seven corrector nodes in parallel,
// every epoch a fresh integration from the previous one, as consecutive propagate_n_body_spk
// calls are (kete_core/propagation/mod.rs:70-118).  The tangents are carried through each
// step attempt as executed, with its step size and iteration count held fixed:
//   dX_j = dx + f_j h dv + f_j^2 h^2 (da/2 + W_j.db),  dV_j = dv + f_j h (da + U_j.db)
//   dE_j = J_j (dX_j, dV_j) + jp_j,   db^m = P (dE^m - da),   P = C_MAT . divided differences
//   db^0 = S(q) db^M of the previous attempt (the predicted corrector start; identity after a
//   failed attempt, zero at the start of an epoch)
//   dx' = dx + h dv + h^2 (da/2 + W.db^M),  dv' = dv + h (da + U.db^M),  da' = J' (dx', dv') + jp'
// where J_j (3 x 6) and jp_j (3 x 2) are the Jacobians of the force (dual numbers,
// tangent.cuh) at node j's point of the attempt's last corrector iteration, for all M
// iterations (the corrector has converged there to 1e-14 of |a| in b6), as the discrete
// adjoint takes them -- evaluated in that iteration's round, while the lane's body cache
// holds the node's time; J' is taken at the accepted state.  Lane j < 7 owns node j + 1 and its
// Jacobian; lane p updates direction p of db and of the state tangents; all tangents of a
// group live in shared memory.  The one-object-per-thread form (nbody_stm_kernel) takes every
// iteration's Jacobian at that iteration's own points; the two agree to about 1e-8 relative.
#pragma once
#include "adjoint.cuh"
#include "common.cuh"
#include "forces.cuh"
#include "internal.h"
#include "radau.cuh"
#include "tangent.cuh"

namespace kb {

constexpr int STM_BLOCK = SENS_BLOCK;   // 16 groups of 8 lanes
constexpr int STM_GROUPS = STM_BLOCK / SG;
// Tangent doubles per group in dynamic shared memory: dx, dv, da (3 x 8 each), db (3 x 8
// rows of 7 coefficients) and the node tangents dE (7 x 3 x 8).
constexpr int STM_DX = 0, STM_DV = 24, STM_DA = 48, STM_DB = 72, STM_DE = 240, STM_ROW = 408;
constexpr int STM_DYN_SMEM = STM_GROUPS * STM_ROW * (int)sizeof(double);

struct StmNodesPolicy {
    const StmArgs* a;
    int64_t obj;
    int lane;
    int k;  // epoch segment being integrated
    unsigned gmask;
    double* sb;         // the group's b (21)
    double* ts;         // the group's tangent row (STM_ROW doubles)
    const double* nrow;  // the lane's node row (w_pow, u_pow, spacing, frac2)
    TangentForce* T;
    EphCache* C;
    double R[3][3];     // d(equatorial) / d(caller frame)

    // J (3 x 6) and jp (3 x 2) at a point; false when the evaluation fails
    __device__ bool jacobian(double t, const double x[3], const double v[3], double J[18],
                             double jp[6]) {
        return sens_jacobian(*T, t, x, v, J, jp, *C) == ST_OK;
    }

    // da = J (dx, dv) + jp for direction p = lane (J, jp given in every lane)
    __device__ void tangent_acc(const double J[18], const double jp[6]) {
        const int p = lane;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < 3; ++i)
                s += J[6 * c + i] * ts[STM_DX + 8 * i + p] + J[6 * c + 3 + i] * ts[STM_DV + 8 * i + p];
            if (p == 6) s += jp[2 * c];
            if (p == 7) s += jp[2 * c + 1];
            ts[STM_DA + 8 * c + p] = s;
        }
    }

    __device__ bool begin_attempt(SensGroup& G) {
        if (G.att == 0) {  // a fresh integration: db = 0 and da at the start
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int kk = 0; kk < 7; ++kk) ts[STM_DB + (8 * c + lane) * 7 + kk] = 0.0;
            double J[18], jp[6];
            const bool ok = jacobian(G.t, G.x, G.v, J, jp);
            __syncwarp(gmask);
            if (!__all_sync(gmask, ok)) {
                G.rc = ST_DAF_LIMITS;
                G.phase = SP_DONE;
                return false;
            }
            tangent_acc(J, jp);
        }
        __syncwarp(gmask);
        return true;
    }

    __device__ void attempt_predict(double q) {
        if (q == 0.0) return;
        // db^0 = S(q) db: the predictor applied to every (component, direction) row
#pragma unroll
        for (int c = 0; c < 3; ++c) predict_b_row(ts + STM_DB + (8 * c + lane) * 7, q);
        __syncwarp(gmask);
    }

    __device__ void iter_round(SensGroup&, double*, int) {}

    // node j's Jacobian at its point of the attempt's last corrector iteration, while the
    // lane's body cache still holds the node's time (kept in registers until end_attempt)
    double Jl[18], jpl[6];
    bool jl_ok;
    __device__ void last_iteration(SensGroup&, double te, const double* xe, const double* ve,
                                   int ln) {
        jl_ok = true;
        if (ln < 7) jl_ok = jacobian(te, xe, ve, Jl, jpl);
    }

    __device__ void end_attempt(SensGroup& G, bool converged) {
        __syncwarp(gmask);
        const double h = G.h, h2 = h * h;
        // node Jacobians at the last corrector iteration's points (lanes 0-6, taken in that
        // round) and, after an accepted step, the Jacobian at the new state (lane 7)
        double J[18], jp[6];
#pragma unroll
        for (int i = 0; i < 18; ++i) J[i] = Jl[i];
#pragma unroll
        for (int i = 0; i < 6; ++i) jp[i] = jpl[i];
        bool ok = jl_ok;
        if (lane == 7 && converged) ok = jacobian(G.t, G.x, G.v, J, jp);
        if (!__all_sync(gmask, ok)) {
            G.rc = ST_DAF_LIMITS;
            G.phase = SP_DONE;
            return;
        }
        if (lane == 7 && converged) {  // lane 7 publishes J' (in the dE area, free until used)
#pragma unroll
            for (int i = 0; i < 18; ++i) ts[STM_DE + i] = J[i];
#pragma unroll
            for (int i = 0; i < 6; ++i) ts[STM_DE + 18 + i] = jp[i];
        }
        __syncwarp(gmask);
        double Jn[18], jpn[6];  // J' in every lane, read before the dE area is reused
        if (converged) {
#pragma unroll
            for (int i = 0; i < 18; ++i) Jn[i] = ts[STM_DE + i];
#pragma unroll
            for (int i = 0; i < 6; ++i) jpn[i] = ts[STM_DE + 18 + i];
        }
        __syncwarp(gmask);
        // the M corrector iterations, linearised
        const int M = G.iter;
        for (int m = 0; m < M; ++m) {
            if (lane < 7) {
                const double f = nrow[14], frac2 = nrow[15];
#pragma unroll 1
                for (int p = 0; p < 8; ++p) {
                    double dX[3], dV[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const double* row = ts + STM_DB + (8 * c + p) * 7;
                        double bw = 0.0, bu = 0.0;
#pragma unroll
                        for (int kk = 0; kk < 7; ++kk) {
                            bw += nrow[kk] * row[kk];
                            bu += nrow[7 + kk] * row[kk];
                        }
                        const double dx = ts[STM_DX + 8 * c + p], dv = ts[STM_DV + 8 * c + p],
                                     da = ts[STM_DA + 8 * c + p];
                        dX[c] = dx + f * dv * h + frac2 * h2 * (da / 2.0 + bw);
                        dV[c] = dv + f * h * (da + bu);
                    }
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double s = 0.0;
#pragma unroll
                        for (int i = 0; i < 3; ++i) s += J[6 * c + i] * dX[i] + J[6 * c + 3 + i] * dV[i];
                        if (p == 6) s += jp[2 * c];
                        if (p == 7) s += jp[2 * c + 1];
                        ts[STM_DE + (lane * 3 + c) * 8 + p] = s;
                    }
                }
            }
            __syncwarp(gmask);
            {  // db = P (dE - da), direction p = lane
                const int p = lane;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const double da = ts[STM_DA + 8 * c + p];
                    double e[7];
#pragma unroll
                    for (int j = 0; j < 7; ++j) e[j] = ts[STM_DE + (j * 3 + c) * 8 + p] - da;
#pragma unroll
                    for (int kk = 0; kk < 7; ++kk) {
                        double s = 0.0;
#pragma unroll
                        for (int j = 0; j < 7; ++j) s += c_tab.adj_p[kk][j] * e[j];
                        ts[STM_DB + (8 * c + p) * 7 + kk] = s;
                    }
                }
            }
            __syncwarp(gmask);
        }
        if (!converged) return;  // a failed attempt keeps the state; its b carries on
        // state tangents of the accepted step, direction p = lane
        {
            const int p = lane;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double* row = ts + STM_DB + (8 * c + p) * 7;
                double dw = 0.0, du = 0.0;
#pragma unroll
                for (int kk = 0; kk < 7; ++kk) {
                    dw += row[kk] * c_tab.w[kk];
                    du += row[kk] * c_tab.u[kk];
                }
                const double dx = ts[STM_DX + 8 * c + p], dv = ts[STM_DV + 8 * c + p],
                             da = ts[STM_DA + 8 * c + p];
                ts[STM_DX + 8 * c + p] = dx + dv * h + h2 * (da * 0.5 + dw);
                ts[STM_DV + 8 * c + p] = dv + h * (da + du);
            }
        }
        // da' from the Jacobian at the accepted state
        tangent_acc(Jn, jpn);
        __syncwarp(gmask);
    }

    __device__ void segment_end(SensGroup& G) {
        const int64_t n = a->n;
        if (lane == 0) {
            double px[3] = {G.x[0], G.x[1], G.x[2]}, pv[3] = {G.v[0], G.v[1], G.v[2]};
            const int orc = from_ssb_equatorial(G.tf, a->frame, a->chain, px, pv);
            double* st = a->out_state + (int64_t)k * 6 * n;
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                st[c * n + obj] = orc == ST_OK ? px[c] : nan;
                st[(3 + c) * n + obj] = orc == ST_OK ? pv[c] : nan;
            }
            if (orc != ST_OK) G.rc = orc;
        }
        G.rc = __shfl_sync(gmask, G.rc, 0, SG);
        {  // column p = lane of the 6 x 8 matrix, back in the caller's frame: R^T d(state)
            const int p = lane;
            double* phi = a->out_stm + (int64_t)k * 48 * n;
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double sx = 0.0, sv = 0.0;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    sx += R[q][c] * ts[STM_DX + 8 * q + p];
                    sv += R[q][c] * ts[STM_DV + 8 * q + p];
                }
                phi[(c * TAN_DIRS + p) * n + obj] = G.rc == ST_OK ? sx : nan;
                phi[((3 + c) * TAN_DIRS + p) * n + obj] = G.rc == ST_OK ? sv : nan;
            }
        }
        if (G.rc != ST_OK || ++k >= a->n_epochs) {
            G.phase = SP_DONE;
            return;
        }
        G.tf = a->epochs[k];
        if (lane < 7) {  // b restarts at zero in every fresh integration (and db with it)
            sb[lane] = 0.0;
            sb[7 + lane] = 0.0;
            sb[14 + lane] = 0.0;
        }
        __syncwarp(gmask);
        G.phase = SP_EXACT_INIT;
    }
};

template <int MINB>
__global__ void __launch_bounds__(STM_BLOCK, MINB) nbody_stm_nodes_kernel(StmArgs a) {
    extern __shared__ double s_tan[];  // STM_ROW doubles per group
    __shared__ double s_node[8 * NODE_ROW_S];
    __shared__ double s_b[STM_GROUPS][21];
    __shared__ double s_e[STM_GROUPS][SG * 3];
    __shared__ double s_cache[EPH_CACHE * STM_BLOCK];  // per-lane body positions
    sens_load_nodes(s_node);
    __syncthreads();
    const int lane = threadIdx.x & (SG - 1);
    const int warp_lane = threadIdx.x & 31;
    const unsigned gmask = 0xFFu << (warp_lane & ~(SG - 1));
    const int64_t obj = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / SG;
    if (obj >= a.n) return;
    double* sb = s_b[threadIdx.x / SG];
    double* se = s_e[threadIdx.x / SG];
    double* ts = s_tan + (threadIdx.x / SG) * STM_ROW;
    const int comp = lane % 3;
    const double* nrow = s_node + (lane < 7 ? lane + 1 : 7) * NODE_ROW_S;
    const int64_t n = a.n;

    SensGroup G;
    G.t = a.jd0[obj];
    G.tf = a.epochs[0];
    G.x[0] = a.pos[obj]; G.x[1] = a.pos[n + obj]; G.x[2] = a.pos[2 * n + obj];
    G.v[0] = a.vel[obj]; G.v[1] = a.vel[n + obj]; G.v[2] = a.vel[2 * n + obj];
    G.h = G.next_h = G.h_prev = 0.0;
    G.predict = false;
    G.acc[0] = G.acc[1] = G.acc[2] = 0.0;
    G.iter = G.failures = G.att = 0;
    G.rc = ST_OK;
    if (lane < 7) {
        sb[lane] = 0.0;
        sb[7 + lane] = 0.0;
        sb[14 + lane] = 0.0;
    }
    SpkForce F;
    F.n_force = a.n_force;
    F.ng.base = a.nongrav ? a.nongrav + obj : nullptr;
    F.ng.stride = n;
    F.ng.kind = a.nongrav ? (int)a.nongrav[obj] : 0;
    F.impact_id = 0;
    F.min_dist = 1e300;
    F.min_id = 0;
    TangentForce T;
    T.n_force = a.n_force;
    T.ng = F.ng;
    T.impact_id = 0;
    T.min_dist = 1e300;
    if (!(isfinite(G.x[0]) && isfinite(G.x[1]) && isfinite(G.x[2]) && isfinite(G.v[0]) &&
          isfinite(G.v[1]) && isfinite(G.v[2]) && isfinite(G.t)))
        G.rc = ST_VALUE_ERROR;
    // the derivative of the comet model is taken with its time delay dt = 0
    if (F.ng.kind == 1 && F.ng.p(9) != 0.0) G.rc = ST_VALUE_ERROR;
    if (G.rc == ST_OK) G.rc = to_ssb_equatorial(G.t, a.frame, a.chain, G.x, G.v);
    const FastPlan& plan = a.n_force == c_eph.n_force_planets ? c_eph.fast_planets : c_eph.fast_all;
    EphCache C{s_cache + threadIdx.x, STM_BLOCK,
               plan.ok && SpkForce::cached_doubles(plan) <= EPH_CACHE,
               __longlong_as_double(0x7ff8000000000000LL)};
    StmNodesPolicy P;
    P.a = &a;
    P.obj = obj;
    P.lane = lane;
    P.k = 0;
    P.gmask = gmask;
    P.sb = sb;
    P.ts = ts;
    P.nrow = nrow;
    P.T = &T;
    P.C = &C;
    P.jl_ok = true;
    sens_rotation(a.frame, P.R);
    {  // tangents of the initial state: d(equatorial state) / d(caller's state), A1, A2
        const int p = lane;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ts[STM_DX + 8 * c + p] = p < 3 ? P.R[c][p] : 0.0;
            ts[STM_DV + 8 * c + p] = (p >= 3 && p < 6) ? P.R[c][p - 3] : 0.0;
        }
    }
    __syncwarp(gmask);
    G.phase = G.rc == ST_OK ? SP_EXACT_INIT : SP_DONE;
    const int max_rounds = a.max_loops * 12;
    sens_rounds(G, F, P, nrow, sb, se, lane, comp, gmask, warp_lane, max_rounds, C);
    if (lane == 0) a.status[obj] = G.rc;
    if (G.rc != ST_OK) {  // epochs not reached are NaN
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        for (int kk = P.k; kk < a.n_epochs; ++kk) {
            if (lane < 6) a.out_state[((int64_t)kk * 6 + lane) * n + obj] = nan;
            for (int r = 0; r < 6; ++r) a.out_stm[((int64_t)kk * 48 + r * TAN_DIRS + lane) * n + obj] = nan;
        }
    }
}

}  // namespace kb
