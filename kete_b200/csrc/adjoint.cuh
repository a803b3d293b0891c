// adjoint.cuh -- reverse-mode gradients of the N-body propagation: a discrete adjoint of
// the executed Gauss-Radau steps with checkpoints and recomputation between them.
//
// Forward (nbody_sens_forward_kernel): every object is integrated by a group of 8 lanes
// with the seven corrector nodes in parallel (as in radau_nodes.cuh, the exact evaluation
// at the updated state in a round of its own, radau.rs:331-338) through n_epochs epochs.
// Each epoch is a fresh integration from the previous one, as consecutive
// propagate_n_body_spk calls are (kete_core/propagation/mod.rs:70-118).  Before every 16th
// step attempt of an epoch segment the group stores a checkpoint: t, h, failures, x, v, a,
// the b carried into the attempt and, after an accepted step, the step size the predicted
// b is scaled from (predict_b_row, radau.cuh).
//
// Backward (nbody_sens_backward_kernel): the segments and their checkpoint blocks are taken
// in reverse.  A block is re-run from its checkpoint with the same step code, recording for
// every attempt its start state, the step size used, its iteration count and the b of its
// last corrector iteration.  The attempts are then transposed, last first.  For one attempt
// with M iterations (step size and iteration count held fixed):
//   x' = x + h v + h^2 (a/2 + W.b^M),  v' = v + h (a + U.b^M),  a' = F(x', v')
//   b^m = P (E^m - a),  E^m_j = F(X_j(b^(m-1)), V_j(b^(m-1))),  P = C_MAT . (divided differences)
//   b^0 = S(q) b^M of the previous attempt (the predictor, q = h / h_prev; identity after a
//   failed attempt, zero at the start of a segment)
//   X_j = x + f_j h v + f_j^2 h^2 (a/2 + W_j.b),  V_j = v + f_j h (a + U_j.b)
// The adjoint runs the M iterations backwards with each node's Jacobian taken at the points
// of the attempt's last iteration (the corrector has converged there to 1e-14 of |a| in
// b6, so the earlier iterations' points differ by the iteration's own convergence).  Lane
// j < 7 owns node j+1 and its 3 x 8 Jacobian (dual numbers, tangent.cuh); lane 7 owns the
// step-end evaluation a' = F(x', v').  The adjoint of b moves through shared memory.
#pragma once
#include "common.cuh"
#include "forces.cuh"
#include "radau.cuh"
#include "internal.h"
#include "tangent.cuh"

namespace kb {

constexpr int SENS_BLOCK = 128;
constexpr int SG = 8;  // lanes per object

enum SensPhase : int { SP_BEGIN = 0, SP_EXACT_INIT = 1, SP_ITER = 2, SP_EXACT_STEP = 3, SP_PAUSE = 4, SP_DONE = 5 };

// Checkpoint and attempt-record layout (SENS_STRIDE doubles each):
//   [0] t  [1] h (checkpoint: proposed; record: used)  [2] failures / iterations
//   [3] record: 1 if the attempt converged  [4..6] x  [7..9] v  [10..12] a  [13..33] b
//   [34] checkpoint: the previous step's h when b is to be predicted, else 0;
//        record: the predictor's scale q used at the attempt's start, else 0
static_assert(SENS_STRIDE == 36, "checkpoint layout");

struct SensGroup {  // one object's integration state, identical in every lane of its group
    double t, tf, h, next_h, h_prev;
    double x[3], v[3], acc[3];
    int iter, failures, phase, att, rc;
    bool predict;  // the next attempt starts from the predicted b
};

__device__ __forceinline__ double group_sum(double v, unsigned gmask) {
    v += __shfl_xor_sync(gmask, v, 4, SG);
    v += __shfl_xor_sync(gmask, v, 2, SG);
    v += __shfl_xor_sync(gmask, v, 1, SG);
    return v;
}

// Write the group's state (and its b, from shared memory) to one checkpoint / record slot.
__device__ __forceinline__ void sens_store_state(double* dst, const SensGroup& G, const double* sb,
                                                 int lane, double w2) {
    if (lane == 0) {
        dst[0] = G.t;
        dst[1] = G.h;
        dst[2] = w2;
        dst[34] = G.predict ? G.h_prev : 0.0;
    } else if (lane == 1) {
        dst[4] = G.x[0]; dst[5] = G.x[1]; dst[6] = G.x[2];
    } else if (lane == 2) {
        dst[7] = G.v[0]; dst[8] = G.v[1]; dst[9] = G.v[2];
    } else if (lane == 3) {
        dst[10] = G.acc[0]; dst[11] = G.acc[1]; dst[12] = G.acc[2];
    }
    if (lane < 7) {
        dst[13 + lane] = sb[lane];
        dst[20 + lane] = sb[7 + lane];
        dst[27 + lane] = sb[14 + lane];
    }
}

// The step loop of RadauIntegrator::integrate / step (radau.rs:160-346) in rounds: every
// round each lane evaluates one point (a corrector node, or the exact evaluation).  The
// policy's hooks see every attempt begin and end, every corrector round and the end of
// the segment.  Returns when the group is done, paused by the policy or failed.
template <class Policy>
__device__ __forceinline__ void sens_rounds(SensGroup& G, SpkForce& F, Policy& P,
                                            const double* nrow, double* sb, double* se, int lane,
                                            int comp, unsigned gmask, int warp_lane,
                                            int max_rounds, EphCache& C) {
    const FastPlan& plan = F.n_force == c_eph.n_force_planets ? c_eph.fast_planets : c_eph.fast_all;
    for (int rounds = 0;; ++rounds) {
        if (G.phase == SP_BEGIN) {  // MIN_STEP, then truncate to the end (radau.rs:187-190,214-216)
            if (!P.begin_attempt(G)) {
                G.phase = SP_PAUSE;
                return;
            }
            if (fabs(G.h) < 0.005) G.h = copysign(0.005, G.h);
            if (fabs(G.t - G.tf) <= fabs(G.h)) G.h = G.tf - G.t;
            double q = 0.0;
            if (G.predict) {
                q = G.h / G.h_prev;
                if (lane < 3) predict_b_row(sb + 7 * lane, q);
                __syncwarp(gmask);
            }
            P.attempt_predict(q);
            G.iter = 0;
            G.att++;
            G.phase = SP_ITER;
        }
        if (G.phase != SP_ITER && G.phase != SP_EXACT_INIT && G.phase != SP_EXACT_STEP) return;
        if (rounds >= max_rounds) {
            G.rc = ST_TIMEOUT;
            G.phase = SP_DONE;
            return;
        }
        const bool iter_round = G.phase == SP_ITER;
        double te, xe[3], ve[3];
        if (!iter_round) {
            te = G.t;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                xe[c] = G.x[c];
                ve[c] = G.v[c];
            }
        } else {
            P.iter_round(G, sb, lane);
            const double f = nrow[14], frac2 = nrow[15];
            const double h2 = G.h * G.h;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double bw = 0.0, bu = 0.0;
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    const double bck = sb[7 * c + k];
                    bw += nrow[k] * bck;
                    bu += nrow[7 + k] * bck;
                }
                xe[c] = G.x[c] + f * G.v[c] * G.h + frac2 * h2 * (G.acc[c] / 2.0 + bw);
                ve[c] = G.v[c] + f * G.h * (G.acc[c] + bu);
            }
            te = G.t + f * G.h;
        }
        double ev[3];
        int erc;
        // the corrector iterations of an attempt share their node times: the bodies'
        // positions come from the lane's cache after the first
        if (C.on && te >= plan.lo && te <= plan.hi) {
            if (te != C.t) {
                SpkForce::fast_positions(plan, te, C.p, C.stride);
                C.t = te;
            }
            erc = F.fast_forces(plan, !iter_round, xe, ve, C.p, C.stride, ev);
        } else {
            erc = F.eval(!iter_round, te, xe, ve, ev);
        }
        const unsigned bad = __ballot_sync(gmask, erc != ST_OK);
        if (bad) {
            const int src = __ffs(bad) - 1 - (warp_lane & ~(SG - 1));
            G.rc = __shfl_sync(gmask, erc, src, SG);
            G.phase = SP_DONE;
            return;
        }
        if (!iter_round) {
            G.acc[0] = ev[0];
            G.acc[1] = ev[1];
            G.acc[2] = ev[2];
            if (G.phase == SP_EXACT_INIT) {
                if (fabs(G.tf - G.t) < 1e-10) {
                    P.segment_end(G);
                    continue;
                }
                G.h = copysign(0.1, G.tf - G.t);
                G.failures = 0;
                G.att = 0;
                G.predict = false;
            } else {
                P.end_attempt(G, true);
                if (G.phase == SP_DONE) return;  // the policy failed the object
                G.h_prev = G.h;
                G.predict = true;
                G.h = G.next_h;
                if (fabs(G.t - G.tf) < 1e-12) {
                    P.segment_end(G);
                    continue;
                }
                G.failures = 0;
            }
            G.phase = SP_BEGIN;
            continue;
        }
        // corrector iteration (radau.rs:292-330): lanes 0-2 form g and b for one component
        se[3 * lane + 0] = ev[0];
        se[3 * lane + 1] = ev[1];
        se[3 * lane + 2] = ev[2];
        const double b6_old0 = sb[6], b6_old1 = sb[13], b6_old2 = sb[20];
        __syncwarp(gmask);
        {
            const double ac = comp == 0 ? G.acc[0] : (comp == 1 ? G.acc[1] : G.acc[2]);
            double g[7];
#pragma unroll
            for (int j = 1; j < 8; ++j) {
                double gk = (se[3 * (j - 1) + comp] - ac) * c_tab.inv_frac[j];
#pragma unroll
                for (int z = 1; z < j; ++z) gk = (gk - g[z - 1]) * c_tab.inv_diff[j][z];
                g[j - 1] = gk;
            }
            if (lane < 3) {
#pragma unroll
                for (int jj = 0; jj < 7; ++jj) {
                    double s2 = g[jj];
#pragma unroll
                    for (int k = jj + 1; k < 7; ++k) s2 += c_tab.c[k][jj] * g[k];
                    sb[7 * comp + jj] = s2;
                }
            }
        }
        __syncwarp(gmask);
        const double e70 = se[18], e71 = se[19], e72 = se[20];
        const double fem0 = fabs(e70) + 1e-6, fem1 = fabs(e71) + 1e-6, fem2 = fabs(e72) + 1e-6;
        const double b60 = sb[6], b61 = sb[13], b62 = sb[20];
        const double ratio = fmax(fmax(fabs(b60 - b6_old0) / fem0, fabs(b61 - b6_old1) / fem1),
                                  fabs(b62 - b6_old2) / fem2);
        ++G.iter;
        // the policy sees the points of an attempt's last iteration (converged or not)
        if (ratio < 1e-14 || G.iter >= 10) P.last_iteration(G, te, xe, ve, lane);
        if (ratio < 1e-14) {
            const double h2 = G.h * G.h;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double dw = 0.0, du = 0.0;
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    const double bck = sb[7 * c + k];
                    dw += bck * c_tab.w[k];
                    du += bck * c_tab.u[k];
                }
                G.x[c] += G.v[c] * G.h + h2 * (G.acc[c] * 0.5 + dw);
                G.v[c] += G.h * (G.acc[c] + du);
            }
            G.t += G.h;
            const double mb6 = fmax(fmax(fabs(b60), fabs(b61)), fabs(b62));
            const double r = pow(1e-6 * fmax(fmax(fem0, fem1), fem2) / mb6, 1.0 / 7.0);
            G.next_h = G.h * clampd(r, 0.25, 4.0);
            G.phase = SP_EXACT_STEP;
            __syncwarp(gmask);
            continue;
        }
        __syncwarp(gmask);
        if (G.iter >= 10) {  // not converged: retry with a smaller step (radau.rs:199-210)
            P.end_attempt(G, false);
            if (G.phase == SP_DONE) return;  // the policy failed the object
            G.predict = false;
            G.failures += 1;
            G.h *= 0.7;
            if (G.failures > 10) {
                G.rc = ST_CONVERGENCE;
                G.phase = SP_DONE;
                return;
            }
            G.phase = SP_BEGIN;
        }
    }
}

// Shared-memory node table (as in nbody_nodes_kernel): per node j, w_pow[j][0..6],
// u_pow[j][0..6], spacing, frac2, padded to NODE_ROW_S doubles.
constexpr int NODE_ROW_S = 17;
__device__ __forceinline__ void sens_load_nodes(double* s_node) {
    for (int i = threadIdx.x; i < 8 * NODE_ROW_S; i += blockDim.x) {
        const int j = i / NODE_ROW_S, k = i % NODE_ROW_S;
        double val = 0.0;
        if (k < 7) val = c_tab.w_pow[j][k];
        else if (k < 14) val = c_tab.u_pow[j][k - 7];
        else if (k == 14) val = c_tab.spacing[j];
        else if (k == 15) val = c_tab.frac2[j];
        s_node[i] = val;
    }
}

__device__ __forceinline__ void sens_rotation(int frame, double R[3][3]) {
    // d(equatorial)/d(caller frame)
    R[0][0] = 1; R[0][1] = 0; R[0][2] = 0;
    R[1][0] = 0; R[1][1] = 1; R[1][2] = 0;
    R[2][0] = 0; R[2][1] = 0; R[2][2] = 1;
    if (frame == FRAME_ECLIPTIC) {
        const double c = c_tab.rot_c, s = c_tab.rot_s;
        R[1][1] = c; R[1][2] = -s; R[2][1] = s; R[2][2] = c;
    }
}

// ---------------------------------------------------------------------------------------
// forward with checkpoints
// ---------------------------------------------------------------------------------------
struct SensForwardPolicy {
    const SensArgs* a;
    int64_t obj;
    int lane;
    int k;    // epoch segment being integrated
    int nck;  // checkpoints taken (stored while below capacity)
    unsigned gmask;
    double* sb;

    __device__ bool begin_attempt(SensGroup& G) {
        if (G.att % SENS_CK_ATTEMPTS == 0) {
            if (nck < a->ckpt_cap)
                sens_store_state(a->ckpt + ((size_t)obj * a->ckpt_cap + nck) * SENS_STRIDE, G, sb,
                                 lane, (double)G.failures);
            nck++;
        }
        return true;
    }
    __device__ void attempt_predict(double) {}
    __device__ void iter_round(SensGroup&, double*, int) {}
    __device__ void last_iteration(SensGroup&, double, const double*, const double*, int) {}
    __device__ void end_attempt(SensGroup&, bool) {}
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
        if (G.rc != ST_OK) {
            G.phase = SP_DONE;
            return;
        }
        if (++k >= a->n_epochs) {
            G.phase = SP_DONE;
            return;
        }
        if (lane == 0) a->ckpt_seg[(int64_t)k * n + obj] = nck;
        G.tf = a->epochs[k];
        if (lane < 7) {  // b restarts at zero in every fresh integration
            sb[lane] = 0.0;
            sb[7 + lane] = 0.0;
            sb[14 + lane] = 0.0;
        }
        __syncwarp(gmask);
        G.phase = SP_EXACT_INIT;
    }
};

template <int MINB>
__global__ void __launch_bounds__(SENS_BLOCK, MINB) nbody_sens_forward_kernel(SensArgs a) {
    __shared__ double s_node[8 * NODE_ROW_S];
    __shared__ double s_b[SENS_BLOCK / SG][21];
    __shared__ double s_e[SENS_BLOCK / SG][SG * 3];
    __shared__ double s_cache[EPH_CACHE * SENS_BLOCK];  // per-lane body positions
    sens_load_nodes(s_node);
    __syncthreads();
    const int lane = threadIdx.x & (SG - 1);
    const int warp_lane = threadIdx.x & 31;
    const unsigned gmask = 0xFFu << (warp_lane & ~(SG - 1));
    const int64_t obj = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / SG;
    if (obj >= a.n) return;
    double* sb = s_b[threadIdx.x / SG];
    double* se = s_e[threadIdx.x / SG];
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
    if (!(isfinite(G.x[0]) && isfinite(G.x[1]) && isfinite(G.x[2]) && isfinite(G.v[0]) &&
          isfinite(G.v[1]) && isfinite(G.v[2]) && isfinite(G.t)))
        G.rc = ST_VALUE_ERROR;
    // the derivative of the comet model is taken with its time delay dt = 0
    if (F.ng.kind == 1 && F.ng.p(9) != 0.0) G.rc = ST_VALUE_ERROR;
    if (G.rc == ST_OK) G.rc = to_ssb_equatorial(G.t, a.frame, a.chain, G.x, G.v);
    SensForwardPolicy P{&a, obj, lane, 0, 0, gmask, sb};
    if (lane == 0) a.ckpt_seg[obj] = 0;
    __syncwarp(gmask);
    G.phase = G.rc == ST_OK ? SP_EXACT_INIT : SP_DONE;
    const int max_rounds = a.max_loops * 12;
    const FastPlan& plan = a.n_force == c_eph.n_force_planets ? c_eph.fast_planets : c_eph.fast_all;
    EphCache C{s_cache + threadIdx.x, SENS_BLOCK,
               plan.ok && SpkForce::cached_doubles(plan) <= EPH_CACHE,
               __longlong_as_double(0x7ff8000000000000LL)};
    sens_rounds(G, F, P, nrow, sb, se, lane, comp, gmask, warp_lane, max_rounds, C);
    if (lane == 0) {
        int rc = G.rc;
        if (rc == ST_OK && P.nck > a.ckpt_cap) rc = ST_CHECKPOINT_FULL;
        a.status[obj] = rc;
        a.ckpt_count[obj] = P.nck;
        if (G.rc != ST_OK) {  // epochs not reached are NaN
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
            for (int k = P.k; k < a.n_epochs; ++k)
                for (int c = 0; c < 6; ++c) a.out_state[((int64_t)k * 6 + c) * n + obj] = nan;
            for (int k = P.k + 1; k < a.n_epochs; ++k) a.ckpt_seg[(int64_t)k * n + obj] = P.nck;
        }
    }
}

// ---------------------------------------------------------------------------------------
// backward: re-run each checkpoint block, then transpose its attempts
// ---------------------------------------------------------------------------------------
struct SensReplayPolicy {
    double* rec;  // SENS_CK_ATTEMPTS + 1 records
    int na;       // attempts recorded
    int lane;
    double* sb;

    __device__ bool begin_attempt(SensGroup& G) {
        sens_store_state(rec + (size_t)na * SENS_STRIDE, G, sb, lane, 0.0);
        if (na == SENS_CK_ATTEMPTS) return false;  // the block's end state is stored
        na++;
        return true;
    }
    __device__ void attempt_predict(double q) {
        if (lane == 0) rec[(size_t)(na - 1) * SENS_STRIDE + 34] = q;
    }
    __device__ void last_iteration(SensGroup&, double, const double*, const double*, int) {}
    __device__ void iter_round(SensGroup&, double* b, int ln) {  // b of the previous iterate
        double* d = rec + (size_t)(na - 1) * SENS_STRIDE;
        if (ln < 7) {
            d[13 + ln] = b[ln];
            d[20 + ln] = b[7 + ln];
            d[27 + ln] = b[14 + ln];
        }
    }
    __device__ void end_attempt(SensGroup& G, bool converged) {
        if (lane == 0) {
            double* d = rec + (size_t)(na - 1) * SENS_STRIDE;
            d[1] = G.h;
            d[2] = (double)G.iter;
            d[3] = converged ? 1.0 : 0.0;
        }
    }
    __device__ void segment_end(SensGroup& G) {
        sens_store_state(rec + (size_t)na * SENS_STRIDE, G, sb, lane, 0.0);
        G.phase = SP_PAUSE;
    }
};

// Jacobian of the force at one point (dual numbers): J (3 x 6) = d a / d(x, v) and
// jp (3 x 2) = d a / d(A1, A2).  Out of line: one copy serves every call site.
static __device__ __noinline__ int sens_jacobian(TangentForce& T, double t, const double* x,
                                          const double* v, double* J, double* jp, EphCache& C) {
    double xx[3] = {x[0], x[1], x[2]}, vv[3] = {v[0], v[1], v[2]};
    double ev[3], JJ[3][6], jj[3][2];
    const FastPlan& plan = T.n_force == c_eph.n_force_planets ? c_eph.fast_planets : c_eph.fast_all;
    const int rc = (C.on && t >= plan.lo && t <= plan.hi)
                       ? T.eval_cached(plan, C, t, xx, vv, ev, JJ, jj)
                       : T.eval(false, t, xx, vv, ev, JJ, jj);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 6; ++c) J[6 * r + c] = JJ[r][c];
        jp[2 * r] = jj[r][0];
        jp[2 * r + 1] = jj[r][1];
    }
    return rc;
}

// Re-run checkpoint block `c` (its segment ends at tf) with the step code, recording every
// attempt into rec (SENS_CK_ATTEMPTS + 1 records).  Returns ST_OK with the attempt count in na,
// or the failure.
__device__ __forceinline__ int sens_replay_block(const double* c, double tf, double* rec,
                                                 SpkForce& F, const double* nrow, double* sb,
                                                 double* se, int lane, int comp, unsigned gmask,
                                                 int warp_lane, int max_rounds, EphCache& C,
                                                 int& na) {
    SensGroup G;
    G.t = c[0];
    G.h = c[1];
    G.failures = (int)c[2];
    G.tf = tf;
    G.next_h = 0.0;
    G.h_prev = c[34];
    G.predict = c[34] != 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        G.x[q] = c[4 + q];
        G.v[q] = c[7 + q];
        G.acc[q] = c[10 + q];
    }
    G.iter = 0;
    G.att = 0;
    G.rc = ST_OK;
    if (lane < 7) {
        sb[lane] = c[13 + lane];
        sb[7 + lane] = c[20 + lane];
        sb[14 + lane] = c[27 + lane];
    }
    __syncwarp(gmask);
    G.phase = SP_BEGIN;
    SensReplayPolicy P{rec, 0, lane, sb};
    sens_rounds(G, F, P, nrow, sb, se, lane, comp, gmask, warp_lane, max_rounds, C);
    na = P.na;
    __syncwarp(gmask);  // the records are complete and visible to the group
    if (G.phase != SP_PAUSE) return G.rc != ST_OK ? G.rc : ST_TIMEOUT;
    return ST_OK;
}

// The replays of every checkpoint block of every object at once, before the adjoint sweep:
// a block's replay depends only on its checkpoint, so groups of 8 lanes re-run the blocks in
// parallel and store each block's attempt records (a.rec_all) and outcome (a.rep_count: the
// attempt count, or -1 - status on failure) for the sweep to read.  The grid is persistent:
// each group takes the next block from a queue (a.rep_first[n + 1]) in the dense order of
// a.rep_first (sens_replay_offsets_kernel), so groups that finish early take more blocks
// instead of leaving their thread block's other groups to run alone.
template <int MINB>
__global__ void __launch_bounds__(SENS_BLOCK, MINB) nbody_sens_replay_kernel(SensArgs a) {
    __shared__ double s_node[8 * NODE_ROW_S];
    __shared__ double s_b[SENS_BLOCK / SG][21];
    __shared__ double s_e[SENS_BLOCK / SG][SG * 3];
    sens_load_nodes(s_node);
    __syncthreads();
    const int lane = threadIdx.x & (SG - 1);
    const int warp_lane = threadIdx.x & 31;
    const unsigned gmask = 0xFFu << (warp_lane & ~(SG - 1));
    const int64_t n = a.n;
    const int64_t total = a.rep_first[n];
    int32_t* queue = a.rep_first + n + 1;
    double* sb = s_b[threadIdx.x / SG];
    double* se = s_e[threadIdx.x / SG];
    const int comp = lane % 3;
    const double* nrow = s_node + (lane < 7 ? lane + 1 : 7) * NODE_ROW_S;
    extern __shared__ double s_dyn[];
    const FastPlan& plan = a.n_force == c_eph.n_force_planets ? c_eph.fast_planets : c_eph.fast_all;
    for (;;) {
        int q = 0;
        if (lane == 0) q = atomicAdd(queue, 1);
        const int64_t idx = __shfl_sync(gmask, q, 0, SG);
        if (idx >= total) return;
        // the object holding block idx: the last o with rep_first[o] <= idx
        int64_t lo = 0, hi = n;  // rep_first[lo] <= idx < rep_first[hi]
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (a.rep_first[mid] <= idx) lo = mid;
            else hi = mid;
        }
        const int64_t obj = lo;
        const int cb = (int)(idx - a.rep_first[obj]);
        const int64_t item = obj * a.ckpt_cap + cb;  // the sweep's layout of records and counts
        int k = 0;  // the epoch segment holding block cb
        while (k + 1 < a.n_epochs && a.ckpt_seg[(int64_t)(k + 1) * n + obj] <= cb) ++k;
        SpkForce F;
        F.n_force = a.n_force;
        F.ng.base = a.nongrav ? a.nongrav + obj : nullptr;
        F.ng.stride = n;
        F.ng.kind = a.nongrav ? (int)a.nongrav[obj] : 0;
        F.impact_id = 0;
        F.min_dist = 1e300;
        F.min_id = 0;
        EphCache C{s_dyn + threadIdx.x, SENS_BLOCK,
                   plan.ok && SpkForce::cached_doubles(plan) <= EPH_CACHE,
                   __longlong_as_double(0x7ff8000000000000LL)};
        double* rec = a.rec_all + (size_t)item * (SENS_CK_ATTEMPTS + 1) * SENS_STRIDE;
        const double* c = a.ckpt + ((size_t)obj * a.ckpt_cap + cb) * SENS_STRIDE;
        int na = 0;
        const int rc = sens_replay_block(c, a.epochs[k], rec, F, nrow, sb, se, lane, comp, gmask,
                                         warp_lane, a.max_loops * 12, C, na);
        if (lane == 0) a.rep_count[item] = rc == ST_OK ? na : -1 - rc;
        __syncwarp(gmask);  // sb, se and the cache are reused by the group's next block
    }
}

// REPLAY: the sweep re-runs each block itself (the records did not fit the up-front replay's
// scratch); otherwise it reads the records nbody_sens_replay_kernel wrote, and carries no
// step code (a smaller kernel with fewer registers).
template <int MINB, bool REPLAY>
__global__ void __launch_bounds__(SENS_BLOCK, MINB) nbody_sens_backward_kernel(SensArgs a) {
    __shared__ double s_node[8 * NODE_ROW_S];
    __shared__ double s_P[49];
    __shared__ double s_b[SENS_BLOCK / SG][21];
    __shared__ double s_e[SENS_BLOCK / SG][SG * 3];
    __shared__ double s_lb[SENS_BLOCK / SG][21];
    __shared__ double s_t[SENS_BLOCK / SG][7 * 6];
    sens_load_nodes(s_node);
    for (int i = threadIdx.x; i < 49; i += blockDim.x) s_P[i] = c_tab.adj_p[i / 7][i % 7];
    __syncthreads();
    const int lane = threadIdx.x & (SG - 1);
    const int warp_lane = threadIdx.x & 31;
    const unsigned gmask = 0xFFu << (warp_lane & ~(SG - 1));
    const int64_t obj = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / SG;
    if (obj >= a.n) return;
    const int64_t n = a.n;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (a.status[obj] != ST_OK) {
        if (lane < 8) a.out_grad[(int64_t)lane * n + obj] = nan;
        return;
    }
    double* sb = s_b[threadIdx.x / SG];
    double* se = s_e[threadIdx.x / SG];
    double* slb = s_lb[threadIdx.x / SG];
    double* stx = s_t[threadIdx.x / SG];
    const int comp = lane % 3;
    const double* nrow = s_node + (lane < 7 ? lane + 1 : 7) * NODE_ROW_S;
    double* rec_own = a.rec + (size_t)obj * (SENS_CK_ATTEMPTS + 1) * SENS_STRIDE;
    const double* ck = a.ckpt + (size_t)obj * a.ckpt_cap * SENS_STRIDE;

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
    // per-lane body positions in dynamic shared memory (EPH_CACHE x SENS_BLOCK doubles,
    // launch_sens_backward), shared by the replay and the Jacobian rounds
    extern __shared__ double s_dyn[];
    const FastPlan& plan = a.n_force == c_eph.n_force_planets ? c_eph.fast_planets : c_eph.fast_all;
    EphCache C{s_dyn + threadIdx.x, SENS_BLOCK,
               plan.ok && SpkForce::cached_doubles(plan) <= EPH_CACHE,
               __longlong_as_double(0x7ff8000000000000LL)};

    double R[3][3];
    sens_rotation(a.frame, R);
    double lx[3] = {0, 0, 0}, lv[3] = {0, 0, 0}, la[3];
    double dA0 = 0.0, dA1 = 0.0;
    int fail = ST_OK;
    const int n_ck = a.ckpt_count[obj];
    const int max_rounds = a.max_loops * 12;

    for (int k = a.n_epochs - 1; k >= 0 && fail == ST_OK; --k) {
        // seed: dL/d(state at epoch k), caller frame -> integration frame (x_eq = R x)
        const double* sd = a.seed + (int64_t)k * 6 * n;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double sx = 0.0, sv = 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                sx += R[c][q] * sd[q * n + obj];
                sv += R[c][q] * sd[(3 + q) * n + obj];
            }
            lx[c] += sx;
            lv[c] += sv;
            la[c] = 0.0;  // the acceleration at the segment end feeds nothing
        }
        if (lane < 7) {  // b restarts at zero in the next segment: no adjoint flows back
            slb[lane] = 0.0;
            slb[7 + lane] = 0.0;
            slb[14 + lane] = 0.0;
        }
        __syncwarp(gmask);
        const int c0 = a.ckpt_seg[(int64_t)k * n + obj];
        const int c1 = k + 1 < a.n_epochs ? a.ckpt_seg[(int64_t)(k + 1) * n + obj] : n_ck;
        const double tf = a.epochs[k];
        for (int cb = c1 - 1; cb >= c0 && fail == ST_OK; --cb) {
            // ---- the block's attempt records: replayed up front, or re-run here ----
            const double* c = ck + (size_t)cb * SENS_STRIDE;
            int na = 0;
            double* rec = rec_own;
            if (!REPLAY) {
                const size_t item = (size_t)obj * a.ckpt_cap + cb;
                rec = a.rec_all + item * (SENS_CK_ATTEMPTS + 1) * SENS_STRIDE;
                const int cnt = a.rep_count[item];
                if (cnt < 0) {
                    fail = -1 - cnt;
                    break;
                }
                na = cnt;
            } else {
                const int rrc = sens_replay_block(c, tf, rec, F, nrow, sb, se, lane, comp, gmask,
                                                  warp_lane, max_rounds, C, na);
                if (rrc != ST_OK) {
                    fail = rrc;
                    break;
                }
            }
            // ---- transpose the attempts, last first ----
            for (int s = na - 1; s >= 0; --s) {
                const double* r0 = rec + (size_t)s * SENS_STRIDE;
                const double* r1 = r0 + SENS_STRIDE;
                const double t0 = r0[0], h = r0[1];
                const int M = (int)r0[2];
                const bool conv = r0[3] != 0.0;
                double te, xe[3], ve[3];
                if (lane < 7) {
                    const double f = nrow[14], frac2 = nrow[15], h2 = h * h;
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        double bw = 0.0, bu = 0.0;
#pragma unroll
                        for (int kk = 0; kk < 7; ++kk) {
                            const double bck = r0[13 + 7 * q + kk];
                            bw += nrow[kk] * bck;
                            bu += nrow[7 + kk] * bck;
                        }
                        xe[q] = r0[4 + q] + f * r0[7 + q] * h + frac2 * h2 * (r0[10 + q] / 2.0 + bw);
                        ve[q] = r0[7 + q] + f * h * (r0[10 + q] + bu);
                    }
                    te = t0 + f * h;
                } else {  // the step end x', v' (meaningful when the attempt converged)
                    te = r1[0];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        xe[q] = r1[4 + q];
                        ve[q] = r1[7 + q];
                    }
                }
                double J[18], jp[6];
                const int jrc = sens_jacobian(T, te, xe, ve, J, jp, C);
                const unsigned bad = __ballot_sync(gmask, jrc != ST_OK && (lane < 7 || conv));
                if (bad) {
                    fail = ST_DAF_LIMITS;
                    break;
                }
                if (conv) {
                    // a' = F(x', v'): lane 7 applies its Jacobian to the adjoint of a'
                    double dx[3] = {0, 0, 0}, dv[3] = {0, 0, 0};
                    if (lane == 7) {
#pragma unroll
                        for (int q = 0; q < 3; ++q)
#pragma unroll
                            for (int r = 0; r < 3; ++r) {
                                dx[q] += J[6 * r + q] * la[r];
                                dv[q] += J[6 * r + 3 + q] * la[r];
                            }
#pragma unroll
                        for (int r = 0; r < 3; ++r) {
                            dA0 += jp[2 * r] * la[r];
                            dA1 += jp[2 * r + 1] * la[r];
                        }
                    }
                    double lxp[3], lvp[3];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        lxp[q] = lx[q] + __shfl_sync(gmask, dx[q], 7, SG);
                        lvp[q] = lv[q] + __shfl_sync(gmask, dv[q], 7, SG);
                    }
                    // x' = x + h v + h^2 (a/2 + W.b),  v' = v + h (a + U.b)
                    if (lane < 7) {
                        const double wk = c_tab.w[lane], uk = c_tab.u[lane];
#pragma unroll
                        for (int q = 0; q < 3; ++q) slb[7 * q + lane] += h * h * wk * lxp[q] + h * uk * lvp[q];
                    }
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        lx[q] = lxp[q];
                        lv[q] = h * lxp[q] + lvp[q];
                        la[q] = 0.5 * h * h * lxp[q] + h * lvp[q];
                    }
                }
                __syncwarp(gmask);
                // ---- the M corrector iterations, last first ----
                double sx[3] = {0, 0, 0}, sv[3] = {0, 0, 0}, sa[3] = {0, 0, 0};
                const double f = nrow[14], F2h2 = nrow[15] * h * h, fh = f * h;
                for (int m = 0; m < M; ++m) {
                    if (lane < 7) {
                        double lE[3];
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            double s2 = 0.0;
#pragma unroll
                            for (int kk = 0; kk < 7; ++kk) s2 += s_P[7 * kk + lane] * slb[7 * q + kk];
                            lE[q] = s2;
                        }
                        double lX[3], lV[3];
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            lX[q] = J[q] * lE[0] + J[6 + q] * lE[1] + J[12 + q] * lE[2];
                            lV[q] = J[3 + q] * lE[0] + J[9 + q] * lE[1] + J[15 + q] * lE[2];
                        }
                        dA0 += jp[0] * lE[0] + jp[2] * lE[1] + jp[4] * lE[2];
                        dA1 += jp[1] * lE[0] + jp[3] * lE[1] + jp[5] * lE[2];
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            sx[q] += lX[q];
                            sv[q] += fh * lX[q] + lV[q];
                            sa[q] += 0.5 * F2h2 * lX[q] + fh * lV[q] - lE[q];
                            stx[6 * lane + q] = F2h2 * lX[q];
                            stx[6 * lane + 3 + q] = fh * lV[q];
                        }
                    }
                    __syncwarp(gmask);
                    // adjoint of the previous iterate's b: sum over the nodes' predictors
                    double nb[3];
#pragma unroll
                    for (int e = 0; e < 3; ++e) {
                        const int idx = lane + 8 * e;
                        double s2 = 0.0;
                        if (idx < 21) {
                            const int q = idx / 7, kk = idx % 7;
#pragma unroll
                            for (int j = 0; j < 7; ++j) {
                                const double* row = s_node + (j + 1) * NODE_ROW_S;
                                s2 += stx[6 * j + q] * row[kk] + stx[6 * j + 3 + q] * row[7 + kk];
                            }
                        }
                        nb[e] = s2;
                    }
                    __syncwarp(gmask);
#pragma unroll
                    for (int e = 0; e < 3; ++e) {
                        const int idx = lane + 8 * e;
                        if (idx < 21) slb[idx] = nb[e];
                    }
                    __syncwarp(gmask);
                }
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    lx[q] += group_sum(sx[q], gmask);
                    lv[q] += group_sum(sv[q], gmask);
                    la[q] += group_sum(sa[q], gmask);
                }
                // b^0 = S(q) b^M of the previous attempt when it was predicted
                const double qs = r0[34];
                if (qs != 0.0) {
                    if (lane < 3) predict_b_row_transposed(slb + 7 * lane, qs);
                    __syncwarp(gmask);
                }
            }
        }
        if (fail != ST_OK) break;
        // segment start: a = F(x, v) of the fresh integration (radau.rs:172-174)
        if (c1 > c0) {
            const double* c = ck + (size_t)c0 * SENS_STRIDE;
            double J[18], jp[6];
            const int jrc = sens_jacobian(T, c[0], c + 4, c + 7, J, jp, C);
            if (__any_sync(gmask, jrc != ST_OK)) {
                fail = ST_DAF_LIMITS;
                break;
            }
            double dx[3], dv[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                dx[q] = J[q] * la[0] + J[6 + q] * la[1] + J[12 + q] * la[2];
                dv[q] = J[3 + q] * la[0] + J[9 + q] * la[1] + J[15 + q] * la[2];
            }
            if (lane == 0) {
                dA0 += jp[0] * la[0] + jp[2] * la[1] + jp[4] * la[2];
                dA1 += jp[1] * la[0] + jp[3] * la[1] + jp[5] * la[2];
            }
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                lx[q] += dx[q];
                lv[q] += dv[q];
            }
        }
    }
    dA0 = group_sum(dA0, gmask);
    dA1 = group_sum(dA1, gmask);
    if (lane == 0) {
        double* g = a.out_grad;
        // back to the caller's frame: d/d(x_caller) = R^T d/d(x_eq)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double gx = 0.0, gv = 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                gx += R[q][c] * lx[q];
                gv += R[q][c] * lv[q];
            }
            g[(int64_t)c * n + obj] = fail == ST_OK ? gx : nan;
            g[(int64_t)(3 + c) * n + obj] = fail == ST_OK ? gv : nan;
        }
        g[6 * n + obj] = fail == ST_OK ? dA0 : nan;
        g[7 * n + obj] = fail == ST_OK ? dA1 : nan;
        if (a.grad_status) a.grad_status[obj] = fail;
    }
}

}  // namespace kb
