// radau_nodes.cuh -- Gauss-Radau 15 with the seven node evaluations of a corrector
// iteration running in parallel lanes.
//
// In kete's step (kete_core/propagation/radau.rs:231-344) the predictor for every node uses
// the b of the previous iteration; b is recomputed from the seven new evaluations only after
// all of them (radau.rs:313).  The seven force evaluations of one iteration are therefore
// independent, so a group of 8 lanes integrates one object: lane l evaluates node l+1 (lane 7
// repeats node 7), then the group exchanges the evaluations with warp shuffles and every
// lane forms the same g, b and convergence decision.  The exact evaluation after an accepted
// step is evaluated by all 8 lanes at the same point.
//
// The loop is organised in rounds with a single force-evaluation call site, so groups of a
// warp that are in different phases (corrector iteration / exact evaluation) still share the
// expensive instruction stream.  The arithmetic of each step is the reference's, except
// that divisions by node spacings use tabulated reciprocals, multiply-adds are fused, each
// corrector starts from the predicted b (predict_b_row) and the state updates are summed
// with compensation (Kahan), which the reference does not do.
#pragma once
#include "common.cuh"
#include "forces.cuh"
#include "radau.cuh"
#include "internal.h"

namespace kb {

constexpr int NODE_G = 8;

enum Phase : int {
    PH_EXACT_INIT = 0,
    PH_ITER = 1,
    PH_EXACT_STEP = 2,
    PH_DONE = 3,
    PH_WAIT = 4,      // WS: step accepted, the next one starts with the warp's other groups
    PH_FINISHED = 5,  // WS: no object left for this group
    PH_STORE = 6,     // pooled form: the object is finished, its outcome stored next round
};

__device__ __forceinline__ void nodes_store(const NBodyArgs& a, int64_t i, int rc, const double x[3],
                                            const double v[3], const SpkForce& F, double t_impact,
                                            const RadauCounters& cnt) {
    const int64_t n = a.n;
    double px = x[0], py = x[1], pz = x[2], vx = v[0], vy = v[1], vz = v[2];
    if (rc != ST_OK) {
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        px = py = pz = vx = vy = vz = nan;
    }
    a.out_pos[i] = px; a.out_pos[n + i] = py; a.out_pos[2 * n + i] = pz;
    a.out_vel[i] = vx; a.out_vel[n + i] = vy; a.out_vel[2 * n + i] = vz;
    a.status[i] = rc;
    if (a.impact_id) a.impact_id[i] = rc == ST_IMPACT ? F.impact_id : 0;
    if (a.impact_jd) a.impact_jd[i] = rc == ST_IMPACT ? t_impact : 0.0;
    if (a.min_dist) a.min_dist[i] = F.min_dist;
    if (a.counters) {
        a.counters[i] = cnt.steps;
        a.counters[n + i] = cnt.iterations;
        a.counters[2 * n + i] = cnt.exact;
    }
}


constexpr int NODES_BLOCK = 128;
constexpr int NODE_ROW = 17;  // doubles per node row in shared memory (16 used + 1 pad)

// MINB: minimum resident blocks per SM requested from the compiler (1 = no register cap);
// the host picks the instantiation (occupancy against spills is measured, not guessed).
// SE (step-end lane): lane 7, otherwise idle during a corrector iteration, evaluates the
// force at the step end t+h with the predictor of the current iteration (f = 1).  When the
// iteration converges, that evaluation becomes the exact evaluation of the new state, so
// no separate round is spent on it.  The point differs from the updated state by the b
// change of the converged iteration (< 1e-14 of |a| in b6 by the convergence test), far
// below the integration tolerance; impacts and closest approaches found by lane 7 only
// count when the iteration converges.  SE = false evaluates the updated state in a round
// of its own, as radau.rs:331-338 does.
//
// WS (warp-synchronous steps): the corrector iterations of a step evaluate the force at the
// same node times, so each lane keeps the bodies' positions at its last evaluation time in
// shared memory and later iterations skip the Chebyshev records (about four fifths of an
// evaluation).  That only saves time when no lane of the warp needs fresh records in the
// round, so a group whose step is accepted waits until the warp's other groups have
// finished their steps too, and all of them start their next steps in the same round; a
// group that finished its object fetches the next one at that point as well.  Each object's
// integration is the same as with WS = false up to rounding: the cached positions are
// rounded to doubles before the force terms read them, where the uncached evaluation may
// fuse the Chebyshev scaling into the difference x - body.
template <int MINB, bool SE, bool WS = false>
__global__ void __launch_bounds__(NODES_BLOCK, MINB) nbody_nodes_kernel(NBodyArgs a) {
    // node table: per node j, w_pow[j][0..6], u_pow[j][0..6], spacing, frac2 (rows padded
    // to 17 doubles so the 8 lanes of a group read 8 different banks); row 8 is the step
    // end (f = 1: W, U, 1, 1)
    __shared__ double s_node[9 * NODE_ROW];
    // per group: b (21 doubles, read by every lane for its predictor) and the 8 lanes'
    // evaluations (3 doubles each), exchanged after each corrector iteration
    __shared__ double s_b[NODES_BLOCK / NODE_G][21];
    __shared__ double s_e[NODES_BLOCK / NODE_G][NODE_G * 3];
    // per group: the running compensations of x and v (compensated summation of the updates)
    __shared__ double s_cmp[NODES_BLOCK / NODE_G][6];
    // WS: per lane, the bodies' positions at cache_t (slot k of lane l at k * NODES_BLOCK + l)
    __shared__ double s_cache[WS ? EPH_CACHE * NODES_BLOCK : 1];
    for (int i = threadIdx.x; i < 9 * NODE_ROW; i += blockDim.x) {
        const int j = i / NODE_ROW, k = i % NODE_ROW;
        double val = 0.0;
        if (j < 8) {
            if (k < 7) val = c_tab.w_pow[j][k];
            else if (k < 14) val = c_tab.u_pow[j][k - 7];
            else if (k == 14) val = c_tab.spacing[j];
            else if (k == 15) val = c_tab.frac2[j];
        } else {
            if (k < 7) val = c_tab.w[k];
            else if (k < 14) val = c_tab.u[k - 7];
            else if (k == 14 || k == 15) val = 1.0;
        }
        s_node[i] = val;
    }
    __syncthreads();

    const int lane = threadIdx.x & (NODE_G - 1);
    const int warp_lane = threadIdx.x & 31;
    const unsigned gmask = 0xFFu << (warp_lane & ~(NODE_G - 1));
    const int64_t group = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / NODE_G;
    double* sb = s_b[threadIdx.x / NODE_G];
    double* se = s_e[threadIdx.x / NODE_G];
    double* scmp = s_cmp[threadIdx.x / NODE_G];
    const int comp = lane % 3;  // component this lane forms g and b for (lanes 0-2 publish)
    const double* nrow = s_node + (lane < 7 ? lane + 1 : (SE ? 8 : 7)) * NODE_ROW;
    const bool se_lane = SE && lane == 7;

    int64_t obj = -1;
    int phase = PH_DONE;
    double t = 0.0, tf = 0.0, h = 0.0, next_h = 0.0;
    double x[3], v[3], acc[3];
    int iter = 0, failures = 0, attempts = 0;
    RadauCounters cnt;
    SpkForce F;
    F.n_force = a.n_force;
    int rc = ST_OK;
    const FastPlan& plan = a.n_force == c_eph.n_force_planets ? c_eph.fast_planets : c_eph.fast_all;
    const bool use_cache = WS && plan.ok && SpkForce::cached_doubles(plan) <= EPH_CACHE;
    double* cache = s_cache + threadIdx.x;
    double cache_t = __longlong_as_double(0x7ff8000000000000LL);  // nothing cached yet
    bool wait_predict = false;  // WS: the waiting step starts from the predicted b

    auto fetch = [&]() -> bool {
        int64_t k;
        if (a.queue) {
            int q = 0;
            if (lane == 0) q = atomicAdd(a.queue, 1);
            k = __shfl_sync(gmask, q, 0, NODE_G);
        } else {
            k = (obj < 0) ? group : a.n;  // one object per group
        }
        if (a.range) {  // a part of the order (launch_nodes_ordered)
            k += a.range[0];
            if (k >= a.range[1]) return false;
        } else if (k >= a.n) {
            return false;
        }
        obj = a.order ? a.order[k] : k;
        const int64_t n = a.n;
        t = a.jd0[obj];
        tf = a.jd1[obj];
        x[0] = a.pos[obj]; x[1] = a.pos[n + obj]; x[2] = a.pos[2 * n + obj];
        v[0] = a.vel[obj]; v[1] = a.vel[n + obj]; v[2] = a.vel[2 * n + obj];
        if (lane < 7) {
            sb[lane] = 0.0;
            sb[7 + lane] = 0.0;
            sb[14 + lane] = 0.0;
        }
        if (lane < 6) scmp[lane] = 0.0;
        F.ng.base = a.nongrav ? a.nongrav + obj : nullptr;
        F.ng.stride = n;
        F.ng.kind = a.nongrav ? (int)a.nongrav[obj] : 0;
        F.impact_id = 0;
        F.min_dist = 1e300;
        F.min_id = 0;
        cnt = RadauCounters();
        iter = 0;
        failures = 0;
        attempts = 0;
        rc = ST_OK;
        const bool finite = isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]) &&
                            isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]) && isfinite(t);
        if (!finite) rc = ST_VALUE_ERROR;
        if (rc == ST_OK) rc = to_ssb_equatorial(t, a.frame, a.chain, x, v);
        phase = PH_EXACT_INIT;
        __syncwarp(gmask);
        return true;
    };

    auto finish = [&](int code) {
        if (code == ST_OK) code = from_ssb_equatorial(tf, a.frame, a.chain, x, v);
        if (lane == 0) nodes_store(a, obj, code, x, v, F, t, cnt);
        phase = PH_DONE;
    };

    // step start: |h| >= MIN_STEP, then truncate to the final time (radau.rs:187-190,214-216);
    // after an accepted step the corrector starts from the predicted b (predict_b_row)
    double h_prev = 0.0;
    auto start_step = [&](bool predict) {
        if (fabs(h) < 0.005) h = copysign(0.005, h);
        if (fabs(t - tf) <= fabs(h)) h = tf - t;
        if (predict) {
            if (lane < 3) predict_b_row(sb + 7 * lane, h / h_prev);
            __syncwarp(gmask);
        }
        iter = 0;
        ++attempts;
        phase = PH_ITER;
    };

    if (!fetch()) {
        if (!WS) return;
        phase = PH_FINISHED;  // WS: the lanes stay for the warp's collective votes
    } else if (rc != ST_OK) {
        finish(rc);
    }

    int obj_rounds = 0;
    const int max_obj_rounds = a.max_loops * 11;
    for (;;) {
        if (WS) {
            // no group of the warp in the middle of a step: waiting groups start their next
            // steps and finished groups take their next objects, all in this round
            const bool busy = phase == PH_ITER || phase == PH_EXACT_INIT || phase == PH_EXACT_STEP;
            if (!__any_sync(0xffffffffu, busy)) {
                if (phase == PH_WAIT) {
                    start_step(wait_predict);
                } else if (phase == PH_DONE) {
                    obj_rounds = 0;
                    if (!a.queue || !fetch()) phase = PH_FINISHED;
                    else if (rc != ST_OK) finish(rc);
                }
            }
            if (__all_sync(0xffffffffu, phase == PH_FINISHED)) break;
            if (phase == PH_WAIT || phase == PH_DONE || phase == PH_FINISHED) continue;
        }
        // the step loop's bound: step attempts (kete_b200_set_step_limit), and rounds as a
        // second guard
        if (phase != PH_DONE && (++obj_rounds > max_obj_rounds || attempts > a.max_loops)) {
            finish(ST_TIMEOUT);
            continue;
        }
        if (phase == PH_DONE) {
            obj_rounds = 0;
            if (!a.queue) break;
            if (!fetch()) break;
            if (rc != ST_OK) {
                finish(rc);
                continue;
            }
        }
        // ---- evaluation point of this lane ----
        const bool iter_round = phase == PH_ITER;
        const bool exact = !iter_round || se_lane;
        double te, xe[3], ve[3];
        double saved_min = F.min_dist;
        int32_t saved_min_id = F.min_id;
        if (!iter_round) {
            te = t;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                xe[c] = x[c];
                ve[c] = v[c];
            }
        } else {
            const double f = nrow[14], frac2 = nrow[15];
            const double h2 = h * h;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double bw = 0.0, bu = 0.0;
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    const double bck = sb[7 * c + k];
                    bw += nrow[k] * bck;
                    bu += nrow[7 + k] * bck;
                }
                xe[c] = x[c] + f * v[c] * h + frac2 * h2 * (acc[c] / 2.0 + bw);
                ve[c] = v[c] + f * h * (acc[c] + bu);
            }
            te = t + f * h;
        }
        double ev[3];
        int erc;
        if (use_cache && te >= plan.lo && te <= plan.hi) {
            if (te != cache_t) {
                F.fast_positions(plan, te, cache, NODES_BLOCK);
                cache_t = te;
            }
            erc = F.fast_forces(plan, exact, xe, ve, cache, NODES_BLOCK, ev);
        } else {
            erc = F.eval(exact, te, xe, ve, ev);
        }
        // any lane of the group failing fails the group (only DAF limits / impacts occur);
        // the step-end lane's outcome only counts once the iteration converges
        const unsigned bad = __ballot_sync(gmask, erc != ST_OK && !(iter_round && se_lane));
        if (bad) {
            const int src = __ffs(bad) - 1 - (warp_lane & ~(NODE_G - 1));
            erc = __shfl_sync(gmask, erc, src, NODE_G);
            finish(erc);
            continue;
        }
        if (!iter_round) {
            cnt.exact++;
            acc[0] = ev[0];
            acc[1] = ev[1];
            acc[2] = ev[2];
            if (phase == PH_EXACT_INIT) {
                if (fabs(tf - t) < 1e-10) {
                    finish(ST_OK);
                    continue;
                }
                h = copysign(0.1, tf - t);
                failures = 0;
                if (WS) {
                    wait_predict = false;
                    phase = PH_WAIT;
                } else {
                    start_step(false);
                }
                continue;
            }
            cnt.steps++;
            h_prev = h;
            h = next_h;
            if (fabs(t - tf) < 1e-12) {
                finish(ST_OK);
                continue;
            }
            failures = 0;
            if (WS) {
                wait_predict = true;
                phase = PH_WAIT;
            } else {
                start_step(true);
            }
            continue;
        }
        // ---- corrector iteration: exchange the 7 node evaluations, form g and b ----
        // (radau.rs:292-313).  Lanes 0-2 each own one component; every lane then reads the
        // new b for the convergence test and the state update.
        cnt.iterations++;
        se[3 * lane + 0] = ev[0];
        se[3 * lane + 1] = ev[1];
        se[3 * lane + 2] = ev[2];
        const double b6_old0 = sb[6], b6_old1 = sb[13], b6_old2 = sb[20];
        __syncwarp(gmask);
        {
            const double ac = comp == 0 ? acc[0] : (comp == 1 ? acc[1] : acc[2]);
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
        const double e70 = se[18], e71 = se[19], e72 = se[20];  // node 7 = lane 6
        const double fem0 = fabs(e70) + 1e-6, fem1 = fabs(e71) + 1e-6, fem2 = fabs(e72) + 1e-6;
        const double b60 = sb[6], b61 = sb[13], b62 = sb[20];
        const double ratio = fmax(fmax(fabs(b60 - b6_old0) / fem0, fabs(b61 - b6_old1) / fem1),
                                  fabs(b62 - b6_old2) / fem2);
        ++iter;
        if (ratio < 1e-14) {
            const double h2 = h * h;
            // x += dx, v += dv with compensated (Kahan) summation: the rounding error of each
            // addition is carried into the next step's, so the many small increments of a long
            // integration do not accumulate rounding in x and v
            double ncx[3], ncv[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double dw = 0.0, du = 0.0;
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    const double bck = sb[7 * c + k];
                    dw += bck * c_tab.w[k];
                    du += bck * c_tab.u[k];
                }
                const double dx = v[c] * h + h2 * (acc[c] * 0.5 + dw);
                const double dv = h * (acc[c] + du);
                const double yx = dx - scmp[c], yv = dv - scmp[3 + c];
                const double tx = x[c] + yx, tv = v[c] + yv;
                ncx[c] = (tx - x[c]) - yx;
                ncv[c] = (tv - v[c]) - yv;
                x[c] = tx;
                v[c] = tv;
            }
            __syncwarp(gmask);  // every lane has read the old compensations
            if (lane < 3) {
                scmp[lane] = lane == 0 ? ncx[0] : (lane == 1 ? ncx[1] : ncx[2]);
                scmp[3 + lane] = lane == 0 ? ncv[0] : (lane == 1 ? ncv[1] : ncv[2]);
            }
            t += h;
            const double mb6 = fmax(fmax(fabs(b60), fabs(b61)), fabs(b62));
            const double r = pow(1e-6 * fmax(fmax(fem0, fem1), fem2) / mb6, 1.0 / 7.0);
            next_h = h * clampd(r, 0.25, 4.0);
            if (!SE) {
                phase = PH_EXACT_STEP;
                __syncwarp(gmask);  // b and evaluations consumed before the next round rewrites them
                continue;
            }
            // the step-end lane's evaluation is the exact evaluation of the new state
            const int se_rc = __shfl_sync(gmask, erc, 7, NODE_G);
            F.min_dist = __shfl_sync(gmask, F.min_dist, 7, NODE_G);
            F.min_id = __shfl_sync(gmask, F.min_id, 7, NODE_G);
            F.impact_id = __shfl_sync(gmask, F.impact_id, 7, NODE_G);
            acc[0] = se[21];
            acc[1] = se[22];
            acc[2] = se[23];
            __syncwarp(gmask);
            cnt.exact++;
            if (se_rc != ST_OK) {
                finish(se_rc);
                continue;
            }
            cnt.steps++;
            h_prev = h;
            h = next_h;
            if (fabs(t - tf) < 1e-12) {
                finish(ST_OK);
                continue;
            }
            failures = 0;
            if (WS) {
                wait_predict = true;
                phase = PH_WAIT;
            } else {
                start_step(true);
            }
            continue;
        }
        if (se_lane) {  // iteration not converged: forget the step-end lane's record
            F.min_dist = saved_min;
            F.min_id = saved_min_id;
        }
        __syncwarp(gmask);
        if (iter >= 10) {  // step failed to converge (radau.rs:345) -> retry smaller
            failures += 1;
            h *= 0.7;
            if (failures > 10) {
                finish(ST_CONVERGENCE);
                continue;
            }
            start_step(false);
        }
    }
}

}  // namespace kb
