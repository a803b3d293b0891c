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
// expensive instruction stream.  The arithmetic of each step is the reference's; only the
// division by node spacings uses tabulated reciprocals and multiply-adds are fused.
#pragma once
#include "common.cuh"
#include "forces.cuh"
#include "radau.cuh"
#include "internal.h"

namespace kb {

constexpr int NODE_G = 8;

enum Phase : int { PH_EXACT_INIT = 0, PH_ITER = 1, PH_EXACT_STEP = 2, PH_DONE = 3 };

// Force evaluation with a runtime exact flag (single call site in the round loop).
__device__ __forceinline__ int spk_eval_rt(SpkForce& F, bool exact, double t, const double x[3],
                                           const double v[3], double out[3]) {
    if (exact) return F.template eval<true>(t, x, v, out);
    return F.template eval<false>(t, x, v, out);
}

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


__global__ void __launch_bounds__(128) nbody_nodes_kernel(NBodyArgs a) {
    const int lane = threadIdx.x & (NODE_G - 1);
    const int warp_lane = threadIdx.x & 31;
    const unsigned gmask = 0xFFu << (warp_lane & ~(NODE_G - 1));
    const int64_t group = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / NODE_G;
    const int64_t n_groups = ((int64_t)gridDim.x * blockDim.x) / NODE_G;

    // node handled by this lane and its predictor coefficients
    const int jn = lane < 7 ? lane + 1 : 7;
    const double f = c_tab.spacing[jn];
    const double frac2 = c_tab.frac2[jn];
    double wp[7], up[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        wp[k] = c_tab.w_pow[jn][k];
        up[k] = c_tab.u_pow[jn][k];
    }

    int64_t obj = -1;
    int phase = PH_DONE;
    RadauObj s;
    double tf = 0.0, h = 0.0, next_h = 0.0;
    int iter = 0, failures = 0;
    RadauCounters cnt;
    SpkForce F;
    F.n_force = a.n_force;
    int rc = ST_OK;

    auto fetch = [&]() -> bool {
        int64_t k;
        if (a.queue) {
            int q = 0;
            if (lane == 0) q = atomicAdd(a.queue, 1);
            k = __shfl_sync(gmask, q, 0, NODE_G);
        } else {
            k = (obj < 0) ? group : a.n;  // one object per group
        }
        if (k >= a.n) return false;
        obj = a.order ? a.order[k] : k;
        const int64_t n = a.n;
        s.t = a.jd0[obj];
        tf = a.jd1[obj];
        s.x[0] = a.pos[obj]; s.x[1] = a.pos[n + obj]; s.x[2] = a.pos[2 * n + obj];
        s.v[0] = a.vel[obj]; s.v[1] = a.vel[n + obj]; s.v[2] = a.vel[2 * n + obj];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k2 = 0; k2 < 7; ++k2) s.b[c][k2] = 0.0;
        F.ng.base = a.nongrav ? a.nongrav + obj : nullptr;
        F.ng.stride = n;
        F.ng.kind = a.nongrav ? (int)a.nongrav[obj] : 0;
        F.impact_id = 0;
        F.min_dist = 1e300;
        F.min_id = 0;
        cnt = RadauCounters();
        iter = 0;
        failures = 0;
        rc = ST_OK;
        const bool finite = isfinite(s.x[0]) && isfinite(s.x[1]) && isfinite(s.x[2]) &&
                            isfinite(s.v[0]) && isfinite(s.v[1]) && isfinite(s.v[2]) && isfinite(s.t);
        if (!finite) rc = ST_VALUE_ERROR;
        if (rc == ST_OK) rc = to_ssb_equatorial(s.t, a.frame, a.chain, s.x, s.v);
        phase = PH_EXACT_INIT;
        return true;
    };

    auto finish = [&](int code) {
        if (code == ST_OK) code = from_ssb_equatorial(tf, a.frame, a.chain, s.x, s.v);
        if (lane == 0) nodes_store(a, obj, code, s.x, s.v, F, s.t, cnt);
        phase = PH_DONE;
    };

    // step start: truncate to the final time and reset the iteration (radau.rs:187-190,226-229)
    auto start_step = [&]() {
        if (fabs(h) < 0.005) h = copysign(0.005, h);
        if (fabs(s.t - tf) <= fabs(h)) h = tf - s.t;
        iter = 0;
        phase = PH_ITER;
    };

    if (group >= n_groups) return;
    if (!fetch()) return;
    if (rc != ST_OK) finish(rc);

    int obj_rounds = 0;
    const int max_obj_rounds = a.max_loops * 11;
    for (;;) {
        if (phase != PH_DONE && ++obj_rounds > max_obj_rounds) {
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
        const bool exact = phase != PH_ITER;
        double te, xe[3], ve[3];
        if (exact) {
            te = s.t;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                xe[c] = s.x[c];
                ve[c] = s.v[c];
            }
        } else {
            const double h2 = h * h;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double bw = 0.0, bu = 0.0;
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    bw += wp[k] * s.b[c][k];
                    bu += up[k] * s.b[c][k];
                }
                xe[c] = s.x[c] + f * s.v[c] * h + frac2 * h2 * (s.a[c] / 2.0 + bw);
                ve[c] = s.v[c] + f * h * (s.a[c] + bu);
            }
            te = s.t + f * h;
        }
        double ev[3];
        int erc = spk_eval_rt(F, exact, te, xe, ve, ev);
        __syncwarp(gmask);
        // any lane of the group failing fails the group (only DAF limits / impacts occur)
        const unsigned bad = __ballot_sync(gmask, erc != ST_OK);
        if (bad) {
            const int src = __ffs(bad) - 1 - (warp_lane & ~(NODE_G - 1));
            erc = __shfl_sync(gmask, erc, src, NODE_G);
            finish(erc);
            continue;
        }
        if (exact) {
            cnt.exact++;
            s.a[0] = ev[0];
            s.a[1] = ev[1];
            s.a[2] = ev[2];
            if (phase == PH_EXACT_INIT) {
                if (fabs(tf - s.t) < 1e-10) {
                    finish(ST_OK);
                    continue;
                }
                h = copysign(0.1, tf - s.t);
                failures = 0;
            } else {
                cnt.steps++;
                h = next_h;
                if (fabs(s.t - tf) < 1e-12) {
                    finish(ST_OK);
                    continue;
                }
                failures = 0;
            }
            start_step();
            continue;
        }
        // ---- corrector iteration: gather the 7 node evaluations ----
        cnt.iterations++;
        double g[3][7];
        double e7[3];
#pragma unroll
        for (int j = 1; j < 8; ++j) {
            double e[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) e[c] = __shfl_sync(gmask, ev[c], j - 1, NODE_G);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double gk = (e[c] - s.a[c]) * c_tab.inv_frac[j];
#pragma unroll
                for (int z = 1; z < j; ++z) gk = (gk - g[c][z - 1]) * c_tab.inv_diff[j][z];
                g[c][j - 1] = gk;
            }
            if (j == 7) {
                e7[0] = e[0];
                e7[1] = e[1];
                e7[2] = e[2];
            }
        }
        const double b6_old[3] = {s.b[0][6], s.b[1][6], s.b[2][6]};
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int jj = 0; jj < 7; ++jj) {
                double acc = g[c][jj];
#pragma unroll
                for (int k = jj + 1; k < 7; ++k) acc += c_tab.c[k][jj] * g[c][k];
                s.b[c][jj] = acc;
            }
        double fem[3], ratio[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            fem[c] = fabs(e7[c]) + 1e-6;
            ratio[c] = fabs(s.b[c][6] - b6_old[c]) / fem[c];
        }
        ++iter;
        if (fmax(fmax(ratio[0], ratio[1]), ratio[2]) < 1e-14) {
            const double h2 = h * h;
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
            const double mb6 = fmax(fmax(fabs(s.b[0][6]), fabs(s.b[1][6])), fabs(s.b[2][6]));
            const double r = pow(1e-6 * fmax(fmax(fem[0], fem[1]), fem[2]) / mb6, 1.0 / 7.0);
            next_h = h * clampd(r, 0.25, 4.0);
            phase = PH_EXACT_STEP;
            continue;
        }
        if (iter >= 10) {  // step failed to converge (radau.rs:345) -> retry smaller
            failures += 1;
            h *= 0.7;
            if (failures > 10) {
                finish(ST_CONVERGENCE);
                continue;
            }
            start_step();
        }
    }
}

}  // namespace kb
