// radau_pool.cuh -- node-parallel Radau (8 lanes per object, as radau_nodes.cuh) whose
// ephemeris records are evaluated by the whole warp as one pool of work.
//
// Every corrector iteration of a step evaluates the force at the same eight times (the
// seven nodes and the step end), and about four fifths of an uncached evaluation is the
// Chebyshev records of the bodies, which depend on the time alone.  Each lane therefore keeps
// the bodies' positions (and the Sun's and Jupiter's velocities) at its last evaluation time
// in shared memory, and only the first iteration of a step needs records.  In the
// warp-synchronous form of radau_nodes.cuh the four objects of a warp start their steps
// together so that such rounds are warp-uniform, which leaves the groups that converge early
// waiting for the slowest.  Here the groups run independently; in every round the lanes that
// need records at a new time are collected with a ballot, and all 32 lanes of the warp share
// their record evaluations: the records whose velocities enter the force (two per lane and
// target, in lockstep) and then the position-only records (three per lane, in lockstep), each
// result written to the target lane's cache.  A round in which one object starts a step thus
// costs every lane about a ninth of that object's records instead of leaving three quarters of
// the warp idle, and no object waits for another.
//
// The integration of each object is the one of radau_nodes.cuh with the step-end lane
// (lane 7 evaluates the step end during each corrector iteration and supplies the exact
// evaluation of the accepted step), the predicted corrector start and the compensated state
// update; the cached positions are rounded to doubles before the force terms read them, so
// results agree with the uncached forms to rounding.
//
// The kernel carries no general ephemeris evaluation: the host orders the objects whose span
// leaves the fast plan's window after the others and integrates those with a form that has
// it (launch_nodes_ordered).  An out-of-line call makes the caller keep its live registers
// across it; with the general evaluation, the non-gravitational term (inside the force loop)
// and the centre changes as calls this kernel spilled about a quarter of a kilobyte per lane
// at 128 registers.  Now the centre changes at an object's start and end run in kernels of
// their own before and after (pool_prepare_kernel, pool_finish_kernel), and the
// non-gravitational term (relative to the Sun) is added after the bodies' terms are summed,
// where few values are live: inline for the JPL comet model without delay, and as the one
// call for the delayed model and dust.  (Without that call, with the delayed comets sent to
// the general form instead, the kernel needs 145 registers and spills nothing at 128, but
// it measured 1.7% slower on the batched workload.)
#pragma once
#include "common.cuh"
#include "forces.cuh"
#include "internal.h"
#include "radau.cuh"
#include "radau_nodes.cuh"

namespace kb {

// One record source of the plan as the pool reads it: the segment's records, the record
// lookup, and the cache slot its evaluation fills.
struct PoolSrc {
    const double* rec0;
    double start_s, inv_intlen, n_rec;
    int rsize, slot;
};

__device__ __forceinline__ const double* pool_record(const PoolSrc& S, double jds) {
    const double fidx = floor((jds - S.start_s) * S.inv_intlen);
    const int idx = fidx < 0.0 ? 0 : (fidx >= S.n_rec ? (int)S.n_rec - 1 : (int)fidx);
    return S.rec0 + (int64_t)idx * S.rsize;
}

// Positions of three records, each at its own time (value recurrences in lockstep); the
// arithmetic of each record is cheb_pos3's.
template <int NC>
__device__ __forceinline__ void cheb_pos3_at(const double* const r[3], const double jds[3],
                                             double out[3][3]) {
    constexpr int NP = (NC + 1) & ~1;
    double x2[3], t1[3], t2[3], acc[3][3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double2 h0 = __ldg(reinterpret_cast<const double2*>(r[q]));
        const double2 h1 = __ldg(reinterpret_cast<const double2*>(r[q] + 2));
        const double xx = (jds[q] - h0.x) * h1.x;
        x2[q] = 2.0 * xx;
        t2[q] = 1.0;
        t1[q] = xx;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double2 a = __ldg(reinterpret_cast<const double2*>(r[q] + 4 + c * NP));
            acc[q][c] = a.x + a.y * xx;
        }
    }
#pragma unroll 1
    for (int k = 1; 2 * k < NC; ++k) {
        double2 co[3][3];
#pragma unroll
        for (int q = 0; q < 3; ++q)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                co[q][c] = __ldg(reinterpret_cast<const double2*>(r[q] + 4 + c * NP) + k);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (2 * k + h < NC) {
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const double nt = x2[q] * t1[q] - t2[q];
#pragma unroll
                    for (int c = 0; c < 3; ++c) acc[q][c] += (h ? co[q][c].y : co[q][c].x) * nt;
                    t2[q] = t1[q];
                    t1[q] = nt;
                }
            }
        }
    }
    constexpr double INV_AU_KM = 1.0 / AU_KM;
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) out[q][c] = acc[q][c] * INV_AU_KM;
}

// The warp's record evaluations of one round.  M: lanes that need records at their time
// te (s_te[warp_base + lane]); s_tgt[warp_base + p] is the p-th of them in lane order.  src:
// the nv velocity sources, then the np position sources.  Called by all 32 lanes.
__device__ __forceinline__ void pool_records(unsigned M, int warp_lane, int warp_base,
                                             const PoolSrc* src, int nv, int np,
                                             const double* s_te, const int* s_tgt,
                                             double* s_cache) {
    const int P = __popc(M);
    const int nvp = (nv + 1) >> 1;  // velocity pairs per target
#pragma unroll 1
    for (int q = warp_lane; q < P * nvp; q += 32) {
        const int p = q / nvp;
        const int k = 2 * (q - p * nvp);
        const int tl = warp_base + s_tgt[warp_base + p];
        const double jds = __dmul_rn(s_te[tl] - 2451545.0, 86400.0);
        const bool has_b = k + 1 < nv;
        const PoolSrc& A = src[k];
        const PoolSrc& B = src[has_b ? k + 1 : k];
        double pa[3], va[3], pb[3], vb[3];
        cheb_pair<FAST_NC, 1>(pool_record(A, jds), pool_record(B, jds), jds, pa, va, pb, vb);
        double* ca = s_cache + A.slot * NODES_BLOCK + tl;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ca[c * NODES_BLOCK] = pa[c];
            ca[(3 + c) * NODES_BLOCK] = va[c];
        }
        if (has_b) {
            double* cb = s_cache + B.slot * NODES_BLOCK + tl;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                cb[c * NODES_BLOCK] = pb[c];
                cb[(3 + c) * NODES_BLOCK] = vb[c];
            }
        }
    }
    const int total = P * np;
#pragma unroll 1
    for (int q0 = 3 * warp_lane; q0 < total; q0 += 96) {
        const double* r[3];
        double jds[3];
        double* dst[3];
#pragma unroll
        for (int h = 0; h < 3; ++h) {
            const int q = q0 + h < total ? q0 + h : total - 1;  // a missing third repeats
            const int p = q / np;
            const int k = q - p * np;
            const int tl = warp_base + s_tgt[warp_base + p];
            jds[h] = __dmul_rn(s_te[tl] - 2451545.0, 86400.0);
            const PoolSrc& S = src[nv + k];
            r[h] = pool_record(S, jds[h]);
            dst[h] = s_cache + S.slot * NODES_BLOCK + tl;
        }
        double out[3][3];
        cheb_pos3_at<FAST_NC>(r, jds, out);
#pragma unroll
        for (int h = 0; h < 3; ++h)
            if (q0 + h < total)
#pragma unroll
                for (int c = 0; c < 3; ++c) dst[h][c * NODES_BLOCK] = out[h][c];
    }
}

// The force at (x, v) from a lane's cached body states, summed in the fast plan's order
// (eval_fast's): the velocity items, then the others, with the chained bodies offset by the
// centre kept before them.  One body at a time: the kernel is bound by its registers, and
// forming several bodies' terms together spills more than it hides.  The non-gravitational
// term is not included (the kernel adds it after this sum).
__device__ __forceinline__ int pool_forces(const FastPlan& P, SpkForce& F, bool exact,
                                           const double x[3], const double v[3],
                                           const double* cache, double out[3]) {
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    const int n_vel = P.n_vel;
    int k = 0;
#pragma unroll 1
    for (int it = 0; it < n_vel; ++it, k += 6) {
        const FastItem& A = P.item[it];
        const double bp[3] = {cache[k * NODES_BLOCK], cache[(k + 1) * NODES_BLOCK],
                              cache[(k + 2) * NODES_BLOCK]};
        const double bv[3] = {cache[(k + 3) * NODES_BLOCK], cache[(k + 4) * NODES_BLOCK],
                              cache[(k + 5) * NODES_BLOCK]};
        const ForceEntry fe{A.mass, A.radius, 0, A.kind, A.naif_id, 0};
        const int rc = F.body<true, false>(fe, exact, x, v, bp, bv, acc0, acc1, acc2);
        if (rc != ST_OK) return rc;
    }
    const double zero[3] = {0.0, 0.0, 0.0};
    double cp[3] = {0.0, 0.0, 0.0};
    const int n_items = P.n_items;
#pragma unroll 1
    for (int it = n_vel; it < n_items; ++it) {
        const FastItem& I = P.item[it];
        if (I.role == -2) continue;
        double bp[3] = {cache[k * NODES_BLOCK], cache[(k + 1) * NODES_BLOCK],
                        cache[(k + 2) * NODES_BLOCK]};
        k += 3;
        if (I.role < 0) {
            cp[0] = bp[0]; cp[1] = bp[1]; cp[2] = bp[2];
            continue;
        }
        if (I.chained) {
            bp[0] += cp[0]; bp[1] += cp[1]; bp[2] += cp[2];
        }
        const ForceEntry fe{I.mass, I.radius, 0, I.kind, I.naif_id, 0};
        const int rc = F.body<false>(fe, exact, x, v, bp, zero, acc0, acc1, acc2);
        if (rc != ST_OK) return rc;
    }
    out[0] = acc0;
    out[1] = acc1;
    out[2] = acc2;
    return ST_OK;
}

// The centre and frame changes of the pooled kernel's objects, in kernels of their own (one
// thread per object of the part order[range[0] .. range[2])): their code (a general state
// query of the centre's chain) runs once per object, and inside the step loop's kernel it
// cost instruction-cache misses to every warp of the SM.
//
// Before the integration: the checks of the inputs and to_ssb_equatorial (mod.rs:79-80) at
// the epoch; the barycentric equatorial state goes to the output arrays, the outcome to
// status, where nbody_pool_kernel reads both.
static __global__ void pool_prepare_kernel(NBodyArgs a) {
    const int64_t first = a.range[0], end = a.range[2], n = a.n;
    for (int64_t k = first + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < end;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t obj = a.order[k];
        const double t0 = a.jd0[obj];
        double p[3] = {a.pos[obj], a.pos[n + obj], a.pos[2 * n + obj]};
        double v[3] = {a.vel[obj], a.vel[n + obj], a.vel[2 * n + obj]};
        const bool finite = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]) &&
                            isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]) && isfinite(t0);
        int rc = finite ? ST_OK : ST_VALUE_ERROR;
        if (rc == ST_OK && (a.chain.len > 0 || a.frame == FRAME_ECLIPTIC))
            rc = to_ssb_equatorial(t0, a.frame, a.chain, p, v);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a.out_pos[c * n + obj] = p[c];
            a.out_vel[c * n + obj] = v[c];
        }
        a.status[obj] = rc;
    }
}

// After it: from_ssb_equatorial (mod.rs:107-116) at the target epoch for every object that
// arrived; a failure there gives NaN and its status, as in the other forms.
static __global__ void pool_finish_kernel(NBodyArgs a) {
    const int64_t first = a.range[0], end = a.range[2], n = a.n;
    if (!(a.chain.len > 0 || a.frame == FRAME_ECLIPTIC)) return;
    for (int64_t k = first + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < end;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t obj = a.order[k];
        if (a.status[obj] != ST_OK) continue;
        double p[3] = {a.out_pos[obj], a.out_pos[n + obj], a.out_pos[2 * n + obj]};
        double v[3] = {a.out_vel[obj], a.out_vel[n + obj], a.out_vel[2 * n + obj]};
        const int rc = from_ssb_equatorial(a.jd1[obj], a.frame, a.chain, p, v);
        if (rc != ST_OK) {
            const double nan = __longlong_as_double(0x7ff8000000000000LL);
            p[0] = p[1] = p[2] = v[0] = v[1] = v[2] = nan;
            a.status[obj] = rc;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a.out_pos[c * n + obj] = p[c];
            a.out_vel[c * n + obj] = v[c];
        }
    }
}

// Dynamic shared memory of the pooled kernel: the body cache.
constexpr int POOL_DYN_SMEM = POOL_CACHE_DOUBLES * NODES_BLOCK * (int)sizeof(double);

// Per-group state in shared memory (doubles): the object's epoch, target epoch, step, previous
// step, position, velocity and acceleration at the epoch.  Every lane of a group needs the
// same values; keeping them out of the lanes' registers leaves the registers to the hot loop.
constexpr int ST_T = 0, ST_TF = 1, ST_H = 2, ST_HP = 3, ST_X = 4, ST_V = 7, ST_A = 10;
constexpr int ST_ROW = 13;

// MINB: minimum resident blocks per SM requested from the compiler (3: 168 registers,
// 4: 128); the host picks the instantiation.  With a.queue the grid is persistent and groups
// take objects from the queue; without, each group integrates one object.
template <int MINB>
__global__ void __launch_bounds__(NODES_BLOCK, MINB) nbody_pool_kernel(NBodyArgs a) {
    extern __shared__ double s_cache[];  // slot k of thread i at k * NODES_BLOCK + i
    __shared__ double s_node[9 * NODE_ROW];
    __shared__ double s_b[NODES_BLOCK / NODE_G][21];
    __shared__ double s_e[NODES_BLOCK / NODE_G][NODE_G * 3];
    __shared__ double s_cmp[NODES_BLOCK / NODE_G][6];
    __shared__ double s_st[NODES_BLOCK / NODE_G][ST_ROW];
    __shared__ double s_te[NODES_BLOCK];
    __shared__ int s_tgt[NODES_BLOCK];
    __shared__ PoolSrc s_src[MAX_ITEMS];
    __shared__ int s_nsrc[2];
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
    const FastPlan& plan = a.n_force == c_eph.n_force_planets ? c_eph.fast_planets : c_eph.fast_all;
    const bool use_pool = plan.ok && pool_plan_doubles(plan) <= POOL_CACHE_DOUBLES;
    if (threadIdx.x == 0) {
        // the record sources in pool order: velocity items, then the other items but padding
        int ns = 0, slot = 0;
        for (int it = 0; it < plan.n_items && use_pool; ++it) {
            const FastItem& I = plan.item[it];
            if (it >= plan.n_vel && I.role == -2) continue;
            PoolSrc& S = s_src[ns++];
            S.rec0 = c_eph.pool + I.offset;
            S.start_s = I.start_s;
            S.inv_intlen = I.inv_intlen;
            S.n_rec = I.n_rec;
            S.rsize = I.rsize;
            S.slot = slot;
            slot += it < plan.n_vel ? 6 : 3;
        }
        s_nsrc[0] = use_pool ? plan.n_vel : 0;
        s_nsrc[1] = use_pool ? ns - plan.n_vel : 0;
    }
    __syncthreads();
    const int nv = s_nsrc[0], np = s_nsrc[1];

    const int lane = threadIdx.x & (NODE_G - 1);
    const int warp_lane = threadIdx.x & 31;
    const int warp_base = threadIdx.x & ~31;
    const unsigned gmask = 0xFFu << (warp_lane & ~(NODE_G - 1));
    const int64_t group = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / NODE_G;
    double* sb = s_b[threadIdx.x / NODE_G];
    double* se = s_e[threadIdx.x / NODE_G];
    double* scmp = s_cmp[threadIdx.x / NODE_G];
    double* st = s_st[threadIdx.x / NODE_G];
    const int comp = lane % 3;  // component this lane forms g and b for (lanes 0-2 publish)
    const double* nrow = s_node + (lane < 7 ? lane + 1 : 8) * NODE_ROW;
    const bool se_lane = lane == 7;
    const double* cache = s_cache + threadIdx.x;

    int64_t obj = -1;
    int phase = PH_DONE;
    int iter = 0, failures = 0, attempts = 0;
    RadauCounters cnt;
    SpkForce F;
    F.n_force = a.n_force;
    F.ng.base = nullptr;
    F.ng.stride = a.n;
    F.ng.kind = 0;
    F.impact_id = 0;
    F.min_dist = 1e300;
    F.min_id = 0;
    double cache_t = __longlong_as_double(0x7ff8000000000000LL);  // nothing cached yet
    bool first = true;
    int outcome = ST_OK;  // outcome of a finished object, stored at the top of the next round

    auto fetch = [&]() -> bool {
        // the objects inside the fast window: order[range[0] .. range[2]), those with a
        // non-gravitational model from range[1] on (launch_nodes_ordered)
        int64_t k;
        if (a.queue) {
            // groups on the first SMs take the non-gravitational part first, the others the
            // rest; each turns to the other part when its own is used up.  Only a few SMs then
            // fetch the non-gravitational model's code, which evicts the step loop from an
            // SM's instruction cache.
            int q = 0;
            if (lane == 0) {
                const int r0 = a.range[0], r1 = a.range[1], r2 = a.range[2];
                unsigned smid, nsm;
                asm("mov.u32 %0, %%smid;" : "=r"(smid));
                asm("mov.u32 %0, %%nsmid;" : "=r"(nsm));
                const bool ng_first =
                    r2 > r1 && (int64_t)smid * (r2 - r0) < (int64_t)nsm * (r2 - r1) + (r2 - r0);
                q = r2;  // nothing left
                for (int pass = 0; pass < 2; ++pass) {
                    const bool ng_part = (pass == 0) == ng_first;
                    const int lo = ng_part ? r1 : r0, hi = ng_part ? r2 : r1;
                    if (hi > lo) {
                        const int t = atomicAdd(ng_part ? a.queue_ng : a.queue, 1);
                        if (t < hi - lo) {
                            q = lo + t;
                            break;
                        }
                    }
                }
            }
            k = __shfl_sync(gmask, q, 0, NODE_G);
        } else {
            k = first ? group + a.range[0] : a.n;  // one object per group
        }
        first = false;
        if (k >= a.range[2]) return false;
        obj = a.order ? a.order[k] : k;
        int frc = ST_OK;
        if (lane == 0) {
            // the state at the epoch as pool_prepare_kernel left it (barycentric equatorial,
            // in the output arrays) and the outcome of its checks
            const int64_t n = a.n;
            frc = a.status[obj];
            st[ST_T] = a.jd0[obj];
            st[ST_TF] = a.jd1[obj];
            st[ST_X] = a.out_pos[obj]; st[ST_X + 1] = a.out_pos[n + obj];
            st[ST_X + 2] = a.out_pos[2 * n + obj];
            st[ST_V] = a.out_vel[obj]; st[ST_V + 1] = a.out_vel[n + obj];
            st[ST_V + 2] = a.out_vel[2 * n + obj];
        }
        if (lane < 7) {
            sb[lane] = 0.0;
            sb[7 + lane] = 0.0;
            sb[14 + lane] = 0.0;
        }
        if (lane < 6) scmp[lane] = 0.0;
        F.ng.base = a.nongrav ? a.nongrav + obj : nullptr;
        F.ng.kind = a.nongrav ? (int)a.nongrav[obj] : 0;
        F.impact_id = 0;
        F.min_dist = 1e300;
        F.min_id = 0;
        cnt = RadauCounters();
        iter = 0;
        failures = 0;
        attempts = 0;
        outcome = __shfl_sync(gmask, frc, 0, NODE_G);
        phase = outcome == ST_OK ? PH_EXACT_INIT : PH_STORE;
        __syncwarp(gmask);
        return true;
    };

    auto finish = [&](int code) {
        outcome = code;
        phase = PH_STORE;
    };

    // step start with step h (every lane computes the same): |h| >= MIN_STEP, then truncate
    // to the final time (radau.rs:187-190,214-216); after an accepted step the corrector
    // starts from the predicted b (predict_b_row).  Lane 0 publishes the step.
    auto start_step = [&](double h, double t, double tf, bool predict, double h_prev) {
        if (fabs(h) < 0.005) h = copysign(0.005, h);
        if (fabs(t - tf) <= fabs(h)) h = tf - t;
        if (predict && lane < 3) predict_b_row(sb + 7 * lane, h / h_prev);
        if (lane == 0) st[ST_H] = h;
        __syncwarp(gmask);
        iter = 0;
        ++attempts;
        phase = PH_ITER;
    };

    int obj_rounds = 0;
    const int max_obj_rounds = a.max_loops * 11;
    for (;;) {
        if (phase == PH_STORE) {  // the finished object's outcome (lane 0 stores)
            if (lane == 0) {  // barycentric equatorial; pool_finish_kernel changes it back
                const double xs[3] = {st[ST_X], st[ST_X + 1], st[ST_X + 2]};
                const double vs[3] = {st[ST_V], st[ST_V + 1], st[ST_V + 2]};
                nodes_store(a, obj, outcome, xs, vs, F, st[ST_T], cnt);
            }
            __syncwarp(gmask);  // st is read before the next object overwrites it
            phase = PH_DONE;
        }
        if (phase == PH_DONE) {  // take the next object (group-collective)
            obj_rounds = 0;
            if (!fetch()) phase = PH_FINISHED;
        }
        // every lane of the warp stays in the loop for the pool's collectives until all
        // four groups have run out of objects
        if (__all_sync(0xffffffffu, phase == PH_FINISHED)) break;
        bool active = phase == PH_ITER || phase == PH_EXACT_INIT;
        // the step loop's bound: step attempts (kete_b200_set_step_limit), and rounds as a
        // second guard
        if (active && (++obj_rounds > max_obj_rounds || attempts > a.max_loops)) {
            finish(ST_TIMEOUT);
            active = false;
        }
        // ---- evaluation time of this lane (the position and velocity follow the record
        // pass, so that they are not live across its recurrences) ----
        const bool iter_round = phase == PH_ITER;
        double te = 0.0;
        if (active) te = iter_round ? st[ST_T] + nrow[14] * st[ST_H] : st[ST_T];
        const bool fast = active && use_pool && te >= plan.lo && te <= plan.hi;
        const bool need = fast && te != cache_t;
        // ---- the warp's record evaluations for every lane at a new time ----
        const unsigned M = __ballot_sync(0xffffffffu, need);
        if (M) {
            if (need) {
                s_tgt[warp_base + __popc(M & ((1u << warp_lane) - 1u))] = warp_lane;
                s_te[threadIdx.x] = te;
            }
            __syncwarp();
            pool_records(M, warp_lane, warp_base, s_src, nv, np, s_te, s_tgt, s_cache);
            __syncwarp();
            if (need) cache_t = te;
        }
        if (!active) continue;
        double xe[3], ve[3];
        if (!iter_round) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                xe[c] = st[ST_X + c];
                ve[c] = st[ST_V + c];
            }
        } else {
            const double f = nrow[14], frac2 = nrow[15];
            const double h = st[ST_H];
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
                const double ac = st[ST_A + c];
                xe[c] = st[ST_X + c] + f * st[ST_V + c] * h + frac2 * h2 * (ac / 2.0 + bw);
                ve[c] = st[ST_V + c] + f * h * (ac + bu);
            }
        }
        const bool exact = !iter_round || se_lane;
        const double saved_min = F.min_dist;
        const int32_t saved_min_id = F.min_id;
        double ev[3] = {0.0, 0.0, 0.0};
        int erc = ST_DAF_LIMITS;  // outside the window: unreachable, the host keeps those objects out
        if (fast) {
            erc = pool_forces(plan, F, exact, xe, ve, cache, ev);
            if (F.ng.kind != 0 && erc == ST_OK && plan.sun_vel >= 0) {
                // non_grav_accel relative to the Sun (acceleration.rs:161-165)
                // (inline for the JPL comet model without delay; a call for the delayed model
                // and dust)
                const double* sc = cache + 6 * plan.sun_vel * NODES_BLOCK;
                const double3 rp = make_double3(xe[0] - sc[0], xe[1] - sc[NODES_BLOCK],
                                                xe[2] - sc[2 * NODES_BLOCK]);
                const double3 rv = make_double3(ve[0] - sc[3 * NODES_BLOCK],
                                                ve[1] - sc[4 * NODES_BLOCK],
                                                ve[2] - sc[5 * NODES_BLOCK]);
                const double3 na = (F.ng.kind == 1 && F.ng.p(9) == 0.0)
                                       ? nongrav_terms<false>(F.ng, rp, rv)
                                       : nongrav_accel(F.ng, rp, rv);
                ev[0] += na.x;
                ev[1] += na.y;
                ev[2] += na.z;
            }
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
        if (!iter_round) {  // the initial exact evaluation (every lane evaluated one point)
            cnt.exact++;
            const double t = st[ST_T], tf = st[ST_TF];
            __syncwarp(gmask);
            if (lane < 3) st[ST_A + lane] = ev[lane == 0 ? 0 : (lane == 1 ? 1 : 2)];
            if (fabs(tf - t) < 1e-10) {
                __syncwarp(gmask);
                finish(ST_OK);
                continue;
            }
            failures = 0;
            start_step(copysign(0.1, tf - t), t, tf, false, 0.0);
            continue;
        }
        // ---- corrector iteration: exchange the 7 node evaluations, form g and b ----
        // (radau.rs:292-313).  Lanes 0-2 each own one component; every lane then reads the
        // new b for the convergence test.
        cnt.iterations++;
        se[3 * lane + 0] = ev[0];
        se[3 * lane + 1] = ev[1];
        se[3 * lane + 2] = ev[2];
        const double b6_old0 = sb[6], b6_old1 = sb[13], b6_old2 = sb[20];
        __syncwarp(gmask);
        {
            const double ac = st[ST_A + comp];
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
            const double h = st[ST_H], t = st[ST_T], tf = st[ST_TF];
            __syncwarp(gmask);  // every lane has read the step before lane 0 replaces it
            if (lane < 3) {
                // x += dx, v += dv with compensated (Kahan) summation; lane c owns component c
                const int c = lane;
                const double h2 = h * h;
                double dw = 0.0, du = 0.0;
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    const double bck = sb[7 * c + k];
                    dw += bck * c_tab.w[k];
                    du += bck * c_tab.u[k];
                }
                const double xc = st[ST_X + c], vc = st[ST_V + c], ac = st[ST_A + c];
                const double dx = vc * h + h2 * (ac * 0.5 + dw);
                const double dv = h * (ac + du);
                const double yx = dx - scmp[c], yv = dv - scmp[3 + c];
                const double tx = xc + yx, tv = vc + yv;
                scmp[c] = (tx - xc) - yx;
                scmp[3 + c] = (tv - vc) - yv;
                st[ST_X + c] = tx;
                st[ST_V + c] = tv;
                // the step-end lane's evaluation is the exact evaluation of the new state
                st[ST_A + c] = se[21 + c];
            }
            const double mb6 = fmax(fmax(fabs(b60), fabs(b61)), fabs(b62));
            const double r = pow(1e-6 * fmax(fmax(fem0, fem1), fem2) / mb6, 1.0 / 7.0);
            const double next_h = h * clampd(r, 0.25, 4.0);
            const double tn = t + h;
            if (lane == 0) {
                st[ST_T] = tn;
                st[ST_HP] = h;
                st[ST_H] = next_h;
            }
            const int se_rc = __shfl_sync(gmask, erc, 7, NODE_G);
            F.min_dist = __shfl_sync(gmask, F.min_dist, 7, NODE_G);
            F.min_id = __shfl_sync(gmask, F.min_id, 7, NODE_G);
            F.impact_id = __shfl_sync(gmask, F.impact_id, 7, NODE_G);
            __syncwarp(gmask);
            cnt.exact++;
            if (se_rc != ST_OK) {
                finish(se_rc);
                continue;
            }
            cnt.steps++;
            if (fabs(tn - tf) < 1e-12) {
                finish(ST_OK);
                continue;
            }
            failures = 0;
            start_step(next_h, tn, tf, true, h);
            continue;
        }
        if (se_lane) {  // iteration not converged: forget the step-end lane's record
            F.min_dist = saved_min;
            F.min_id = saved_min_id;
        }
        __syncwarp(gmask);
        if (iter >= 10) {  // step failed to converge (radau.rs:345) -> retry smaller
            failures += 1;
            if (failures > 10) {
                finish(ST_CONVERGENCE);
                continue;
            }
            const double h = st[ST_H] * 0.7, t = st[ST_T], tf = st[ST_TF];
            __syncwarp(gmask);  // read before lane 0 replaces the step
            start_step(h, t, tf, false, 0.0);
        }
    }
}

}  // namespace kb
