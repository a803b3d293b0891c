// fov.cuh -- field-of-view visibility of many objects in many rectangular fields.
//
// Restates FovLike::check_visible (kete_core/fov/fov_like.rs:134-192) with check_linear
// (:43-66), check_two_body (:71-85), the n-body branch (:90-108, finished by
// fov_nbody_finish_kernel after a batched Radau pass) and SphericalPolygon::contains
// (kete_core/fov/patches.rs:214-234).  States and observers are heliocentric ecliptic.
#pragma once
#include "common.cuh"
#include "fov_args.h"
#include "kepler.cuh"

namespace kb {


// SphericalPolygon::contains: inside when no edge normal has a negative (or -0.0) dot
// product; otherwise the distance to move inside, min(largest violation, |v|).
__device__ __forceinline__ bool rect_contains(const double* __restrict__ nrm, const double v[3],
                                              double& dist) {
    double closest = -INFINITY;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const double d = v[0] * nrm[3 * e] + v[1] * nrm[3 * e + 1] + v[2] * nrm[3 * e + 2];
        if (isnan(d)) {
            dist = d;
            return false;
        }
        if (signbit(d) && fabs(d) > closest) closest = fabs(d);
    }
    if (isfinite(closest)) {
        dist = fmin(closest, norm3(v[0], v[1], v[2]));
        return false;
    }
    dist = 0.0;
    return true;
}

// SphericalCone::contains (fov/patches.rs:300-337): the angle between the unit pointing and
// the normalised direction; outside, the distance to move into the cone.
__device__ __forceinline__ bool cone_contains(const double* __restrict__ prm, const double v[3],
                                              double& dist) {
    const double r = norm3(v[0], v[1], v[2]);
    const double d = fabs(acos(prm[0] * (v[0] / r) + prm[1] * (v[1] / r) + prm[2] * (v[2] / r)));
    if (d <= prm[3]) {
        dist = 0.0;
        return true;
    }
    const double min_angle = fabs(d - prm[3]);
    dist = min_angle > 1.5707963267948966 ? r : sin(min_angle) * r;
    return false;
}

// The containment test of one field row by its patch kind (OmniDirectional::contains,
// fov/generic.rs:123-125, is always inside).
__device__ __forceinline__ bool patch_contains(const double* __restrict__ f, const double v[3],
                                               double& dist) {
    const int kind = (int)f[FOV_KIND_ROW];
    if (kind == 1) return cone_contains(f + 7, v, dist);
    if (kind == 2) {
        dist = 0.0;
        return true;
    }
    return rect_contains(f + 7, v, dist);
}

// check_two_body: Kepler to the observer epoch, back by the light time, Kepler again.
__device__ __forceinline__ int fov_two_body(const double* __restrict__ f, double jd,
                                            const double pos[3], const double vel[3], bool& inside,
                                            double& dist, double fin[7]) {
    double p[3] = {pos[0], pos[1], pos[2]}, v[3] = {vel[0], vel[1], vel[2]};
    const double ojd = f[0];
    int rc = analytic_2_body(ojd - jd, p, v);
    if (rc != ST_OK) return rc;
    const double dt = -norm3(p[0] - f[1], p[1] - f[2], p[2] - f[3]) * C_AU_PER_DAY_INV;
    const double t2 = ojd + dt;
    rc = analytic_2_body(t2 - ojd, p, v);
    if (rc != ST_OK) return rc;
    const double rel[3] = {p[0] - f[1], p[1] - f[2], p[2] - f[3]};
    inside = patch_contains(f, rel, dist);
    fin[0] = t2;
    fin[1] = p[0]; fin[2] = p[1]; fin[3] = p[2];
    fin[4] = v[0]; fin[5] = v[1]; fin[6] = v[2];
    return ST_OK;
}

__device__ __forceinline__ void fov_emit(const FovArgs& a, int f, int64_t i, const double fin[7]) {
    const unsigned long long k = atomicAdd(&a.counters[0], 1ULL);
    if ((int64_t)k < a.capacity) {
        a.out_fov[k] = f;
        a.out_obj[k] = (int32_t)i;
#pragma unroll
        for (int q = 0; q < 7; ++q) a.out_state[(int64_t)q * a.capacity + k] = fin[q];
    }
}

// One thread per object, looping over a tile of fields staged in shared memory.
__global__ void __launch_bounds__(128) fov_prefilter_kernel(FovArgs a) {
    __shared__ double s_f[FOV_TILE * FOV_STRIDE];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < a.n_obj && (a.valid == nullptr || a.valid[i]);
    double pos[3] = {0, 0, 0}, vel[3] = {0, 0, 0}, jd = 0.0;
    if (active) {
        pos[0] = a.pos[i]; pos[1] = a.pos[a.n_obj + i]; pos[2] = a.pos[2 * a.n_obj + i];
        vel[0] = a.vel[i]; vel[1] = a.vel[a.n_obj + i]; vel[2] = a.vel[2 * a.n_obj + i];
        jd = a.jd[i];
    }
    for (int64_t base = 0; base < a.n_fov; base += FOV_TILE) {
        const int nt = (int)((a.n_fov - base) < FOV_TILE ? (a.n_fov - base) : FOV_TILE);
        __syncthreads();
        for (int q = threadIdx.x; q < nt * FOV_STRIDE; q += blockDim.x) {
            const int f = q / FOV_STRIDE, c = q % FOV_STRIDE;
            s_f[q] = a.fov[(int64_t)c * a.n_fov + base + f];
        }
        __syncthreads();
        if (!active) continue;
        for (int t = 0; t < nt; ++t) {
            const double* f = s_f + t * FOV_STRIDE;
            const double dvx = vel[0] - f[4], dvy = vel[1] - f[5], dvz = vel[2] - f[6];
            const double max_dist = norm3(dvx, dvy, dvz) * a.dt_limit * 2.0;
            double dist;
            double fin[7];
            bool inside;
            if (fabs(jd - f[0]) < a.dt_limit) {
                // check_linear: first-order light delay, straight-line motion
                const double rel0 = pos[0] - f[1], rel1 = pos[1] - f[2], rel2 = pos[2] - f[3];
                const double dt = f[0] - jd - norm3(rel0, rel1, rel2) * C_AU_PER_DAY_INV;
                const double nrel[3] = {pos[0] + vel[0] * dt - f[1], pos[1] + vel[1] * dt - f[2],
                                        pos[2] + vel[2] * dt - f[3]};
                if (!patch_contains(f, nrel, dist) && dist > max_dist) continue;
                if (fov_two_body(f, jd, pos, vel, inside, dist, fin) == ST_OK && inside)
                    fov_emit(a, (int)(base + t), i, fin);
            } else {
                if (fov_two_body(f, jd, pos, vel, inside, dist, fin) != ST_OK) continue;
                if (!inside && dist > max_dist) continue;
                const unsigned long long k = atomicAdd(&a.counters[1], 1ULL);
                if ((int64_t)k < a.cand_capacity) {
                    a.cand_fov[k] = (int32_t)(base + t);
                    a.cand_obj[k] = (int32_t)i;
                }
            }
        }
    }
}

// Appends (f, i) for every lane of the warp with `take` set, one atomic per warp.
__device__ __forceinline__ void fov_append_pair(const FovArgs& a, bool take, int f, int64_t i) {
    const unsigned active = __activemask();
    const unsigned want = __ballot_sync(active, take);
    if (!want) return;
    const int leader = __ffs(want) - 1;
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(&a.counters[2], (unsigned long long)__popc(want));
    base = __shfl_sync(active, base, leader);
    if (take) {
        const unsigned long long k = base + __popc(want & ((1u << lane) - 1u));
        if ((int64_t)k < a.pair_capacity) {
            a.pair_fov[k] = f;
            a.pair_obj[k] = (int32_t)i;
        }
    }
}

// Two-pass form of fov_prefilter_kernel.  First pass: one thread per object over tiles of
// fields, the first-order linear screen of check_linear only (a few dozen uniform FP64
// operations per pair); the pairs that pass are appended to a list.  Fields at least
// dt_limit away from the object's epoch take check_visible's n-body branch here as in
// fov_prefilter_kernel (its two-body screen in place), which the fov_state_check schedule
// never reaches.  The second pass (fov_pairs_kernel) runs the two-body light-time solve on the
// listed pairs only, one thread per pair, so the solve's Newton iterations no longer leave the
// lanes of screened-out pairs idle.
__global__ void __launch_bounds__(128) fov_screen_kernel(FovArgs a) {
    __shared__ double s_f[FOV_TILE * FOV_STRIDE];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < a.n_obj && (a.valid == nullptr || a.valid[i]);
    double pos[3] = {0, 0, 0}, vel[3] = {0, 0, 0}, jd = 0.0;
    if (active) {
        pos[0] = a.pos[i]; pos[1] = a.pos[a.n_obj + i]; pos[2] = a.pos[2 * a.n_obj + i];
        vel[0] = a.vel[i]; vel[1] = a.vel[a.n_obj + i]; vel[2] = a.vel[2 * a.n_obj + i];
        jd = a.jd[i];
    }
    for (int64_t base = 0; base < a.n_fov; base += FOV_TILE) {
        const int nt = (int)((a.n_fov - base) < FOV_TILE ? (a.n_fov - base) : FOV_TILE);
        __syncthreads();
        for (int q = threadIdx.x; q < nt * FOV_STRIDE; q += blockDim.x) {
            const int f = q / FOV_STRIDE, c = q % FOV_STRIDE;
            s_f[q] = a.fov[(int64_t)c * a.n_fov + base + f];
        }
        __syncthreads();
        for (int t = 0; t < nt; ++t) {
            const double* f = s_f + t * FOV_STRIDE;
            bool take = false;
            if (active) {
                const double dvx = vel[0] - f[4], dvy = vel[1] - f[5], dvz = vel[2] - f[6];
                const double max_dist = norm3(dvx, dvy, dvz) * a.dt_limit * 2.0;
                if (fabs(jd - f[0]) < a.dt_limit) {
                    // check_linear: first-order light delay, straight-line motion
                    const double rel0 = pos[0] - f[1], rel1 = pos[1] - f[2], rel2 = pos[2] - f[3];
                    const double dt = f[0] - jd - norm3(rel0, rel1, rel2) * C_AU_PER_DAY_INV;
                    const double nrel[3] = {pos[0] + vel[0] * dt - f[1],
                                            pos[1] + vel[1] * dt - f[2],
                                            pos[2] + vel[2] * dt - f[3]};
                    double dist;
                    take = patch_contains(f, nrel, dist) || !(dist > max_dist);
                } else {
                    double dist, fin[7];
                    bool inside;
                    if (fov_two_body(f, jd, pos, vel, inside, dist, fin) == ST_OK &&
                        (inside || !(dist > max_dist))) {
                        const unsigned long long k = atomicAdd(&a.counters[1], 1ULL);
                        if ((int64_t)k < a.cand_capacity) {
                            a.cand_fov[k] = (int32_t)(base + t);
                            a.cand_obj[k] = (int32_t)i;
                        }
                    }
                }
            }
            fov_append_pair(a, take, (int)(base + t), i);
        }
    }
}

// Second pass: check_two_body for every screened pair (one thread per pair); visible pairs
// are emitted as in fov_prefilter_kernel.
__global__ void __launch_bounds__(128) fov_pairs_kernel(FovArgs a, int64_t m) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int f = a.pair_fov[k];
    const int64_t i = a.pair_obj[k];
    double fcol[FOV_STRIDE];
#pragma unroll
    for (int c = 0; c < FOV_STRIDE; ++c) fcol[c] = a.fov[(int64_t)c * a.n_fov + f];
    const double pos[3] = {a.pos[i], a.pos[a.n_obj + i], a.pos[2 * a.n_obj + i]};
    const double vel[3] = {a.vel[i], a.vel[a.n_obj + i], a.vel[2 * a.n_obj + i]};
    double dist, fin[7];
    bool inside;
    if (fov_two_body(fcol, a.jd[i], pos, vel, inside, dist, fin) == ST_OK && inside)
        fov_emit(a, f, i, fin);
}

// Gather the n-body candidates' states (object state, target epoch = observer epoch).
__global__ void fov_gather_kernel(FovArgs a, int64_t m, double* __restrict__ gpos,
                                  double* __restrict__ gvel, double* __restrict__ gjd0,
                                  double* __restrict__ gjd1) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int64_t i = a.cand_obj[k];
    const int f = a.cand_fov[k];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        gpos[c * m + k] = a.pos[c * a.n_obj + i];
        gvel[c * m + k] = a.vel[c * a.n_obj + i];
    }
    gjd0[k] = a.jd[i];
    gjd1[k] = a.fov[f];  // row 0 = observer jd
}

// check_n_body after the Radau pass: light delay by two-body, then containment.
__global__ void fov_nbody_finish_kernel(FovArgs a, int64_t m, const double* __restrict__ npos,
                                        const double* __restrict__ nvel,
                                        const int32_t* __restrict__ nst) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m || nst[k] != ST_OK) return;
    const int f = a.cand_fov[k];
    double fcol[FOV_STRIDE];
#pragma unroll
    for (int c = 0; c < FOV_STRIDE; ++c) fcol[c] = a.fov[(int64_t)c * a.n_fov + f];
    double p[3] = {npos[k], npos[m + k], npos[2 * m + k]};
    double v[3] = {nvel[k], nvel[m + k], nvel[2 * m + k]};
    const double ojd = fcol[0];
    const double dt = -norm3(p[0] - fcol[1], p[1] - fcol[2], p[2] - fcol[3]) * C_AU_PER_DAY_INV;
    const double t2 = ojd + dt;
    if (analytic_2_body(t2 - ojd, p, v) != ST_OK) return;
    const double rel[3] = {p[0] - fcol[1], p[1] - fcol[2], p[2] - fcol[3]};
    double dist;
    if (!patch_contains(fcol, rel, dist)) return;
    const double fin[7] = {t2, p[0], p[1], p[2], v[0], v[1], v[2]};
    fov_emit(a, f, a.cand_obj[k], fin);
}

// FovLike::check_static (fov/fov_like.rs:228-250 through contains): which fields contain
// each fixed direction (observer to target, heliocentric ecliptic).  One thread per
// direction, looping over tiles of fields staged in shared memory; every (field, direction)
// pair inside is appended at an atomic counter (pairs beyond `capacity` are counted, not
// written).
__global__ void __launch_bounds__(128) fov_contains_kernel(int64_t n_vec, const double* __restrict__ vec,
                                                           int64_t n_fov, const double* __restrict__ fov,
                                                           int64_t capacity,
                                                           unsigned long long* __restrict__ counter,
                                                           int32_t* __restrict__ out_fov,
                                                           int32_t* __restrict__ out_idx) {
    __shared__ double s_f[FOV_TILE * FOV_STRIDE];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n_vec;
    double v[3] = {0.0, 0.0, 0.0};
    if (active) {
        v[0] = vec[i];
        v[1] = vec[n_vec + i];
        v[2] = vec[2 * n_vec + i];
    }
    for (int64_t base = 0; base < n_fov; base += FOV_TILE) {
        const int nt = (int)((n_fov - base) < FOV_TILE ? (n_fov - base) : FOV_TILE);
        __syncthreads();
        for (int q = threadIdx.x; q < nt * FOV_STRIDE; q += blockDim.x) {
            const int f = q / FOV_STRIDE, c = q % FOV_STRIDE;
            s_f[q] = fov[(int64_t)c * n_fov + base + f];
        }
        __syncthreads();
        if (!active) continue;
        for (int t = 0; t < nt; ++t) {
            double dist;
            if (!patch_contains(s_f + t * FOV_STRIDE, v, dist)) continue;
            const unsigned long long k = atomicAdd(counter, 1ULL);
            if ((int64_t)k < capacity) {
                out_fov[k] = (int32_t)(base + t);
                out_idx[k] = (int32_t)i;
            }
        }
    }
}

}  // namespace kb
