// long.cu -- system integration (propagate_n_body_long, long.cuh) and its host launcher.
#include "common.cuh"
#include "forces.cuh"
#include "internal.h"
#include "long.cuh"

namespace kb {
KB_CONSTANT_UPLOADER(long)
}  // namespace kb

namespace kb {

int launch_nbody_long(const LongArgs& a, cudaStream_t stream) {
    if (a.n <= 0 || a.batch < 1 || a.batch > 64 - LONG_MASSIVE) return 0;  // checked by the caller
    const int64_t n_batch = (a.n + a.batch - 1) / a.batch;
    // the seven nodes in parallel when all batches fit on the GPU at once: the node form
    // cuts each batch's latency, but its blocks are seven times larger, so beyond one wave
    // the one-thread-per-body form finishes first
    int dev = 0, sms = 0, per_sm = 0;
    int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (rc) return rc;
    if ((rc = cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attr")))
        return rc;
    if ((rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                             &per_sm, nbody_long_nodes_kernel, 32 * LN_WARPS, 0),
                         "occupancy")))
        return rc;
    if (LONG_MASSIVE + a.batch <= LN_BODIES && n_batch <= (int64_t)sms * per_sm) {
        nbody_long_nodes_kernel<<<(unsigned)n_batch, 32 * LN_WARPS, 0, stream>>>(a);
        return launched(1, "nbody_long_nodes_kernel launch");
    }
    const int block = LONG_MASSIVE + a.batch <= 32 ? 32 : 64;
    nbody_long_kernel<<<(unsigned)n_batch, block, 0, stream>>>(a);
    return launched(1, "nbody_long_kernel launch");
}

}  // namespace kb

namespace kb {

// -------------------------------------------------------------------------------------------
// The accelerations on their own, at n points: spk_accel (acceleration.rs:121-168, the
// perturbers' states from the device SPK, the force code of the propagation kernels) and
// vec_accel (acceleration.rs:197-249) on test particles under massive bodies whose states
// the caller gives (the system integration's force code, long_pair, for SIMPLE_PLANETS; the
// propagation kernels' per-body term for PLANETS / MASSES).  Positions and velocities are
// relative to the solar-system barycentre in the equatorial frame, AU and AU/day.
// -------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) spk_accel_kernel(AccelArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t n = a.n;
    SpkForceUnrolled F;
    F.n_force = a.n_force;
    F.ng.base = a.nongrav ? a.nongrav + i : nullptr;
    F.ng.stride = n;
    F.ng.kind = a.nongrav ? (int)a.nongrav[i] : 0;
    F.impact_id = 0;
    F.min_dist = 1e300;
    F.min_id = 0;
    const double x[3] = {a.pos[i], a.pos[n + i], a.pos[2 * n + i]};
    const double v[3] = {a.vel[i], a.vel[n + i], a.vel[2 * n + i]};
    double acc[3] = {0.0, 0.0, 0.0};
    const int rc = F.eval(a.exact != 0, a.jd[i], x, v, acc);
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int c = 0; c < 3; ++c) a.out[c * n + i] = rc == ST_OK ? acc[c] : nan;
    a.status[i] = rc;
    if (a.impact_id) a.impact_id[i] = rc == ST_IMPACT ? F.impact_id : 0;
}

__global__ void __launch_bounds__(128) vec_accel_kernel(AccelArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t n = a.n;
    const int m = a.n_massive;
    const double x[3] = {a.pos[i], a.pos[n + i], a.pos[2 * n + i]};
    const double v[3] = {a.vel[i], a.vel[n + i], a.vel[2 * n + i]};
    NonGrav ng;
    ng.base = a.nongrav ? a.nongrav + i : nullptr;
    ng.stride = n;
    ng.kind = a.nongrav ? (int)a.nongrav[i] : 0;
    SpkForceUnrolled F;
    F.n_force = 0;
    F.ng = ng;
    F.impact_id = 0;
    F.min_dist = 1e300;
    F.min_id = 0;
    double acc[3] = {0.0, 0.0, 0.0};
    int rc = ST_OK;
    for (int k = 0; k < m && rc == ST_OK; ++k) {
        const double bp[3] = {a.massive[k], a.massive[m + k], a.massive[2 * m + k]};
        const double bv[3] = {a.massive[3 * m + k], a.massive[4 * m + k], a.massive[5 * m + k]};
        if (a.simple) {  // SIMPLE_PLANETS: the system integration's pair term
            const double rp[3] = {x[0] - bp[0], x[1] - bp[1], x[2] - bp[2]};
            const double rv[3] = {v[0] - bv[0], v[1] - bv[1], v[2] - bv[2]};
            if (a.exact && norm3(rp[0], rp[1], rp[2]) <= c_tab.simple_radius[k]) {
                F.impact_id = c_tab.simple_naif[k];
                rc = ST_IMPACT;
                break;
            }
            double w[3] = {0.0, 0.0, 0.0};
            long_pair(k, rp, rv, w);
            if (c_tab.simple_naif[k] == 10 && ng.kind != 0) {
                const double3 na = nongrav_accel(ng, make_double3(rp[0], rp[1], rp[2]),
                                                 make_double3(rv[0], rv[1], rv[2]));
                w[0] += na.x;
                w[1] += na.y;
                w[2] += na.z;
            }
            acc[0] += w[0];
            acc[1] += w[1];
            acc[2] += w[2];
        } else {  // PLANETS / MASSES: the propagation kernels' per-body term
            double w0 = 0.0, w1 = 0.0, w2 = 0.0;
            rc = F.body<true>(a.bodies[k], a.exact != 0, x, v, bp, bv, w0, w1, w2);
            acc[0] += w0;
            acc[1] += w1;
            acc[2] += w2;
        }
    }
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int c = 0; c < 3; ++c) a.out[c * n + i] = rc == ST_OK ? acc[c] : nan;
    a.status[i] = rc;
    if (a.impact_id) a.impact_id[i] = rc == ST_IMPACT ? F.impact_id : 0;
}

int launch_accel(const AccelArgs& a, bool vec, cudaStream_t stream) {
    if (a.n <= 0) return 0;
    const unsigned grid = (unsigned)((a.n + 127) / 128);
    if (vec) {
        vec_accel_kernel<<<grid, 128, 0, stream>>>(a);
        return launched(1, "vec_accel_kernel launch");
    }
    spk_accel_kernel<<<grid, 128, 0, stream>>>(a);
    return launched(1, "spk_accel_kernel launch");
}

}  // namespace kb
