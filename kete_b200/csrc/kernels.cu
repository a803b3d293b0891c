// kernels.cu -- two-body, thread-per-object N-body Radau, ephemeris queries, processing
// order, flux, FOV and two-body STM kernels with their host launchers.  The node-parallel
// Radau launchers (nodes.cu), the sensitivity kernels (sens.cu, adjoint.cu) and system integration
// (long.cu) are translation units of their own; each carries its own copy of the device
// constants, which upload_tables / upload_ephem write to all of them.
#include <atomic>
#include <cstdio>

#include "common.cuh"
#include "ephem.cuh"
#include "forces.cuh"
#include "internal.h"
#include "kepler.cuh"
#include "radau.cuh"

namespace kb {

// Kernels launched by this library since it was loaded (kete_b200_kernel_launches): every
// launch helper below adds the kernels it enqueued when it checks the launch.
std::atomic<int64_t> g_kernel_launches{0};
std::atomic<int64_t> g_device_allocations{0};

KB_CONSTANT_UPLOADER(kernels)

int upload_tables(const Tables& t) {
    int rc = 0;
    for (auto up : {upload_consts_kernels, upload_consts_nodes, upload_consts_sens,
                    upload_consts_adjoint, upload_consts_long})
        if ((rc = up(&t, nullptr))) return rc;
    return 0;
}
int upload_ephem(const EphemConst& e) {
    int rc = 0;
    for (auto up : {upload_consts_kernels, upload_consts_nodes, upload_consts_sens,
                    upload_consts_adjoint, upload_consts_long})
        if ((rc = up(nullptr, &e))) return rc;
    return 0;
}

// -------------------------------------------------------------------------------------------
// two-body (kete_core/propagation/kepler.rs:306-322 with the light-delay second pass of the
// PyO3 binding, src/kete/rust/kepler.rs:89-102).  One thread per object, SoA FP64.
// -------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) two_body_kernel(
    int64_t n, const double* __restrict__ pos, const double* __restrict__ vel,
    const double* __restrict__ jd0, const double* __restrict__ jd1,
    const double* __restrict__ obs, double* __restrict__ out_pos, double* __restrict__ out_vel,
    double* __restrict__ out_jd, int32_t* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double p[3] = {pos[i], pos[n + i], pos[2 * n + i]};
    double v[3] = {vel[i], vel[n + i], vel[2 * n + i]};
    const double t0 = jd0[i], t1 = jd1[i];
    double tj = t1;
    int rc = analytic_2_body(t1 - t0, p, v);
    if (rc == ST_OK && obs != nullptr) {
        const double o0 = obs[0], o1 = obs[1], o2 = obs[2];
        const double delay = -norm3(p[0] - o0, p[1] - o1, p[2] - o2) / C_AU_PER_DAY;
        const double t2 = tj + delay;
        rc = analytic_2_body(t2 - tj, p, v);
        tj = t2;
    }
    if (rc != ST_OK) {
        p[0] = p[1] = p[2] = v[0] = v[1] = v[2] = __longlong_as_double(0x7ff8000000000000LL);
        tj = t1;
    }
    out_pos[i] = p[0];
    out_pos[n + i] = p[1];
    out_pos[2 * n + i] = p[2];
    out_vel[i] = v[0];
    out_vel[n + i] = v[1];
    out_vel[2 * n + i] = v[2];
    if (out_jd) out_jd[i] = tj;
    status[i] = rc;
}

int launch_two_body(int64_t n, const double* pos, const double* vel, const double* jd0,
                    const double* jd1, const double* obs, double* out_pos, double* out_vel,
                    double* out_jd, int32_t* status, cudaStream_t stream) {
    if (n <= 0) return 0;
    const int block = 128;
    const int64_t grid = (n + block - 1) / block;
    two_body_kernel<<<(unsigned)grid, block, 0, stream>>>(n, pos, vel, jd0, jd1, obs, out_pos,
                                                          out_vel, out_jd, status);
    return launched(1, "two_body_kernel launch");
}

// -------------------------------------------------------------------------------------------
// N-body Radau, one object per thread (the plain form of propagate_n_body_spk,
// kete_core/propagation/mod.rs:70-118).
// -------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) nbody_thread_kernel(NBodyArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t n = a.n;
    RadauObj s;
    s.t = a.jd0[i];
    const double tf = a.jd1[i];
    s.x[0] = a.pos[i]; s.x[1] = a.pos[n + i]; s.x[2] = a.pos[2 * n + i];
    s.v[0] = a.vel[i]; s.v[1] = a.vel[n + i]; s.v[2] = a.vel[2 * n + i];
    SpkForceUnrolled F;  // one object per thread: fully unrolled Chebyshev loops
    F.n_force = a.n_force;
    F.ng.base = a.nongrav ? a.nongrav + i : nullptr;
    F.ng.stride = n;
    F.ng.kind = a.nongrav ? (int)a.nongrav[i] : 0;
    F.impact_id = 0;
    F.min_dist = 1e300;
    F.min_id = 0;
    RadauCounters cnt;
    int rc = ST_OK;
    bool finite = isfinite(s.x[0]) && isfinite(s.x[1]) && isfinite(s.x[2]) && isfinite(s.v[0]) &&
                  isfinite(s.v[1]) && isfinite(s.v[2]) && isfinite(s.t);
    if (!finite) rc = ST_VALUE_ERROR;
    if (rc == ST_OK) rc = to_ssb_equatorial(s.t, a.frame, a.chain, s.x, s.v);
    if (rc == ST_OK) rc = radau_integrate(s, tf, F, cnt, a.max_loops);
    if (rc == ST_OK) rc = from_ssb_equatorial(tf, a.frame, a.chain, s.x, s.v);
    if (rc != ST_OK) {
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        s.x[0] = s.x[1] = s.x[2] = s.v[0] = s.v[1] = s.v[2] = nan;
    }
    a.out_pos[i] = s.x[0]; a.out_pos[n + i] = s.x[1]; a.out_pos[2 * n + i] = s.x[2];
    a.out_vel[i] = s.v[0]; a.out_vel[n + i] = s.v[1]; a.out_vel[2 * n + i] = s.v[2];
    a.status[i] = rc;
    if (a.impact_id) a.impact_id[i] = rc == ST_IMPACT ? F.impact_id : 0;
    if (a.impact_jd) a.impact_jd[i] = rc == ST_IMPACT ? s.t : 0.0;
    if (a.min_dist) a.min_dist[i] = F.min_dist;
    if (a.counters) {
        a.counters[i] = cnt.steps;
        a.counters[n + i] = cnt.iterations;
        a.counters[2 * n + i] = cnt.exact;
    }
}

int launch_nbody_thread(const NBodyArgs& a, int block, cudaStream_t stream) {
    if (a.n <= 0) return 0;
    if (block <= 0) block = 128;
    const int64_t grid = (a.n + block - 1) / block;
    nbody_thread_kernel<<<(unsigned)grid, block, 0, stream>>>(a);
    return launched(1, "nbody_thread_kernel launch");
}

// -------------------------------------------------------------------------------------------
// Radau with the central force only (propagate_two_body_radau / propagation_central,
// kete_core/propagation/mod.rs:35-46,126-138): checks the integrator in isolation.
// -------------------------------------------------------------------------------------------
__global__ void radau_central_kernel(int64_t n, const double* pos, const double* vel,
                                     const double* t0, const double* t1, double* out_pos,
                                     double* out_vel, int32_t* status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    RadauObj s;
    s.t = t0[i];
    s.x[0] = pos[i]; s.x[1] = pos[n + i]; s.x[2] = pos[2 * n + i];
    s.v[0] = vel[i]; s.v[1] = vel[n + i]; s.v[2] = vel[2 * n + i];
    CentralForce F;
    F.impact_id = 0;
    F.min_dist = 0.0;
    F.min_id = 0;
    RadauCounters cnt;
    int rc = radau_integrate(s, t1[i], F, cnt, 1 << 20);
    out_pos[i] = s.x[0]; out_pos[n + i] = s.x[1]; out_pos[2 * n + i] = s.x[2];
    out_vel[i] = s.v[0]; out_vel[n + i] = s.v[1]; out_vel[2 * n + i] = s.v[2];
    status[i] = rc;
}

int launch_radau_central(int64_t n, const double* pos, const double* vel, const double* t0,
                         const double* t1, double* out_pos, double* out_vel, int32_t* status,
                         cudaStream_t stream) {
    if (n <= 0) return 0;
    const int block = 128;
    radau_central_kernel<<<(unsigned)((n + block - 1) / block), block, 0, stream>>>(
        n, pos, vel, t0, t1, out_pos, out_vel, status);
    return launched(1, "radau_central_kernel launch");
}

// -------------------------------------------------------------------------------------------
// batched SpkCollection::try_get_state (spk.rs:87-96): state of body `slot` (chained to the
// barycentre) minus the centre chain, in `frame`.
// -------------------------------------------------------------------------------------------
constexpr int SPK_BLOCK = 64;
__global__ void __launch_bounds__(SPK_BLOCK) spk_states_kernel(int64_t n, int32_t slot,
                                                               const double* jd,
                                                               CenterChain center_chain,
                                                               int frame, double* out6,
                                                               int32_t* status) {
    // the modified-difference work arrays of types 1/21 (76 doubles a thread) in shared
    // memory rather than local memory
    __shared__ double s_work[76 * SPK_BLOCK];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double t = jd[i];
    double p[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    int rc = ST_OK;
    // the body's own chain: raw(body) + raw(parent) ...
    int s = slot;
    for (int k = 0; k < 3 && s >= 0 && rc == ST_OK; ++k) {
        double sp[3], sv[3];
        rc = eph_raw(c_eph, s, t, sp, sv, s_work + threadIdx.x, SPK_BLOCK);
        for (int q = 0; q < 3; ++q) {
            p[q] += sp[q];
            v[q] += sv[q];
        }
        s = c_eph.slot[s].parent_slot;
    }
    if (s < -1 || s >= 0) rc = ST_DAF_LIMITS;  // centre chain not complete
    if (rc == ST_OK) rc = from_ssb_equatorial(t, frame, center_chain, p, v);
    for (int q = 0; q < 3; ++q) {
        out6[q * n + i] = p[q];
        out6[(3 + q) * n + i] = v[q];
    }
    status[i] = rc;
}

int launch_spk_states(int64_t n, int32_t slot, const double* jd,
                      const CenterChain& center_chain, int frame, double* out6, int32_t* status,
                      cudaStream_t stream) {
    if (n <= 0) return 0;
    const int block = SPK_BLOCK;
    spk_states_kernel<<<(unsigned)((n + block - 1) / block), block, 0, stream>>>(
        n, slot, jd, center_chain, frame, out6, status);
    return launched(1, "spk_states_kernel launch");
}

}  // namespace kb

namespace kb {

// -------------------------------------------------------------------------------------------
// FP64 pipe probe: independent DFMA chains, for the roofline denominator.  Each thread
// runs 16 independent accumulators for `iters` iterations (2 flops per FMA).
// -------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) dfma_probe_kernel(int64_t iters, double seed, double* out) {
    double a[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = seed + threadIdx.x * 1e-9 + k * 1e-7;
    const double m = 0.999999999, c = 1e-9;
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) a[k] = fma(a[k], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += a[k];
    if (s == 12345.678) out[0] = s;  // practically never true; keeps the chains live
}

int fp64_probe(int64_t iters, double* tflops, float* ms_out) {
    int dev = 0, sms = 0;
    int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (rc) return rc;
    if ((rc = cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attr")))
        return rc;
    double* d_out = nullptr;
    if ((rc = cuda_check(counted_malloc((void**)&d_out, sizeof(double)), "cudaMalloc probe"))) return rc;
    const int block = 256, grid = sms * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    dfma_probe_kernel<<<grid, block>>>(iters / 10, 1.0, d_out);  // warm-up
    cudaEventRecord(e0);
    dfma_probe_kernel<<<grid, block>>>(iters, 1.0, d_out);
    cudaEventRecord(e1);
    rc = cuda_check(cudaEventSynchronize(e1), "probe synchronize");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_out);
    if (rc) return rc;
    const double flops = 2.0 * 16.0 * (double)iters * (double)grid * (double)block;
    *tflops = flops / (ms * 1e-3) / 1e12;
    if (ms_out) *ms_out = ms;
    return 0;
}

}  // namespace kb

namespace kb {

// -------------------------------------------------------------------------------------------
// Processing order of the node kernel: objects with the most work first, where the work is
// the integration span in units of the object's orbital period (span x two-body mean motion
// from the vis-viva energy; r^-1.5 for unbound orbits), since the Radau steps scale with
// the orbit.  With a persistent grid the groups that finish early pick up the small ones
// and the tail is short; with one group per object, neighbours in a warp get similar work,
// so the warp-synchronous forms' groups wait less for each other.  Work is bucketed on a
// log2 scale (quarter-octave classes from 2^-8 to 2^7 radians, each split by the direction
// of integration); within a bucket the order is whatever the atomics give -- it does not
// affect any object's result.
//
// The warp-pooled node kernel evaluates the ephemeris from the fast plan's records alone, so
// the objects whose span [jd0, jd1] does not lie inside the plan's window (with a margin of
// 1e-6 day: every evaluation time of a Radau integration lies between jd0 and jd1 up to
// rounding) go to one last bucket.  Before it, one bucket holds the objects with a
// non-gravitational model (given ng), which the pooled kernel integrates on a few SMs of
// their own: the model's code, fetched by any warp of an SM, evicts the step loop from the
// SM's instruction cache.  The header's range {0, ng start, outside start, n} splits the
// order.  Callers without a window pass [-inf, inf] and ng = null.
//
// Scratch layout (ints): [0] object queue, [1..ORDER_ALL_BUCKETS] bucket histogram, then the
// bucket cursors, the range at ORDER_RANGE, further queues at ORDER_QUEUE2 and ORDER_QUEUE3,
// then order[n] from int offset ORDER_SCRATCH_HEADER.
// -------------------------------------------------------------------------------------------
static_assert(ORDER_QUEUE3 + 1 <= ORDER_SCRATCH_HEADER, "order header too small");

__device__ __forceinline__ bool in_window(double jd0, double jd1, double lo, double hi) {
    constexpr double MARGIN = 1e-6;  // NaN epochs compare false: outside
    return jd0 >= lo + MARGIN && jd1 >= lo + MARGIN && jd0 <= hi - MARGIN && jd1 <= hi - MARGIN;
}

__device__ __forceinline__ int work_bucket(int64_t i, int64_t n, const double* __restrict__ pos,
                                           const double* __restrict__ vel, double jd0, double jd1) {
    const double span = fabs(jd1 - jd0);
    const double px = pos[i], py = pos[n + i], pz = pos[2 * n + i];
    const double vx = vel[i], vy = vel[n + i], vz = vel[2 * n + i];
    const double r = sqrt(px * px + py * py + pz * pz);
    const double inv_a = 2.0 / r - (vx * vx + vy * vy + vz * vz) / GMS;
    const double mean_motion = inv_a > 0.0 ? sqrt(GMS * inv_a * inv_a * inv_a) : sqrt(GMS / (r * r * r));
    const double work = span * mean_motion;
    if (!(work > 0.0) || !isfinite(work)) return ORDER_BUCKETS - 1;  // no work, NaN last
    // quarter-octave work classes, most work first; within a class the objects integrated
    // forwards in time come before those integrated backwards, so that neighbours in the
    // order (the lane groups of a warp, the groups of a block) also move through the
    // ephemeris in the same direction and share more of its records
    constexpr int CLASSES = ORDER_BUCKETS / 2;
    const int b = (int)floor(log2(work) * 4.0) + 32;
    const int cls = CLASSES - 1 - (b < 0 ? 0 : (b > CLASSES - 1 ? CLASSES - 1 : b));
    return 2 * cls + (jd1 < jd0 ? 1 : 0);
}

__device__ __forceinline__ int order_bucket(int64_t i, int64_t n, const double* __restrict__ pos,
                                            const double* __restrict__ vel, double t0, double t1,
                                            double lo, double hi, const double* __restrict__ ng) {
    if (!in_window(t0, t1, lo, hi)) return ORDER_OUT_BUCKET;
    if (ng && ng[i] != 0.0) return ORDER_NG_BUCKET;
    return work_bucket(i, n, pos, vel, t0, t1);
}

__global__ void order_hist_kernel(int64_t n, const double* __restrict__ pos,
                                  const double* __restrict__ vel, const double* __restrict__ jd0,
                                  const double* __restrict__ jd1, double lo, double hi,
                                  const double* __restrict__ ng, int* __restrict__ scratch) {
    __shared__ int h[ORDER_ALL_BUCKETS];
    for (int i = threadIdx.x; i < ORDER_ALL_BUCKETS; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&h[order_bucket(i, n, pos, vel, jd0[i], jd1[i], lo, hi, ng)], 1);
    __syncthreads();
    for (int i = threadIdx.x; i < ORDER_ALL_BUCKETS; i += blockDim.x)
        if (h[i]) atomicAdd(&scratch[1 + i], h[i]);
}

__global__ void order_scan_kernel(int* __restrict__ scratch) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int run = 0;
        for (int b = 0; b < ORDER_ALL_BUCKETS; ++b) {
            if (b == ORDER_NG_BUCKET) scratch[ORDER_RANGE + 1] = run;
            if (b == ORDER_OUT_BUCKET) scratch[ORDER_RANGE + 2] = run;  // objects inside the window
            scratch[1 + ORDER_ALL_BUCKETS + b] = run;
            run += scratch[1 + b];
        }
        scratch[ORDER_RANGE] = 0;
        scratch[ORDER_RANGE + 3] = run;
    }
}

__global__ void order_scatter_kernel(int64_t n, const double* __restrict__ pos,
                                     const double* __restrict__ vel, const double* __restrict__ jd0,
                                     const double* __restrict__ jd1, double lo, double hi,
                                     const double* __restrict__ ng, int* __restrict__ scratch,
                                     int32_t* __restrict__ order) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int b = order_bucket(i, n, pos, vel, jd0[i], jd1[i], lo, hi, ng);
        const int p = atomicAdd(&scratch[1 + ORDER_ALL_BUCKETS + b], 1);
        if (p >= 0 && p < n) order[p] = (int32_t)i;
    }
}

int preload_order_kernels() {
    cudaFuncAttributes fa;
    int rc = 0;
    for (const void* f : {(const void*)order_hist_kernel, (const void*)order_scan_kernel,
                          (const void*)order_scatter_kernel})
        if ((rc = cuda_check(cudaFuncGetAttributes(&fa, f), "load ordering kernels"))) return rc;
    return 0;
}

// Zero the header, histogram the work, scan, scatter.  scratch must hold
// ORDER_SCRATCH_HEADER + n ints; order = scratch + ORDER_SCRATCH_HEADER.  [lo, hi]: the fast
// plan's window whose outsiders are ordered last, ng: the non-gravitational rows whose
// objects are ordered just before them ([-inf, inf] and null: no split).
int launch_span_order(int64_t n, const double* pos, const double* vel, const double* jd0,
                      const double* jd1, double lo, double hi, const double* ng, int* scratch,
                      cudaStream_t stream) {
    int rc = cuda_check(cudaMemsetAsync(scratch, 0, ORDER_SCRATCH_HEADER * sizeof(int), stream),
                        "clear order header");
    if (rc || n <= 0) return rc;
    const int block = 256;
    int64_t g = (n + block - 1) / block;
    const int grid = (int)(g > 1184 ? 1184 : g);
    order_hist_kernel<<<grid, block, 0, stream>>>(n, pos, vel, jd0, jd1, lo, hi, ng, scratch);
    order_scan_kernel<<<1, 32, 0, stream>>>(scratch);
    order_scatter_kernel<<<grid, block, 0, stream>>>(n, pos, vel, jd0, jd1, lo, hi, ng, scratch,
                                                     (int32_t*)(scratch + ORDER_SCRATCH_HEADER));
    return launched(3, "span order launch");
}

}  // namespace kb

#include "flux.cuh"

namespace kb {

// -------------------------------------------------------------------------------------------
// hg_apparent_mag for n geometries (src/kete/rust/flux/reflected.rs:120-132)
// -------------------------------------------------------------------------------------------
__global__ void hg_mag_kernel(int64_t n, const double* __restrict__ s2obj,
                              const double* __restrict__ s2obs, const double* __restrict__ h,
                              const double* __restrict__ g, double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a[3] = {s2obj[i], s2obj[n + i], s2obj[2 * n + i]};
    const double b[3] = {s2obs[i], s2obs[n + i], s2obs[2 * n + i]};
    out[i] = hg_apparent_mag(a, b, h[i], g[i]);
}

int launch_hg_mag(int64_t n, const double* s2obj, const double* s2obs, const double* h,
                  const double* g, double* out, cudaStream_t stream) {
    if (n <= 0) return 0;
    hg_mag_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(n, s2obj, s2obs, h, g, out);
    return launched(1, "hg_mag_kernel launch");
}

// -------------------------------------------------------------------------------------------
// NEATM and FRM total flux (NeatmParams / FrmParams::apparent_total_flux, flux/neatm.rs:143-185,
// flux/frm.rs:137-185).  One warp per geometry.  A facet adds to the thermal sum only when
// the observer sees it and its temperature is above black_body_flux's 30 K floor
// (common.rs:139-154), and on a sphere that is a scattered half or less of the 2048 facets.
// So the warp first tests 32 facets at a time (two dot products), appends the survivors'
// (cos, seen) pairs to a per-warp queue in shared memory, and evaluates the black bodies
// only in full 32-facet batches: every lane busy on the exp-heavy part.  Band sums are
// reduced across the warp at the end.
// -------------------------------------------------------------------------------------------
constexpr int THERMAL_WARPS = 4;

// Black-body sum of one surviving facet into th[]: temperature from the cos term, then per
// band coef / (exp(k / T) - 1) (common.rs:139-154) with the WISE colour correction folded
// into the same division (constants/wise.rs:40-85).
template <int NB, bool CC>
__device__ __forceinline__ void thermal_facet(const NeatmArgs& a, double tmp, double seen,
                                              double ss_temp, double (&th)[NB]) {
    const double temp = sqrt(sqrt(tmp)) * ss_temp;
    if (!(temp >= 30.0)) return;
    const double inv_t = 1.0 / temp;
    double t = 0.0, t2 = 0.0, t3 = 0.0, t4 = 0.0, w4 = 0.0;
    if (CC) {
        t = clampd(temp, 100.0, 400.0);
        t2 = t * t;
        t3 = t * t2;
        t4 = t2 * t2;
        const double l = log(t), l2 = l * l;
        w4 = 2.17247804e+01 + -1.46084733e+01 * l + 3.85364000e+00 * l2 -
             4.51512551e-01 * (l * l2) + 1.98397252e-02 * (l2 * l2);
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        if (b >= a.n_bands || a.bb_coef[b] == 0.0) continue;
        const double em1 = exp(a.bb_k[b] * inv_t) - 1.0;
        double ff;
        if (CC && b == 0)
            ff = a.bb_coef[b] / (em1 * (-3.78226591e-01 + 3.50431748e-03 * t + 1.45866307e-05 * t2 -
                                        6.67674083e-08 * t3 + 7.03651986e-11 * t4));
        else if (CC && b == 1)
            ff = a.bb_coef[b] / (em1 * (-8.60229377e-01 + 1.54988562e-02 * t - 5.10705456e-05 * t2 +
                                        7.68314436e-08 * t3 - 4.32238900e-11 * t4));
        else if (CC && b == 2)
            ff = a.bb_coef[b] / (em1 * (-1.29814355 + 2.43268763e-02 * t - 9.05178737e-05 * t2 +
                                        1.50095351e-07 * t3 - 9.35433316e-11 * t4));
        else if (CC)
            ff = a.bb_coef[b] / em1 * w4;
        else
            ff = a.bb_coef[b] / em1;
        th[b] += seen * ff;
    }
}

template <int NB, bool CC>
__global__ void __launch_bounds__(32 * THERMAL_WARPS, 8) thermal_kernel(NeatmArgs a) {
    __shared__ double2 queue[THERMAL_WARPS][64];
    const int lane = threadIdx.x & 31;
    double2* q = queue[threadIdx.x >> 5];
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= a.n) return;  // warp-uniform
    const int64_t n = a.n;
    double ss_temp, o2s[3], o2o[3], cs = 0.0, sn = 0.0;
    {
        const double s2obj[3] = {a.sun2obj[i], a.sun2obj[n + i], a.sun2obj[2 * n + i]};
        const double s2obs[3] = {a.sun2obs[i], a.sun2obs[n + i], a.sun2obs[2 * n + i]};
        const double obj2sun[3] = {-s2obj[0], -s2obj[1], -s2obj[2]};
        const double obs2obj[3] = {s2obj[0] - s2obs[0], s2obj[1] - s2obs[1], s2obj[2] - s2obs[2]};
        const double obs2obj_r = norm3(obs2obj[0], obs2obj[1], obs2obj[2]);
        // sub_solar_temperature (common.rs:220-236); the FRM's beaming is pi (frm.rs:95-101)
        const double emis = a.emissivity[i];
        const double phase_integral = 0.29 + 0.684 * a.g_param[i];
        const double bond_albedo = a.vis_albedo[i] * phase_integral;
        const double r2 = obj2sun[0] * obj2sun[0] + obj2sun[1] * obj2sun[1] + obj2sun[2] * obj2sun[2];
        const double reflected = (1.0 - bond_albedo) * SOLAR_FLUX / r2;
        const double beam = a.model == 1 ? PI : a.beaming[i];
        ss_temp = reflected / (beam * emis * STEFAN_BOLTZMANN);
        ss_temp = ss_temp <= 0.0 ? 0.0 : sqrt(sqrt(ss_temp));
        const double ns = norm3(obj2sun[0], obj2sun[1], obj2sun[2]);
        for (int c = 0; c < 3; ++c) {
            o2s[c] = obj2sun[c] / ns;
            o2o[c] = obs2obj[c] / obs2obj_r;
        }
        // FRM: cos(lat_facet - lat_sun) (frm_facet_temperature, frm.rs:19-30) expanded with
        // the facet's cos/sin of latitude from the table
        if (a.model == 1) {
            const double sun_lat = asin(o2s[2]);
            cs = cos(sun_lat);
            sn = sin(sun_lat);
        }
    }
    double th[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) th[b] = 0.0;
    const unsigned below = (1u << lane) - 1u;
    int count = 0;  // queued facets, warp-uniform
    for (int base = 0; base < N_FACETS; base += 32) {
        const int f = base + lane;
        const double nx = __ldg(a.facets + f), ny = __ldg(a.facets + N_FACETS + f),
                     nz = __ldg(a.facets + 2 * N_FACETS + f);
        const double seen = -(nx * o2o[0] + ny * o2o[1] + nz * o2o[2]);
        double tmp = 0.0;
        if (seen > 0.0)
            tmp = a.model == 1 ? __ldg(a.facets + 3 * N_FACETS + f) * cs +
                                     __ldg(a.facets + 4 * N_FACETS + f) * sn
                               : nx * o2s[0] + ny * o2s[1] + nz * o2s[2];
        const bool keep = seen > 0.0 && tmp > 0.0;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) q[count + __popc(m & below)] = make_double2(tmp, seen);
        count += __popc(m);
        if (count >= 32) {
            __syncwarp();
            const double2 e = q[lane];
            thermal_facet<NB, CC>(a, e.x, e.y, ss_temp, th);
            __syncwarp();
            if (lane < count - 32) q[lane] = q[lane + 32];
            __syncwarp();
            count -= 32;
        }
    }
    __syncwarp();
    if (lane < count) {
        const double2 e = q[lane];
        thermal_facet<NB, CC>(a, e.x, e.y, ss_temp, th);
    }
    // the geometry again, from memory rather than held in registers through the loop
    const double s2obj[3] = {a.sun2obj[i], a.sun2obj[n + i], a.sun2obj[2 * n + i]};
    const double s2obs[3] = {a.sun2obs[i], a.sun2obs[n + i], a.sun2obs[2 * n + i]};
    const double g = a.g_param[i], diam = a.diam[i];
    // Lambertian scale emissivity * pi * (r / D)^-2 (common.rs:190-205) and the facet area
    const double obs2obj_r = norm3(s2obj[0] - s2obs[0], s2obj[1] - s2obs[1], s2obj[2] - s2obs[2]);
    const double dscale = obs2obj_r * AU_KM / diam;
    const double sc = a.emissivity[i] * PI * (1.0 / (dscale * dscale)) * a.facet_area;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) th[b] += __shfl_xor_sync(0xffffffffu, th[b], o);
        th[b] *= sc;
    }
    if (lane < a.n_bands) {
        const int b = lane;
        double thb = 0.0;
#pragma unroll
        for (int c = 0; c < NB; ++c)
            if (c == b) thb = th[c];
        const double refl =
            hg_apparent_flux(s2obj, s2obs, g, diam, a.wavelength[b], a.band_albedo[(int64_t)b * n + i]) *
            a.sun_correction[b];
        const double total = thb + refl;
        a.thermal[(int64_t)b * n + i] = thb;
        a.hg_fluxes[(int64_t)b * n + i] = refl;
        a.fluxes[(int64_t)b * n + i] = total;
        if (a.mags) a.mags[(int64_t)b * n + i] = a.have_zero_mags ? -2.5 * log10(total / a.zero_mag[b])
                                                                  : __longlong_as_double(0x7ff8000000000000LL);
    }
    if (lane == 0) {
        const double vm = hg_apparent_mag(s2obj, s2obs, a.h_mag[i], g);
        a.v_mag[i] = vm;
        a.v_flux[i] = -2.5 * log10(vm / V_MAG_ZERO);  // flux_to_mag(v_mag, V_MAG_ZERO), neatm.rs:167
    }
}

int launch_neatm(const NeatmArgs& a, cudaStream_t stream) {
    if (a.n <= 0) return 0;
    const int64_t threads = a.n * 32;
    const unsigned grid = (unsigned)((threads + 32 * THERMAL_WARPS - 1) / (32 * THERMAL_WARPS));
    const unsigned block = 32 * THERMAL_WARPS;
    if (a.wise_cc)  // the capi admits colour corrections only with the 4 WISE bands
        thermal_kernel<4, true><<<grid, block, 0, stream>>>(a);
    else if (a.n_bands <= 2)
        thermal_kernel<2, false><<<grid, block, 0, stream>>>(a);
    else if (a.n_bands <= 4)
        thermal_kernel<4, false><<<grid, block, 0, stream>>>(a);
    else
        thermal_kernel<MAX_BANDS, false><<<grid, block, 0, stream>>>(a);
    return launched(1, "thermal_kernel launch");
}

}  // namespace kb

#include "fov.cuh"

namespace kb {

int launch_fov_prefilter(const FovArgs& a, cudaStream_t stream) {
    if (a.n_obj <= 0 || a.n_fov <= 0) return 0;
    fov_prefilter_kernel<<<(unsigned)((a.n_obj + 127) / 128), 128, 0, stream>>>(a);
    return launched(1, "fov_prefilter_kernel launch");
}

int launch_fov_screen(const FovArgs& a, cudaStream_t stream) {
    if (a.n_obj <= 0 || a.n_fov <= 0) return 0;
    fov_screen_kernel<<<(unsigned)((a.n_obj + 127) / 128), 128, 0, stream>>>(a);
    return launched(1, "fov_screen_kernel launch");
}

int launch_fov_pairs(const FovArgs& a, int64_t m, cudaStream_t stream) {
    if (m <= 0) return 0;
    fov_pairs_kernel<<<(unsigned)((m + 127) / 128), 128, 0, stream>>>(a, m);
    return launched(1, "fov_pairs_kernel launch");
}

int launch_fov_gather(const FovArgs& a, int64_t m, double* gpos, double* gvel, double* gjd0,
                      double* gjd1, cudaStream_t stream) {
    if (m <= 0) return 0;
    fov_gather_kernel<<<(unsigned)((m + 127) / 128), 128, 0, stream>>>(a, m, gpos, gvel, gjd0, gjd1);
    return launched(1, "fov_gather_kernel launch");
}

int launch_fov_contains(int64_t n_vec, const double* vec, int64_t n_fov, const double* fov,
                        int64_t capacity, unsigned long long* counter, int32_t* out_fov,
                        int32_t* out_idx, cudaStream_t stream) {
    if (n_vec <= 0 || n_fov <= 0) return 0;
    fov_contains_kernel<<<(unsigned)((n_vec + 127) / 128), 128, 0, stream>>>(
        n_vec, vec, n_fov, fov, capacity, counter, out_fov, out_idx);
    return launched(1, "fov_contains_kernel launch");
}

int launch_fov_finish(const FovArgs& a, int64_t m, const double* npos, const double* nvel,
                      const int32_t* nst, cudaStream_t stream) {
    if (m <= 0) return 0;
    fov_nbody_finish_kernel<<<(unsigned)((m + 127) / 128), 128, 0, stream>>>(a, m, npos, nvel, nst);
    return launched(1, "fov_nbody_finish_kernel launch");
}

}  // namespace kb

// -------------------------------------------------------------------------------------------
// Two-body state-transition matrices with covariance propagation (compute_stm,
// propagate_covariance: src/kete/state_transition.py:8-59, corrected as kepler_stm.cuh
// describes), and the covariance sandwich Phi C Phi^T on its own for other matrices.
// -------------------------------------------------------------------------------------------
#include "kepler_stm.cuh"

namespace kb {

// out (rows x rows) = Phi (rows x cols) C (cols x cols) Phi^T for object i; SoA with the
// object index fastest.
__device__ __forceinline__ void covariance_sandwich(int64_t n, int64_t i, int rows, int cols,
                                                    const double* Phi, bool phi_soa,
                                                    const double* C, double* out) {
    for (int r = 0; r < rows; ++r)
        for (int q = r; q < rows; ++q) {
            double acc = 0.0;
            for (int a = 0; a < cols; ++a) {
                const double pra = phi_soa ? Phi[(int64_t)(r * cols + a) * n + i] : Phi[r * cols + a];
                double inner = 0.0;
                for (int b = 0; b < cols; ++b) {
                    const double pqb = phi_soa ? Phi[(int64_t)(q * cols + b) * n + i] : Phi[q * cols + b];
                    inner += C[(int64_t)(a * cols + b) * n + i] * pqb;
                }
                acc += pra * inner;
            }
            out[(int64_t)(r * rows + q) * n + i] = acc;
            out[(int64_t)(q * rows + r) * n + i] = acc;
        }
}

__global__ void __launch_bounds__(128) two_body_stm_kernel(
    int64_t n, const double* __restrict__ pos, const double* __restrict__ vel,
    const double* __restrict__ jd0, const double* __restrict__ jd1, double mu,
    const double* __restrict__ cov, double* __restrict__ out_pos, double* __restrict__ out_vel,
    double* __restrict__ out_stm, double* __restrict__ out_cov, int32_t* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double p[3] = {pos[i], pos[n + i], pos[2 * n + i]};
    double v[3] = {vel[i], vel[n + i], vel[2 * n + i]};
    double Phi[36];
    int rc = analytic_2_body_stm(jd1[i] - jd0[i], p, v, mu, Phi);
    if (rc != ST_OK) {
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        p[0] = p[1] = p[2] = v[0] = v[1] = v[2] = nan;
#pragma unroll
        for (int k = 0; k < 36; ++k) Phi[k] = nan;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        out_pos[c * n + i] = p[c];
        out_vel[c * n + i] = v[c];
    }
    if (out_stm)
#pragma unroll
        for (int k = 0; k < 36; ++k) out_stm[k * n + i] = Phi[k];
    if (cov && out_cov) covariance_sandwich(n, i, 6, 6, Phi, false, cov, out_cov);
    status[i] = rc;
}

__global__ void __launch_bounds__(128) covariance_kernel(int64_t n, int rows, int cols,
                                                         const double* __restrict__ phi,
                                                         const double* __restrict__ cov,
                                                         double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    covariance_sandwich(n, i, rows, cols, phi, true, cov, out);
}

int launch_two_body_stm(int64_t n, const double* pos, const double* vel, const double* jd0,
                        const double* jd1, double mu, const double* cov, double* out_pos,
                        double* out_vel, double* out_stm, double* out_cov, int32_t* status,
                        cudaStream_t stream) {
    if (n <= 0) return 0;
    two_body_stm_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(
        n, pos, vel, jd0, jd1, mu, cov, out_pos, out_vel, out_stm, out_cov, status);
    return launched(1, "two_body_stm_kernel launch");
}

int launch_covariance(int64_t n, int rows, int cols, const double* phi, const double* cov,
                      double* out, cudaStream_t stream) {
    if (n <= 0) return 0;
    covariance_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(n, rows, cols, phi, cov, out);
    return launched(1, "covariance_kernel launch");
}

}  // namespace kb
