// adjoint.cu -- reverse-mode gradients: the checkpointed forward pass and the discrete
// adjoint pass (adjoint.cuh) with their host launchers.
// every object of the differentiation workloads carries the comet model: inline it
#define KB_FORCE_NG_INLINE 1
#include "common.cuh"
#include "forces.cuh"
#include "internal.h"
#include "adjoint.cuh"

namespace kb {
KB_CONSTANT_UPLOADER(adjoint)
}  // namespace kb

namespace kb {

// Exclusive prefix sums of the blocks each object replays (its checkpoint count when its
// forward pass succeeded, else none) into a.rep_first[0 .. n], and the replay's queue
// counter a.rep_first[n + 1] cleared; one thread block, each thread a contiguous run of
// objects.
constexpr int OFFSETS_THREADS = 1024;
__global__ void __launch_bounds__(OFFSETS_THREADS) sens_replay_offsets_kernel(SensArgs a) {
    __shared__ int64_t s_sum[OFFSETS_THREADS];
    const int64_t n = a.n;
    const int64_t per = (n + OFFSETS_THREADS - 1) / OFFSETS_THREADS;
    const int64_t o0 = (int64_t)threadIdx.x * per;
    const int64_t o1 = o0 + per < n ? o0 + per : n;
    auto blocks = [&](int64_t o) -> int64_t {
        if (a.status[o] != ST_OK) return 0;
        const int c = a.ckpt_count[o];
        return c < 0 ? 0 : (c > a.ckpt_cap ? a.ckpt_cap : c);
    };
    int64_t own = 0;
    for (int64_t o = o0; o < o1; ++o) own += blocks(o);
    s_sum[threadIdx.x] = own;
    __syncthreads();
    for (int d = 1; d < OFFSETS_THREADS; d <<= 1) {  // inclusive scan (Hillis-Steele)
        const int64_t add = threadIdx.x >= (unsigned)d ? s_sum[threadIdx.x - d] : 0;
        __syncthreads();
        s_sum[threadIdx.x] += add;
        __syncthreads();
    }
    int64_t run = s_sum[threadIdx.x] - own;
    for (int64_t o = o0; o < o1; ++o) {
        a.rep_first[o] = (int32_t)run;
        run += blocks(o);
    }
    if (threadIdx.x == OFFSETS_THREADS - 1) {
        a.rep_first[n] = (int32_t)s_sum[threadIdx.x];
        a.rep_first[n + 1] = 0;
    }
}

int launch_sens_forward(const SensArgs& a, cudaStream_t stream) {
    if (a.n <= 0) return 0;
    const int64_t threads = a.n * SG;
    nbody_sens_forward_kernel<1><<<(unsigned)((threads + SENS_BLOCK - 1) / SENS_BLOCK), SENS_BLOCK, 0, stream>>>(a);
    return launched(1, "nbody_sens_forward_kernel launch");
}

int launch_sens_backward(const SensArgs& a, cudaStream_t stream) {
    if (a.n <= 0) return 0;
    const int64_t threads = a.n * SG;
    // the per-lane ephemeris cache takes the block past the 48 KB of shared memory a kernel
    // gets without opting in (a function attribute, not a stream operation)
    constexpr int cache_bytes = EPH_CACHE * SENS_BLOCK * (int)sizeof(double);
    int rc = 0;
    const unsigned grid = (unsigned)((threads + SENS_BLOCK - 1) / SENS_BLOCK);
    if (!a.rec_all) {  // the sweep re-runs each block itself
        if ((rc = cuda_check(cudaFuncSetAttribute(nbody_sens_backward_kernel<1, true>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  cache_bytes),
                             "cudaFuncSetAttribute")))
            return rc;
        nbody_sens_backward_kernel<1, true><<<grid, SENS_BLOCK, cache_bytes, stream>>>(a);
        return launched(1, "nbody_sens_backward_kernel launch");
    }
    // every block's replay first (groups taking the blocks from a queue), then the sweep. The
    // replay is throughput bound (every block of every object), so it is capped at 168
    // registers for 12 resident warps per SM; the sweep is one partial wave and keeps the full
    // register file.
    for (const void* f : {(const void*)nbody_sens_replay_kernel<3>,
                          (const void*)nbody_sens_backward_kernel<1, false>})
        if ((rc = cuda_check(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  cache_bytes),
                             "cudaFuncSetAttribute")))
            return rc;
    sens_replay_offsets_kernel<<<1, OFFSETS_THREADS, 0, stream>>>(a);
    if ((rc = launched(1, "sens_replay_offsets_kernel launch"))) return rc;
    // persistent grid: as many thread blocks as are resident at once, and no more than the
    // blocks to replay could occupy
    int dev = 0, sms = 0, per_sm = 0;
    if ((rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice")) ||
        (rc = cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                         "attr")) ||
        (rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                             &per_sm, nbody_sens_replay_kernel<3>, SENS_BLOCK, cache_bytes),
                         "occupancy")))
        return rc;
    const int64_t resident = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
    const int64_t rthreads = a.n * (int64_t)a.ckpt_cap * SG;
    const int64_t need = (rthreads + SENS_BLOCK - 1) / SENS_BLOCK;
    const unsigned rgrid = (unsigned)(need < resident ? need : resident);
    nbody_sens_replay_kernel<3><<<rgrid, SENS_BLOCK, cache_bytes, stream>>>(a);
    if ((rc = launched(1, "nbody_sens_replay_kernel launch"))) return rc;
    nbody_sens_backward_kernel<1, false><<<grid, SENS_BLOCK, cache_bytes, stream>>>(a);
    return launched(1, "nbody_sens_backward_kernel launch");
}

}  // namespace kb
