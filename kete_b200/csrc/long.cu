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
