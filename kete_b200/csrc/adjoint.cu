// adjoint.cu -- reverse-mode gradients: the checkpointed forward pass and the discrete
// adjoint pass (adjoint.cuh) with their host launchers.
#include "common.cuh"
#include "forces.cuh"
#include "internal.h"
#include "adjoint.cuh"

namespace kb {
KB_CONSTANT_UPLOADER(adjoint)
}  // namespace kb

namespace kb {

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
    // every block's replay first, one group per (object, block); then the sweep. The replay
    // is throughput bound (n x blocks groups), so it is capped at 168 registers for 12
    // resident warps per SM; the sweep is one partial wave and keeps the full register file.
    for (const void* f : {(const void*)nbody_sens_replay_kernel<3>,
                          (const void*)nbody_sens_backward_kernel<1, false>})
        if ((rc = cuda_check(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  cache_bytes),
                             "cudaFuncSetAttribute")))
            return rc;
    const int64_t rthreads = a.n * (int64_t)a.ckpt_cap * SG;
    nbody_sens_replay_kernel<3><<<(unsigned)((rthreads + SENS_BLOCK - 1) / SENS_BLOCK), SENS_BLOCK,
                                  cache_bytes, stream>>>(a);
    if ((rc = launched(1, "nbody_sens_replay_kernel launch"))) return rc;
    nbody_sens_backward_kernel<1, false><<<grid, SENS_BLOCK, cache_bytes, stream>>>(a);
    return launched(1, "nbody_sens_backward_kernel launch");
}

}  // namespace kb
