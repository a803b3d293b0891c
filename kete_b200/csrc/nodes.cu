// nodes.cu -- host launchers of the node-parallel Radau kernels (radau_nodes.cuh and the
// warp-pooled form of radau_pool.cuh): every register-cap / step-end / warp-synchronous /
// pooled instantiation the tuner chooses from.  Its own translation unit so the
// instantiations compile in parallel with the other kernels.
#include <algorithm>
#include <atomic>

#include "../../include/kete_b200.h"

#include "common.cuh"
#include "forces.cuh"
#include "internal.h"
#include "radau_nodes.cuh"
#include "radau_pool.cuh"

namespace kb {
KB_CONSTANT_UPLOADER(nodes)
}  // namespace kb

namespace kb {

// Node-parallel Radau: 8 lanes per object.  With a.queue == null each group integrates one
// object (grid covers n groups); with a queue the grid is persistent and groups refill.
// variant: 0 = no register cap, 1 = >= 3 blocks/SM (168 registers), 2 = >= 4 blocks/SM;
// +3: the step-end lane form (exact evaluations taken from lane 7, see radau_nodes.cuh);
// 6-8: the step-end form with warp-synchronous steps and the per-lane ephemeris cache;
// 9, 10: the warp-pooled record evaluations (radau_pool.cuh) at 168 / 128 registers.
static const void* nodes_kernel_ptr(int variant) {
    switch (variant) {
        case 9: return (const void*)nbody_pool_kernel<3>;
        case 10: return (const void*)nbody_pool_kernel<4>;
        case 1: return (const void*)nbody_nodes_kernel<3, false>;
        case 2: return (const void*)nbody_nodes_kernel<4, false>;
        case 3: return (const void*)nbody_nodes_kernel<1, true>;
        case 4: return (const void*)nbody_nodes_kernel<3, true>;
        case 5: return (const void*)nbody_nodes_kernel<4, true>;
        case 6: return (const void*)nbody_nodes_kernel<1, true, true>;
        case 7: return (const void*)nbody_nodes_kernel<3, true, true>;
        case 8: return (const void*)nbody_nodes_kernel<4, true, true>;
        default: return (const void*)nbody_nodes_kernel<1, false>;
    }
}

static int dyn_smem(int variant) { return variant >= 9 ? POOL_DYN_SMEM : 0; }

// The pooled kernels keep their body cache in dynamic shared memory above the 48 KB static
// limit: allow it once per device (a function attribute, not a stream operation).
static int allow_dyn_smem(int variant) {
    static std::atomic<unsigned long long> done[2];
    if (variant < 9) return 0;
    int dev = 0;
    int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (rc) return rc;
    const unsigned long long bit = 1ull << (dev & 63);
    auto& d = done[variant - 9];
    if (d.load() & bit) return 0;
    if ((rc = cuda_check(cudaFuncSetAttribute(nodes_kernel_ptr(variant),
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              dyn_smem(variant)),
                         "pooled kernel shared memory")))
        return rc;
    d.fetch_or(bit);
    return 0;
}

int launch_nbody_nodes(const NBodyArgs& a, int variant, int grid, cudaStream_t stream) {
    if (a.n <= 0) return 0;
    if (variant >= 9 && !a.range)
        return set_error(KETE_B200_E_ARGUMENT,
                         "the warp-pooled node kernels take the window split of the processing "
                         "order (launch_nodes_ordered)");
    const int block = NODES_BLOCK;
    if (grid <= 0) grid = (int)((a.n * NODE_G + block - 1) / block);
    int rc = allow_dyn_smem(variant);
    if (rc) return rc;
    switch (variant) {
        case 9: nbody_pool_kernel<3><<<grid, block, POOL_DYN_SMEM, stream>>>(a); break;
        case 10: nbody_pool_kernel<4><<<grid, block, POOL_DYN_SMEM, stream>>>(a); break;
        case 1: nbody_nodes_kernel<3, false><<<grid, block, 0, stream>>>(a); break;
        case 2: nbody_nodes_kernel<4, false><<<grid, block, 0, stream>>>(a); break;
        case 3: nbody_nodes_kernel<1, true><<<grid, block, 0, stream>>>(a); break;
        case 4: nbody_nodes_kernel<3, true><<<grid, block, 0, stream>>>(a); break;
        case 5: nbody_nodes_kernel<4, true><<<grid, block, 0, stream>>>(a); break;
        case 6: nbody_nodes_kernel<1, true, true><<<grid, block, 0, stream>>>(a); break;
        case 7: nbody_nodes_kernel<3, true, true><<<grid, block, 0, stream>>>(a); break;
        case 8: nbody_nodes_kernel<4, true, true><<<grid, block, 0, stream>>>(a); break;
        default: nbody_nodes_kernel<1, false><<<grid, block, 0, stream>>>(a); break;
    }
    return launched(1, "nbody_nodes_kernel launch");
}

// Persistent grid of a variant, capped at one lane group per object.
static int refill_grid(int variant, int64_t n, int* grid) {
    int rc = nodes_grid_size(variant, grid);
    if (rc) return rc;
    const int64_t need = (n * NODE_G + NODES_BLOCK - 1) / NODES_BLOCK;
    if (*grid > need) *grid = (int)need;
    return 0;
}

int launch_nodes_ordered(NBodyArgs a, int variant, int general_variant, bool refill,
                         int* scratch, cudaStream_t stream) {
    a.order = (const int32_t*)(scratch + ORDER_SCRATCH_HEADER);
    int grid = 0, rc = 0;
    if (variant < 9) {  // one launch over the whole order
        a.range = nullptr;
        a.queue = refill ? scratch : nullptr;
        if (refill && (rc = refill_grid(variant, a.n, &grid))) return rc;
        return launch_nbody_nodes(a, variant, grid, stream);
    }
    // objects inside the window: the pooled kernel between its centre-change kernels; the
    // others: the general form.  The counts are on the device, so every grid covers every
    // object (threads and groups past their part exit).
    a.range = scratch + ORDER_RANGE;
    a.queue = refill ? scratch : nullptr;
    a.queue_ng = refill ? scratch + ORDER_QUEUE3 : nullptr;
    const int64_t cgrid = std::min<int64_t>((a.n + 255) / 256, 1184);
    pool_prepare_kernel<<<(int)cgrid, 256, 0, stream>>>(a);
    if ((rc = launched(1, "pool_prepare_kernel launch"))) return rc;
    if (refill && (rc = refill_grid(variant, a.n, &grid))) return rc;
    if ((rc = launch_nbody_nodes(a, variant, grid, stream))) return rc;
    pool_finish_kernel<<<(int)cgrid, 256, 0, stream>>>(a);
    if ((rc = launched(1, "pool_finish_kernel launch"))) return rc;
    a.range = scratch + ORDER_RANGE + 2;
    a.queue = refill ? scratch + ORDER_QUEUE2 : nullptr;
    a.queue_ng = nullptr;
    grid = 0;
    if (refill && (rc = refill_grid(general_variant, a.n, &grid))) return rc;
    return launch_nbody_nodes(a, general_variant, grid, stream);
}

int preload_nodes_kernels() {
    cudaFuncAttributes fa;
    int rc = 0;
    for (int v = 0; v <= 10; ++v) {
        if ((rc = cuda_check(cudaFuncGetAttributes(&fa, nodes_kernel_ptr(v)), "load node kernels")))
            return rc;
        if ((rc = allow_dyn_smem(v))) return rc;
    }
    for (const void* f : {(const void*)pool_prepare_kernel, (const void*)pool_finish_kernel})
        if ((rc = cuda_check(cudaFuncGetAttributes(&fa, f), "load node kernels"))) return rc;
    return 0;
}

// Resident grid for the persistent (refill) form: blocks per SM from the occupancy API.
int nodes_grid_size(int variant, int* grid) {
    int dev = 0, sms = 0, per_sm = 0;
    int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (rc) return rc;
    if ((rc = cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attr")))
        return rc;
    if ((rc = allow_dyn_smem(variant))) return rc;
    if ((rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                             &per_sm, nodes_kernel_ptr(variant), NODES_BLOCK, dyn_smem(variant)),
                         "occupancy")))
        return rc;
    *grid = sms * (per_sm > 0 ? per_sm : 1);
    return 0;
}

}  // namespace kb
