// noalloc.cu -- N-body propagation that allocates no device memory on the call.
//
// Who needs this: callers that cannot let a library call cudaMalloc/cudaFree while they
// run.  cudaMalloc and cudaFree synchronize the device and can fail under memory pressure,
// so a real-time or steady-state loop (a survey pipeline re-propagating every few seconds,
// a service that sizes all of its GPU memory up front, code running while another
// allocator owns the device's free memory) must not hit them mid-loop.  The regular entry
// point takes its per-call scratch -- the object queue, the span histogram and the
// processing order of the persistent grid -- from buffers it allocates and grows.  This
// variant keeps that scratch in a fixed array of device memory reserved in the library
// image instead.
//
// The fixed array is a file-scope __device__ object of KETE_B200_NOALLOC_MAX_OBJECTS * 4 +
// 1024 bytes (4 MiB + 1 KiB).  CUDA loads modules lazily, so a device holds the array from
// the moment its module is loaded until the process exits: kete_b200_init loads it (and the
// kernels this entry point launches) on the device it prepares, and looks the array's
// device address up there with cudaGetSymbolAddress -- host code cannot use the array's name
// as a device address.  A device that kete_b200_init has not prepared gets the same lookup,
// with the module loading it implies, on its first call here, which should then come before
// any stream capture.  All calls share the one array: calls whose work overlaps on the GPU
// (different streams, or different host threads) race on it and must be serialized by the
// caller, as must a concurrent SPK load or kete_b200_set_launch_config on another thread
// (the call reads the ephemeris table and launch configuration, then enqueues).  The header
// that must start at zero (queues, histogram, cursors) is cleared by every call.
#include <cstring>
#include <mutex>

#include "../../include/kete_b200.h"
#include "common.cuh"
#include "ephem.cuh"
#include "internal.h"

namespace kb {

static_assert(KETE_B200_NOALLOC_MAX_OBJECTS > 0, "maximum object count");

// queue counter, span histogram and cursors (ORDER_SCRATCH_HEADER ints), then the order
static __device__ __align__(256) int g_noalloc_scratch[ORDER_SCRATCH_HEADER + KETE_B200_NOALLOC_MAX_OBJECTS];

constexpr int NOALLOC_MAX_DEVICES = 64;
static int* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};
static std::mutex g_noalloc_mu;

// Device address of the scratch array on the current device (looked up once per device).
static int noalloc_scratch(int** out) {
    int dev = 0;
    int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (rc) return rc;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return set_error(KETE_B200_E_UNSUPPORTED, "device index beyond the allocation-free table");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        rc = cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch),
                        "cudaGetSymbolAddress of the allocation-free scratch");
        if (rc) return rc;
        g_noalloc_ptr[dev] = (int*)p;
    }
    *out = g_noalloc_ptr[dev];
    return 0;
}

int noalloc_prepare() {
    int* p = nullptr;
    return noalloc_scratch(&p);
}

}  // namespace kb

using namespace kb;

extern "C" int kete_b200_propagate_n_body_noalloc(
    int64_t n, const double* pos, const double* vel, const double* jd0, const double* jd1,
    int frame, int64_t center, int include_asteroids, const double* nongrav, double* out_pos,
    double* out_vel, int32_t* status, int32_t* impact_id, double* impact_jd, double* min_dist,
    int32_t* counters, void* stream) {
    if (n < 0 || (n > 0 && (!pos || !vel || !jd0 || !jd1 || !out_pos || !out_vel || !status)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    if (n > KETE_B200_NOALLOC_MAX_OBJECTS)
        return set_error(KETE_B200_E_ARGUMENT,
                         "kete_b200_propagate_n_body_noalloc: " + std::to_string(n) +
                             " objects exceed the fixed scratch of " +
                             std::to_string(KETE_B200_NOALLOC_MAX_OBJECTS) +
                             " objects; split the call or use kete_b200_propagate_n_body");
    if (frame != FRAME_EQUATORIAL && frame != FRAME_ECLIPTIC)
        return set_error(KETE_B200_E_UNSUPPORTED, "frame must be equatorial (1) or ecliptic (2)");
    NBodyArgs a;
    std::memset(&a, 0, sizeof a);
    LaunchConfig cfg;
    NodesPlan plan;
    int rc = noalloc_snapshot(include_asteroids, center, a, cfg, plan);
    if (rc) return rc;
    int* scratch = nullptr;
    if ((rc = noalloc_scratch(&scratch))) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    a.n = n;
    a.pos = pos;
    a.vel = vel;
    a.jd0 = jd0;
    a.jd1 = jd1;
    a.nongrav = nongrav;
    a.frame = frame;
    a.out_pos = out_pos;
    a.out_vel = out_vel;
    a.status = status;
    a.impact_id = impact_id;
    a.impact_jd = impact_jd;
    a.min_dist = min_dist;
    a.counters = counters;
    a.max_loops = cfg.max_loops;
    if ((rc = launch_span_order(n, pos, vel, jd0, jd1, plan.lo, plan.hi,
                                cfg.nodes_variant >= 9 ? nongrav : nullptr, scratch, st)))
        return rc;
    return launch_nodes_ordered(a, cfg.nodes_variant, plan.general_variant, true, scratch, st);
}
