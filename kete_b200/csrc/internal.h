// internal.h -- host-side declarations shared by the C-ABI layer and the kernel TU.
#pragma once
#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ephem.cuh"

namespace kb {

struct Tables;
struct EphemConst;

// set the thread's last error message; returns `code`
int set_error(int code, const std::string& msg);
int cuda_check(cudaError_t e, const char* what);
extern std::atomic<int64_t> g_kernel_launches;  // kernels.cu
// device allocations the library has made since it was loaded (kete_b200_device_allocations)
extern std::atomic<int64_t> g_device_allocations;  // kernels.cu

// cudaMalloc counted in g_device_allocations
inline cudaError_t counted_malloc(void** p, size_t bytes) {
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) g_device_allocations.fetch_add(1, std::memory_order_relaxed);
    return e;
}

// every launch helper adds the kernels it enqueued when it checks the launch
inline int launched(int kernels, const char* what) {
    g_kernel_launches.fetch_add(kernels, std::memory_order_relaxed);
    return cuda_check(cudaGetLastError(), what);
}

// kernels.cu: write the device constants of every kernel translation unit
int upload_tables(const Tables& t);
int upload_ephem(const EphemConst& e);
int upload_consts_kernels(const Tables* t, const EphemConst* e);
int upload_consts_nodes(const Tables* t, const EphemConst* e);
int upload_consts_sens(const Tables* t, const EphemConst* e);
int upload_consts_adjoint(const Tables* t, const EphemConst* e);
int upload_consts_long(const Tables* t, const EphemConst* e);

struct NBodyArgs {
    int64_t n;
    const double* pos;  // 3 x n
    const double* vel;
    const double* jd0;
    const double* jd1;
    const double* nongrav;  // 10 x n or null
    int frame;
    CenterChain chain;
    int n_force;
    double* out_pos;
    double* out_vel;
    int32_t* status;
    int32_t* impact_id;   // may be null
    double* impact_jd;    // may be null
    double* min_dist;     // may be null
    int32_t* counters;    // 3 x n (steps, iterations, exact evals) or null
    int max_loops;        // step-loop bound per object (ST_TIMEOUT beyond)
    int* queue;           // refill counter for the node kernel (null: one object per group)
    const int32_t* order; // processing order (permutation of 0..n-1) or null
    const int* range;     // device {first, end}: the node kernel takes order[first .. end)
                          // (null: order[0 .. n)); the pooled kernel: {first, start of the
                          // non-gravitational part, end}
    int* queue_ng;        // pooled kernel with refill: the queue of the non-gravitational part
};

int launch_two_body(int64_t n, const double* pos, const double* vel, const double* jd0,
                    const double* jd1, const double* obs, double* out_pos, double* out_vel,
                    double* out_jd, int32_t* status, cudaStream_t stream);
int launch_two_body_stm(int64_t n, const double* pos, const double* vel, const double* jd0,
                        const double* jd1, double mu, const double* cov, double* out_pos,
                        double* out_vel, double* out_stm, double* out_cov, int32_t* status,
                        cudaStream_t stream);
int launch_covariance(int64_t n, int rows, int cols, const double* phi, const double* cov,
                      double* out, cudaStream_t stream);
int launch_nbody_thread(const NBodyArgs& a, int block, cudaStream_t stream);
int launch_nbody_nodes(const NBodyArgs& a, int variant, int grid, cudaStream_t stream);
int nodes_grid_size(int variant, int* grid);
// load the node kernels and the processing-order kernels into the current context (module
// loading is lazy: done here, it does not happen inside a later call)
int preload_nodes_kernels();
int preload_order_kernels();
// resolve the allocation-free entry point's scratch address on the current device
int noalloc_prepare();
int launch_span_order(int64_t n, const double* pos, const double* vel, const double* jd0,
                      const double* jd1, double lo, double hi, const double* ng, int* scratch,
                      cudaStream_t stream);
// The node kernels over the processing order that launch_span_order wrote into scratch
// (variant as launch_nbody_nodes; refill: persistent grid with the object queue).  A
// warp-pooled variant integrates the objects inside the fast plan's window (those with a
// non-gravitational model from a queue of their own, first on a few SMs) and general_variant
// (a form with the general ephemeris evaluation) the others, in a second launch; every other
// variant takes the whole order in one launch.
int launch_nodes_ordered(NBodyArgs a, int variant, int general_variant, bool refill,
                         int* scratch, cudaStream_t stream);

// launch configuration chosen by the tuner (kete_b200_set_launch_config)
struct LaunchConfig {
    int nodes_variant = 7;  // node-kernel form (see launch_nbody_nodes); 7 measured fastest
    int nodes_refill = 0;   // 1: persistent grid with an object queue
    int thread_block = 128;
    // bound on each object's Radau step loop (kete_b200_set_step_limit): an integration that
    // has not reached its target after this many step attempts returns ST_TIMEOUT
    int max_loops = 1 << 20;
    int max_loops_long = 1 << 24;  // system integration (every batch's whole span)
    int sens_form = 0;  // forward sensitivities: 0 node-parallel, 1 one object per thread
    int fov_form = 0;   // field checks: 0 linear screen + two-body pass, 1 one fused pass
    int adjoint_parallel_replay = 1;  // adjoint: replay every checkpoint block up front
};
// scratch bound of the adjoint's up-front replay (every block's attempt records)
constexpr size_t ADJOINT_REPLAY_BYTES = size_t(8) << 30;
LaunchConfig& launch_config();
// What the allocation-free entry point launches: the node variant in cfg.nodes_variant, the
// variant with the general ephemeris evaluation, and the window of launch_span_order.
struct NodesPlan {
    int general_variant;
    double lo, hi;
};
int noalloc_snapshot(int include_asteroids, int64_t center, NBodyArgs& a, LaunchConfig& cfg,
                     NodesPlan& plan);
int launch_radau_central(int64_t n, const double* pos, const double* vel, const double* t0,
                         const double* t1, double* out_pos, double* out_vel, int32_t* status,
                         cudaStream_t stream);
int launch_spk_states(int64_t n, int32_t slot, const double* jd,
                      const CenterChain& center_chain, int frame, double* out6, int32_t* status,
                      cudaStream_t stream);

int fp64_probe(int64_t iters, double* tflops, float* ms_out);

struct StmArgs {
    int64_t n;
    const double* pos;
    const double* vel;
    const double* jd0;
    int n_epochs;
    const double* epochs;   // device, n_epochs
    const double* nongrav;  // 10 x n or null
    int frame;
    CenterChain chain;
    int n_force;
    double* out_state;  // n_epochs x 6 x n
    double* out_stm;    // n_epochs x 48 x n (row-major 6 x 8 per object)
    int32_t* status;
    int max_loops;
};
// form: 0 = node-parallel (8 lanes per object), 1 = one object per thread
int launch_nbody_stm(const StmArgs& a, int form, cudaStream_t stream);

// reverse-mode gradients: checkpointed forward pass and adjoint pass (adjoint.cuh)
constexpr int SENS_STRIDE = 36;       // doubles per checkpoint / attempt record
constexpr int SENS_CK_ATTEMPTS = 16;  // step attempts between checkpoints
struct SensArgs {
    int64_t n;
    const double* pos;  // 3 x n (forward)
    const double* vel;
    const double* jd0;
    int n_epochs;
    const double* epochs;   // n_epochs
    const double* nongrav;  // 10 x n or null
    int frame;
    CenterChain chain;
    int n_force;
    double* out_state;   // n_epochs x 6 x n (forward)
    int32_t* status;     // n: written by the forward pass, read by the adjoint pass
    double* ckpt;        // n x ckpt_cap x SENS_STRIDE
    int ckpt_cap;
    int32_t* ckpt_count; // n: checkpoints taken (may exceed ckpt_cap: ST_CHECKPOINT_FULL)
    int32_t* ckpt_seg;   // n_epochs x n: first checkpoint of each epoch segment
    const double* seed;  // n_epochs x 6 x n: dL/d(state at each epoch) (adjoint)
    double* out_grad;    // 8 x n: dL/d(pos0, vel0, A1, A2) (adjoint)
    int32_t* grad_status;  // n or null (adjoint)
    double* rec;         // n x (SENS_CK_ATTEMPTS + 1) x SENS_STRIDE scratch (adjoint)
    double* rec_all;     // n x ckpt_cap x (SENS_CK_ATTEMPTS + 1) x SENS_STRIDE, or null: the
                         // records of every block, replayed up front (adjoint)
    int32_t* rep_count;  // n x ckpt_cap: attempts of each replayed block, -1 - status on failure
    int32_t* rep_first;  // n + 2 (with rec_all): exclusive prefix sums of the blocks to replay
                         // per object (the replay takes the blocks in this dense order), then
                         // the replay's queue counter
    int max_loops;
};
int launch_sens_forward(const SensArgs& a, cudaStream_t stream);
int launch_sens_backward(const SensArgs& a, cudaStream_t stream);

// system integration (long.cuh): SIMPLE_PLANETS integrated with batches of test particles
struct LongArgs {
    int64_t n;
    const double* pos;  // 3 x n heliocentric equatorial at jd0
    const double* vel;
    double jd0, jd1;
    const double* planets;        // 9 x 6 heliocentric equatorial at jd0 (row per body)
    const int32_t* planet_status; // 9 or null: the SPK lookups that produced planets
    const double* nongrav;        // 10 x n or null
    int batch;                    // test particles per batch (<= 55)
    double* out_pos;
    double* out_vel;
    double* out_planets;          // 9 x 6 or null: the last batch's massive bodies
    int32_t* status;
    int max_loops;
};
int launch_nbody_long(const LongArgs& a, cudaStream_t stream);

// the accelerations at n points (long.cu): spk_accel, or vec_accel under given massive bodies
struct AccelArgs {
    int64_t n;
    const double* jd;       // n (spk_accel)
    const double* pos;      // 3 x n, SSB-centred equatorial
    const double* vel;
    const double* nongrav;  // 10 x n or null
    int n_force;            // spk_accel: PLANETS or MASSES length of the device force table
    int n_massive;          // vec_accel: bodies in massive (6 x n_massive) and bodies
    int simple;             // vec_accel: 1 = SIMPLE_PLANETS (system integration's pair term)
    const double* massive;
    ForceEntry bodies[MAX_FORCE];  // vec_accel with PLANETS / MASSES
    int exact;
    double* out;            // 3 x n
    int32_t* status;
    int32_t* impact_id;     // n or null
};
int launch_accel(const AccelArgs& a, bool vec, cudaStream_t stream);

struct NeatmArgs;
struct FovArgs;
int launch_fov_prefilter(const FovArgs& a, cudaStream_t stream);
int launch_fov_screen(const FovArgs& a, cudaStream_t stream);
int launch_fov_pairs(const FovArgs& a, int64_t m, cudaStream_t stream);
int launch_fov_gather(const FovArgs& a, int64_t m, double* gpos, double* gvel, double* gjd0,
                      double* gjd1, cudaStream_t stream);
int launch_fov_contains(int64_t n_vec, const double* vec, int64_t n_fov, const double* fov,
                        int64_t capacity, unsigned long long* counter, int32_t* out_fov,
                        int32_t* out_idx, cudaStream_t stream);
int launch_fov_finish(const FovArgs& a, int64_t m, const double* npos, const double* nvel,
                      const int32_t* nst, cudaStream_t stream);
int launch_hg_mag(int64_t n, const double* s2obj, const double* s2obs, const double* h,
                  const double* g, double* out, cudaStream_t stream);
int launch_neatm(const NeatmArgs& a, cudaStream_t stream);

}  // namespace kb
