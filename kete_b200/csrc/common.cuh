// common.cuh -- constants, status codes and small FP64 helpers shared by every kernel.
//
// Constants restate kete_core/constants/gravity.rs:9-153 and constants/universal.rs:2-36.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace kb {

// per-object status, mirroring kete_core::errors::Error (kete_core/errors.rs:14-32)
enum Status : int32_t {
    ST_OK = 0,
    ST_CONVERGENCE = 1,
    ST_VALUE_ERROR = 2,
    ST_DAF_LIMITS = 3,
    ST_UNKNOWN_FRAME = 4,
    ST_IO_ERROR = 5,
    ST_IMPACT = 6,
    ST_TIMEOUT = 7,  // a bounded device loop ran out of iterations
    ST_CHECKPOINT_FULL = 8,  // more checkpoints were needed than the caller provided
};

enum Frame : int32_t { FRAME_EQUATORIAL = 1, FRAME_ECLIPTIC = 2 };

constexpr double GMS = 0.00029591220828411956;
constexpr double GMS_SQRT = 0.01720209894996;
constexpr double SUN_J2 = 2.2e-7;
constexpr double EARTH_J2 = 0.00108262998905;
constexpr double JUPITER_J2 = 0.014696572;
constexpr double C_AU_PER_DAY = 173.14463267424034;
constexpr double C_AU_PER_DAY_INV = 0.005775518331436995;
constexpr double C_AU_PER_DAY_INV_SQUARED = 3.33566119967647e-05;
constexpr double AU_KM = 149597870.7;
constexpr double TAU = 6.283185307179586;
constexpr double PI = 3.141592653589793;

// rotation constants and Radau tables computed once on the host (glibc libm) and copied
// to constant memory, so host and device agree bit for bit on them.
struct Tables {
    double rot_c, rot_s;    // cos / sin of the J2000 obliquity
    double spacing[8];      // Gauss-Radau spacings (radau.rs:24-33)
    double w[7], u[7];      // W_VEC / U_VEC (radau.rs:37-51)
    double c[7][7];         // C_MAT (radau.rs:54-66)
    double w_pow[8][7];     // spacing^(k+1) * w[k]
    double u_pow[8][7];     // spacing^(k+1) * u[k]
    double frac2[8];        // spacing^2
    double inv_frac[8];     // 1 / spacing
    double inv_diff[8][8];  // 1 / (spacing[j] - spacing[z])
    double adj_p[7][7];     // b = adj_p (E - a): divided differences, then C_MAT
    double shift_c[7][7];   // binomial C(k+1, m+1) at [m][k], k >= m: b carried to a new step
    // SIMPLE_PLANETS (constants/gravity.rs:137-153) for the system integration:
    // mass (GM, AU^3/day^2), radius (AU), ForceKind, NAIF id
    double simple_mass[9], simple_radius[9];
    int32_t simple_kind[9], simple_naif[9];
};

// LLVM's constant-exponent powi: repeated squaring, reciprocal for negative exponents.
template <int N>
__host__ __device__ __forceinline__ double powi(double x) {
    constexpr int A = N < 0 ? -N : N;
    double res = 1.0;
    bool have = false;
    double sq = x;
#pragma unroll
    for (int v = A; v; v >>= 1) {
        if (v & 1) {
            res = have ? res * sq : sq;
            have = true;
        }
        if (v >> 1) sq = sq * sq;
    }
    if (N < 0) res = 1.0 / res;
    return res;
}

__host__ __device__ __forceinline__ double norm3(double x, double y, double z) {
    return sqrt(x * x + y * y + z * z);
}

// f64::clamp keeps NaN
__host__ __device__ __forceinline__ double clampd(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

}  // namespace kb
