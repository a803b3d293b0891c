// fov_args.h -- launch arguments of the field-of-view kernels (shared by host and device code).
#pragma once
#include <cstdint>

namespace kb {

constexpr int FOV_TILE = 128;   // fields staged in shared memory per pass
// doubles per field (patch): observer jd, pos[3], vel[3], then 12 patch parameters and the
// patch kind: 0 rectangle (4 edge normals), 1 cone (unit pointing[3], half-angle),
// 2 omnidirectional (no parameters)
constexpr int FOV_STRIDE = 20;
constexpr int FOV_KIND_ROW = 19;

struct FovArgs {
    int64_t n_obj;
    const double* pos;  // 3 x n_obj
    const double* vel;
    const double* jd;
    const uint8_t* valid;  // may be null: all valid
    int64_t n_fov;
    const double* fov;     // FOV_STRIDE x n_fov (column per field)
    double dt_limit;
    int64_t capacity;      // visible outputs
    int64_t cand_capacity; // n-body candidates
    int64_t pair_capacity; // (field, object) pairs that pass the linear screen
    unsigned long long* counters;  // [0] visible, [1] n-body candidates, [2] screened pairs
    int32_t* out_fov;
    int32_t* out_obj;
    double* out_state;     // 7 x capacity
    int32_t* cand_fov;
    int32_t* cand_obj;
    int32_t* pair_fov;
    int32_t* pair_obj;
};

}  // namespace kb
