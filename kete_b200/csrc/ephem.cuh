// ephem.cuh -- SPK type-2 ephemeris resident in device memory.
//
// Restates SpkCollection::try_get_raw_state (kete_core/spice/spk.rs:65-82),
// SpkSegmentType2::try_get_pos_vel (kete_core/spice/spk_segments.rs:355-376) and
// chebyshev_evaluate_both (kete_core/spice/interpolation.rs:25-77).
//
// Device layout.  Every type-2 record is re-laid out by the host as
//   [mid_s, radius_s, 1/radius_s, 86400/radius_s/AU_KM, x[npad], y[npad], z[npad]]
// with npad = n_coef rounded up to an even count (zero padding), so each coefficient
// block starts on a 16-byte boundary and is read with double2 loads.  Segments are
// grouped per body in the reference's scan order; the table lives in constant memory
// (uniform across a warp), the coefficient pool in global memory (L2 resident: ~0.5 MB
// for a decade of planetary ephemeris).
#pragma once
#include "common.cuh"

namespace kb {

constexpr int MAX_SEG = 96;
constexpr int MAX_SLOT = 32;
constexpr int MAX_FORCE = 16;
constexpr int MAX_CHAIN = 3;
// span ordering of the persistent N-body grid: buckets and scratch header size (ints)
constexpr int ORDER_BUCKETS = 64;
constexpr int ORDER_SCRATCH_HEADER = 256;

struct SegDesc {
    double jd_start, jd_end;  // JD, as spice_jds_to_jd(summary) (spice/mod.rs:25-28)
    double start_s;           // jd_to_spice_jd(jd_start), what the reference indexes from
    double intlen;            // record length in seconds (INTLEN)
    double inv_intlen;        // 1 / intlen
    int64_t offset;           // doubles into the pool of record 0
    int32_t n_coef, n_pad, n_rec, rsize;
};

// One body id with its segments [first, first+count) and the slot of its centre body
// (-1 when the centre is the solar-system barycentre 0).
struct Slot {
    int32_t naif_id;
    int32_t center_id;
    int32_t first, count;
    int32_t parent_slot;
    int32_t pad_;
};

// Force model entry (GravParams, kete_core/constants/gravity.rs:155-216).
enum ForceKind : int32_t { FK_PLAIN = 0, FK_SUN = 1, FK_JUPITER = 2, FK_EARTH = 3 };
struct ForceEntry {
    double mass, radius;
    int32_t slot, kind, naif_id, pad_;
};

// Chain of SPK slots from a state's centre up to the barycentre (empty for centre 0).
struct CenterChain {
    int len = 0;
    int slot[3] = {-1, -1, -1};
};

struct EphemConst {
    int32_t n_seg, n_slot;
    int32_t n_force_planets, n_force_all;  // PLANETS (10) and MASSES (15) lengths
    int32_t sun_slot, loaded;
    SegDesc seg[MAX_SEG];
    Slot slot[MAX_SLOT];
    ForceEntry force[MAX_FORCE];
    const double* pool;
};

// Evaluate one record: position (AU) and velocity (AU/day) of the segment's body.
__device__ __forceinline__ void cheb_record(const double* __restrict__ rec, int n_coef, int n_pad,
                                            double tau_num, double p[3], double v[3]) {
    const double2 hdr0 = __ldg(reinterpret_cast<const double2*>(rec));      // mid, radius
    const double2 hdr1 = __ldg(reinterpret_cast<const double2*>(rec + 2));  // 1/radius, tss
    const double x = (tau_num - hdr0.x) * hdr1.x;
    const double x2 = 2.0 * x;
    const double2* cx = reinterpret_cast<const double2*>(rec + 4);
    const double2* cy = reinterpret_cast<const double2*>(rec + 4 + n_pad);
    const double2* cz = reinterpret_cast<const double2*>(rec + 4 + 2 * n_pad);
    double2 ax = __ldg(cx), ay = __ldg(cy), az = __ldg(cz);
    double vx = ax.x + ax.y * x, vy = ay.x + ay.y * x, vz = az.x + az.y * x;
    double dx = ax.y, dy = ay.y, dz = az.y;
    double second_t = 1.0, last_t = x;
    double second_u = 1.0, last_u = x2;
    // coefficients idx = 2 .. n_coef-1, two per double2 load
    for (int k = 1; 2 * k < n_coef; ++k) {
        ax = __ldg(cx + k);
        ay = __ldg(cy + k);
        az = __ldg(cz + k);
        {
            const double idx = (double)(2 * k);
            double next_t = x2 * last_t - second_t;
            vx += ax.x * next_t;
            vy += ay.x * next_t;
            vz += az.x * next_t;
            second_t = last_t;
            last_t = next_t;
            double next_u = x2 * last_u - second_u;
            const double lu = last_u * idx;
            dx += ax.x * lu;
            dy += ay.x * lu;
            dz += az.x * lu;
            second_u = last_u;
            last_u = next_u;
        }
        if (2 * k + 1 < n_coef) {
            const double idx = (double)(2 * k + 1);
            double next_t = x2 * last_t - second_t;
            vx += ax.y * next_t;
            vy += ay.y * next_t;
            vz += az.y * next_t;
            second_t = last_t;
            last_t = next_t;
            double next_u = x2 * last_u - second_u;
            const double lu = last_u * idx;
            dx += ax.y * lu;
            dy += ay.y * lu;
            dz += az.y * lu;
            second_u = last_u;
            last_u = next_u;
        }
    }
    constexpr double INV_AU_KM = 1.0 / AU_KM;
    p[0] = vx * INV_AU_KM;
    p[1] = vy * INV_AU_KM;
    p[2] = vz * INV_AU_KM;
    const double tss = hdr1.y;
    v[0] = dx * tss;
    v[1] = dy * tss;
    v[2] = dz * tss;
}

// try_get_raw_state for the body in `slot`: first segment (scan order) whose
// [jd_start, jd_end] contains jd.
__device__ __forceinline__ int eph_raw(const EphemConst& E, int slot, double jd, double p[3],
                                       double v[3]) {
    const Slot& s = E.slot[slot];
    for (int q = 0; q < s.count; ++q) {
        const SegDesc& d = E.seg[s.first + q];
        if (jd >= d.jd_start && jd <= d.jd_end) {
            // jd_to_spice_jd (spice/mod.rs:31-34), rounded as the reference rounds it: an
            // explicit multiply so the compiler cannot fuse it into the subtraction below
            const double jds = __dmul_rn(jd - 2451545.0, 86400.0);
            // record index floor((t - start) / intlen) (spk_segments.rs:358); the quotient
            // is formed with the tabulated reciprocal
            double fidx = floor((jds - d.start_s) * d.inv_intlen);
            int idx = fidx < 0.0 ? 0 : (fidx >= (double)d.n_rec ? d.n_rec - 1 : (int)fidx);
            const double* rec = E.pool + d.offset + (int64_t)idx * d.rsize;
            cheb_record(rec, d.n_coef, d.n_pad, jds, p, v);
            return ST_OK;
        }
    }
    return ST_DAF_LIMITS;
}

}  // namespace kb
