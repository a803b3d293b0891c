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
// span ordering of the persistent N-body grid: work buckets, and the scratch header (ints):
// [0] object queue, [1 ..] bucket histogram, then the bucket cursors (ORDER_BUCKETS work
// buckets, then one bucket for the objects with a non-gravitational model and one for the
// objects whose span leaves the fast plan's window; the first two kinds only when the caller
// asks for the split), ORDER_RANGE: {0, start of the non-gravitational bucket, start of the
// outside bucket, n}, ORDER_QUEUE2: the queue of the objects outside the window,
// ORDER_QUEUE3: the queue of the non-gravitational bucket; the processing order follows the
// header
constexpr int ORDER_BUCKETS = 120;
constexpr int ORDER_NG_BUCKET = ORDER_BUCKETS;
constexpr int ORDER_OUT_BUCKET = ORDER_BUCKETS + 1;
constexpr int ORDER_ALL_BUCKETS = ORDER_BUCKETS + 2;
constexpr int ORDER_RANGE = 1 + 2 * ORDER_ALL_BUCKETS;
constexpr int ORDER_QUEUE2 = ORDER_RANGE + 4;
constexpr int ORDER_QUEUE3 = ORDER_RANGE + 5;
constexpr int EPH_CACHE = 38;  // body-position cache, doubles per lane (the planets need 36)

constexpr int ORDER_SCRATCH_HEADER = 256;

// Segment types held on the device: 2 and 3 (Chebyshev position / position and velocity),
// 1 and 21 (modified difference arrays).
struct SegDesc {
    double jd_start, jd_end;  // JD, as spice_jds_to_jd(summary) (spice/mod.rs:25-28)
    double start_s;           // jd_to_spice_jd(jd_start), what the reference indexes from
    double intlen;            // types 2, 3: record length in seconds (INTLEN)
    double inv_intlen;        // 1 / intlen
    int64_t offset;           // doubles into the pool of record 0
    int64_t epoch_offset;     // types 1, 21: doubles into the pool of the final-epoch list
    int32_t n_coef;           // types 2, 3: coefficients per coordinate; 1, 21: MAXDIM
    int32_t n_pad, n_rec, rsize;
    int32_t type, pad_;
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

// Fast evaluation plan: inside [fast_lo, fast_hi] every force body and every centre it is
// chained through is covered by its first segment (the one the reference's scan returns),
// all with FAST_NC coefficients.  Items are evaluated two at a time in this order; an item
// is either a force body (role = index into force[]) or a centre kept for the bodies after
// it (role = -1).
constexpr int FAST_NC = 14;
constexpr int MAX_ITEMS = 24;
// One item of the fast plan, holding everything its evaluation reads (its segment's record
// table and, for a force body, the body's gravity parameters), so the force loop makes no
// dependent table lookups.
struct FastItem {
    int64_t offset;                     // pool offset of the segment's record 0
    double start_s, inv_intlen, n_rec;  // record = clamp(floor((t - start_s) * inv_intlen))
    double mass, radius;
    int32_t rsize;    // doubles per record
    int32_t role;     // -2 padding, -1 a centre kept for later bodies, else the force index
    int32_t kind;     // ForceKind of a force body
    int32_t naif_id;
    int32_t chained;  // 1: the body is centred on the kept centre (add its position)
    int32_t pad_;
};

// The first n_vel items are the bodies whose velocity enters the force (relativistic
// correction of the Sun and Jupiter, non-gravitational term relative to the Sun): they are
// evaluated two at a time with velocities.  The others (bodies whose position alone enters,
// and centres) follow in the reference's order, three at a time, positions only; role -2
// pads their count to a multiple of three.
struct FastPlan {
    double lo, hi;
    int32_t n_items, ok;
    int32_t n_vel;
    int32_t sun_vel;  // index of the Sun among the first n_vel items (-1: no Sun)
    FastItem item[MAX_ITEMS];
};

// Body cache of the warp-pooled node kernel (radau_pool.cuh), doubles per lane: position and
// velocity of the first n_vel items, positions of every other item but padding (centres
// included: the bodies chained to them add the centre's position when the force terms read
// them).  The planets need 39.
constexpr int POOL_CACHE_DOUBLES = 40;
inline __host__ __device__ int pool_plan_doubles(const FastPlan& P) {
    int k = 6 * P.n_vel;
    for (int it = P.n_vel; it < P.n_items; ++it)
        if (P.item[it].role != -2) k += 3;
    return k;
}

// Doubles a lane's body-position cache needs for a fast plan (SpkForceT::fast_positions):
// position and velocity of the first n_vel bodies, positions of the other force bodies.
inline __host__ __device__ int fast_plan_cache_doubles(const FastPlan& P) {
    int k = 6 * P.n_vel;
    for (int it = P.n_vel; it < P.n_items; ++it)
        if (P.item[it].role >= 0) k += 3;
    return k;
}

struct EphemConst {
    int32_t n_seg, n_slot;
    int32_t n_force_planets, n_force_all;  // PLANETS (10) and MASSES (15) lengths
    int32_t sun_slot, loaded;
    FastPlan fast_planets, fast_all;
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

// Position/velocity of two records evaluated in lockstep (two independent recurrence chains),
// NC coefficients per coordinate.  KU: coefficient pairs per unrolled loop body (a small
// body keeps the lane-parallel kernels' code in the instruction cache; the one-object-per-
// thread kernel prefers the loop fully unrolled).
template <int NC, int KU = NC>
__device__ __forceinline__ void cheb_pair(const double* __restrict__ ra, const double* __restrict__ rb,
                                          double jds, double pa[3], double va[3], double pb[3],
                                          double vb[3]) {
    constexpr int NP = (NC + 1) & ~1;
    const double2 ha0 = __ldg(reinterpret_cast<const double2*>(ra));
    const double2 ha1 = __ldg(reinterpret_cast<const double2*>(ra + 2));
    const double2 hb0 = __ldg(reinterpret_cast<const double2*>(rb));
    const double2 hb1 = __ldg(reinterpret_cast<const double2*>(rb + 2));
    const double xa = (jds - ha0.x) * ha1.x, xb = (jds - hb0.x) * hb1.x;
    const double xa2 = 2.0 * xa, xb2 = 2.0 * xb;
    const double2* cxa = reinterpret_cast<const double2*>(ra + 4);
    const double2* cya = reinterpret_cast<const double2*>(ra + 4 + NP);
    const double2* cza = reinterpret_cast<const double2*>(ra + 4 + 2 * NP);
    const double2* cxb = reinterpret_cast<const double2*>(rb + 4);
    const double2* cyb = reinterpret_cast<const double2*>(rb + 4 + NP);
    const double2* czb = reinterpret_cast<const double2*>(rb + 4 + 2 * NP);
    double2 ax = __ldg(cxa), ay = __ldg(cya), az = __ldg(cza);
    double2 bx = __ldg(cxb), by = __ldg(cyb), bz = __ldg(czb);
    double avx = ax.x + ax.y * xa, avy = ay.x + ay.y * xa, avz = az.x + az.y * xa;
    double bvx = bx.x + bx.y * xb, bvy = by.x + by.y * xb, bvz = bz.x + bz.y * xb;
    double adx = ax.y, ady = ay.y, adz = az.y;
    double bdx = bx.y, bdy = by.y, bdz = bz.y;
    double at2 = 1.0, at1 = xa, au2 = 1.0, au1 = xa2;
    double bt2 = 1.0, bt1 = xb, bu2 = 1.0, bu1 = xb2;
#pragma unroll KU
    for (int k = 1; 2 * k < NC; ++k) {
        ax = __ldg(cxa + k); ay = __ldg(cya + k); az = __ldg(cza + k);
        bx = __ldg(cxb + k); by = __ldg(cyb + k); bz = __ldg(czb + k);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int idx = 2 * k + h;
            if (idx < NC) {
                const double cax = h ? ax.y : ax.x, cay = h ? ay.y : ay.x, caz = h ? az.y : az.x;
                const double cbx = h ? bx.y : bx.x, cby = h ? by.y : by.x, cbz = h ? bz.y : bz.x;
                const double fi = (double)idx;
                const double ant = xa2 * at1 - at2, bnt = xb2 * bt1 - bt2;
                avx += cax * ant; avy += cay * ant; avz += caz * ant;
                bvx += cbx * bnt; bvy += cby * bnt; bvz += cbz * bnt;
                at2 = at1; at1 = ant;
                bt2 = bt1; bt1 = bnt;
                const double anu = xa2 * au1 - au2, bnu = xb2 * bu1 - bu2;
                const double alu = au1 * fi, blu = bu1 * fi;
                adx += cax * alu; ady += cay * alu; adz += caz * alu;
                bdx += cbx * blu; bdy += cby * blu; bdz += cbz * blu;
                au2 = au1; au1 = anu;
                bu2 = bu1; bu1 = bnu;
            }
        }
    }
    constexpr double INV_AU_KM = 1.0 / AU_KM;
    pa[0] = avx * INV_AU_KM; pa[1] = avy * INV_AU_KM; pa[2] = avz * INV_AU_KM;
    pb[0] = bvx * INV_AU_KM; pb[1] = bvy * INV_AU_KM; pb[2] = bvz * INV_AU_KM;
    va[0] = adx * ha1.y; va[1] = ady * ha1.y; va[2] = adz * ha1.y;
    vb[0] = bdx * hb1.y; vb[1] = bdy * hb1.y; vb[2] = bdz * hb1.y;
}

// Positions of three records evaluated in lockstep (value recurrence only), NC coefficients;
// KU as for cheb_pair.
template <int NC, int KU = NC>
__device__ __forceinline__ void cheb_pos3(const double* __restrict__ ra, const double* __restrict__ rb,
                                          const double* __restrict__ rc, double jds, double pa[3],
                                          double pb[3], double pc[3]) {
    constexpr int NP = (NC + 1) & ~1;
    const double* r[3] = {ra, rb, rc};
    double xx[3], x2[3], t1[3], t2[3], acc[3][3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double2 h0 = __ldg(reinterpret_cast<const double2*>(r[q]));
        const double2 h1 = __ldg(reinterpret_cast<const double2*>(r[q] + 2));
        xx[q] = (jds - h0.x) * h1.x;
        x2[q] = 2.0 * xx[q];
        t2[q] = 1.0;
        t1[q] = xx[q];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double2 a = __ldg(reinterpret_cast<const double2*>(r[q] + 4 + c * NP));
            acc[q][c] = a.x + a.y * xx[q];
        }
    }
#pragma unroll KU
    for (int k = 1; 2 * k < NC; ++k) {
        double2 co[3][3];
#pragma unroll
        for (int q = 0; q < 3; ++q)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                co[q][c] = __ldg(reinterpret_cast<const double2*>(r[q] + 4 + c * NP) + k);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (2 * k + h < NC) {
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const double nt = x2[q] * t1[q] - t2[q];
#pragma unroll
                    for (int c = 0; c < 3; ++c) acc[q][c] += (h ? co[q][c].y : co[q][c].x) * nt;
                    t2[q] = t1[q];
                    t1[q] = nt;
                }
            }
        }
    }
    constexpr double INV_AU_KM = 1.0 / AU_KM;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        pa[c] = acc[0][c] * INV_AU_KM;
        pb[c] = acc[1][c] * INV_AU_KM;
        pc[c] = acc[2][c] * INV_AU_KM;
    }
}

// Record of a fast-plan item holding TDB seconds `jds` (index clamped to the segment).
__device__ __forceinline__ const double* fast_record(const double* pool, const FastItem& I,
                                                     double jds) {
    const double fidx = floor((jds - I.start_s) * I.inv_intlen);
    const int idx = fidx < 0.0 ? 0 : (fidx >= I.n_rec ? (int)I.n_rec - 1 : (int)fidx);
    return pool + I.offset + (int64_t)idx * I.rsize;
}

// Record of segment `seg` holding TDB seconds `jds` (index clamped to the segment).
__device__ __forceinline__ const double* eph_record(const EphemConst& E, int seg, double jds) {
    const SegDesc& d = E.seg[seg];
    const double fidx = floor((jds - d.start_s) * d.inv_intlen);
    const int idx = fidx < 0.0 ? 0 : (fidx >= (double)d.n_rec ? d.n_rec - 1 : (int)fidx);
    return E.pool + d.offset + (int64_t)idx * d.rsize;
}

// Type 3 record (SpkSegmentType3::try_get_pos_vel, spk_segments.rs:446-480): position and
// velocity from their own Chebyshev series, values only.  Device layout:
//   [mid_s, radius_s, 1/radius_s, 86400/AU_KM, x, y, z, vx, vy, vz] (n_pad each)
__device__ __forceinline__ void cheb_record3(const double* __restrict__ rec, int n_coef, int n_pad,
                                             double tau_num, double p[3], double v[3]) {
    const double x = (tau_num - rec[0]) * rec[2];
    const double x2 = 2.0 * x;
    double acc[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] = rec[4 + c * n_pad] + rec[4 + c * n_pad + 1] * x;
    double second_t = 1.0, last_t = x;
    for (int k = 2; k < n_coef; ++k) {
        const double next_t = x2 * last_t - second_t;
#pragma unroll
        for (int c = 0; c < 6; ++c) acc[c] += rec[4 + c * n_pad + k] * next_t;
        second_t = last_t;
        last_t = next_t;
    }
    constexpr double INV_AU_KM = 1.0 / AU_KM;
    const double vs = rec[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        p[c] = acc[c] * INV_AU_KM;
        v[c] = acc[3 + c] * vs;
    }
}

// Types 1 and 21 (SpkSegmentType1 / 21::try_get_pos_vel, spk_segments.rs:207-290,
// 1008-1090; SPICE's SPKE21): the modified difference array of the first record whose final
// epoch is at or after t.  Records are kept as the DAF stores them (4*MAXDIM + 11 doubles);
// the host has checked every record's orders and step sizes, so the indices below stay in
// bounds (KQMAX1 <= MAXDIM + 1 <= 26, KQ <= KQMAX1 - 1, no zero step).
// work: 76 doubles per thread at work[k * stride] (shared memory), or null for local arrays.
__device__ __forceinline__ void mda_record(const double* __restrict__ pool, const SegDesc& d,
                                           double jds, double p[3], double v[3],
                                           double* work = nullptr, int stride = 1) {
    const double* epochs = pool + d.epoch_offset;
    int lo = 0, hi = d.n_rec;
    while (lo < hi) {  // first record whose final epoch is >= jds
        const int mid = (lo + hi) >> 1;
        if (epochs[mid] < jds) lo = mid + 1;
        else hi = mid;
    }
    if (lo >= d.n_rec) lo = d.n_rec - 1;
    const int md = d.n_coef;
    const double* rec = pool + d.offset + (int64_t)lo * d.rsize;
    const double* g = rec + 1;
    const double* ref = rec + 1 + md;
    const double* dt_arr = rec + 7 + md;
    const int kqmax1 = (int)rec[4 * md + 7];
    const double delta = jds - rec[0];
    double lfc[25], lwc[25], lw[26];
    // the work arrays: the caller's shared-memory columns, or this thread's local arrays
    const int sd = work ? stride : 1;
    double* fcp = work ? work : lfc;
    double* wcp = work ? work + 25 * stride : lwc;
    double* wp = work ? work + 50 * stride : lw;
#define FC(j) fcp[(j) * sd]
#define WC(j) wcp[(j) * sd]
#define WW(j) wp[(j) * sd]
    double tp = delta;
    for (int j = 0; j < kqmax1 - 2; ++j) {
        FC(j) = tp / g[j];
        WC(j) = delta / g[j];
        tp = delta + g[j];
    }
    for (int j = 0; j < kqmax1; ++j) WW(j) = 1.0 / (double)(j + 1);
    int ks = kqmax1 - 1, ks1 = ks - 1, jx = 0;
    while (ks >= 2) {
        jx += 1;
        for (int j = 0; j < jx; ++j) WW(j + ks) = FC(j) * WW(j + ks1) - WC(j) * WW(j + ks);
        ks = ks1;
        ks1 -= 1;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double sum = 0.0;
        for (int j = (int)rec[4 * md + 8 + c]; j >= 1; --j) sum += dt_arr[c * md + j - 1] * WW(j + ks - 1);
        p[c] = (ref[2 * c] + delta * (sum * delta + ref[2 * c + 1])) / AU_KM;
    }
    for (int j = 0; j < jx; ++j) WW(j + ks) = FC(j) * WW(j + ks1) - WC(j) * WW(j + ks);
    ks -= 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double sum = 0.0;
        for (int j = (int)rec[4 * md + 8 + c]; j >= 1; --j) sum += dt_arr[c * md + j - 1] * WW(j + ks - 1);
        v[c] = (ref[2 * c + 1] + delta * sum) / AU_KM * 86400.0;
    }
#undef FC
#undef WC
#undef WW
}

// try_get_raw_state for the body in `slot`: first segment (scan order) whose
// [jd_start, jd_end] contains jd.
__device__ __forceinline__ int eph_raw(const EphemConst& E, int slot, double jd, double p[3],
                                       double v[3], double* work = nullptr, int stride = 1) {
    const Slot& s = E.slot[slot];
    for (int q = 0; q < s.count; ++q) {
        const SegDesc& d = E.seg[s.first + q];
        if (jd >= d.jd_start && jd <= d.jd_end) {
            // jd_to_spice_jd (spice/mod.rs:31-34), rounded as the reference rounds it: an
            // explicit multiply so the compiler cannot fuse it into the subtraction below
            const double jds = __dmul_rn(jd - 2451545.0, 86400.0);
            if (d.type == 1 || d.type == 21) {
                mda_record(E.pool, d, jds, p, v, work, stride);
                return ST_OK;
            }
            // record index floor((t - start) / intlen) (spk_segments.rs:358); the quotient
            // is formed with the tabulated reciprocal
            double fidx = floor((jds - d.start_s) * d.inv_intlen);
            int idx = fidx < 0.0 ? 0 : (fidx >= (double)d.n_rec ? d.n_rec - 1 : (int)fidx);
            const double* rec = E.pool + d.offset + (int64_t)idx * d.rsize;
            if (d.type == 3) cheb_record3(rec, d.n_coef, d.n_pad, jds, p, v);
            else cheb_record(rec, d.n_coef, d.n_pad, jds, p, v);
            return ST_OK;
        }
    }
    return ST_DAF_LIMITS;
}

}  // namespace kb
