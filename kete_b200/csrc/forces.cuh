// forces.cuh -- accelerations used by the Radau integrators.
//
// SpkForce restates spk_accel (kete_core/propagation/acceleration.rs:121-168) with
// GravParams::add_acceleration, j2_correction and apply_gr_correction
// (kete_core/constants/gravity.rs:171-253) and NonGravModel::add_acceleration
// (kete_core/propagation/nongrav.rs:114-157).  Bodies are summed in the reference's
// order (Sun, Mercury, Venus, Earth, Moon, Mars, Jupiter, Saturn, Uranus, Neptune).  A
// body whose SPK centre is not the barycentre (Earth and Moon, centred on the Earth-Moon
// barycentre) reuses the centre state evaluated for the previous body when it is the same
// centre, so a force evaluation costs 11 Chebyshev records instead of the reference's 12.
#pragma once
#include "common.cuh"
#include "ephem.cuh"
#include "kepler.cuh"

namespace kb {

// Device constants.  Every kernel translation unit (kernels.cu, nodes.cu, sens.cu, adjoint.cu,
// long.cu)
// holds its own copy (internal linkage); KB_CONSTANT_UPLOADER defines the TU's writer and
// upload_tables / upload_ephem call all of them.
static __constant__ Tables c_tab;
static __constant__ EphemConst c_eph;

// Defines upload_consts_<tu>(tables, ephem): copies whichever argument is non-null into this
// translation unit's constants.
#define KB_CONSTANT_UPLOADER(tu)                                                              \
    int upload_consts_##tu(const Tables* t, const EphemConst* e) {                            \
        if (t) {                                                                               \
            const int rc = cuda_check(cudaMemcpyToSymbol(c_tab, t, sizeof(Tables)),            \
                                      "upload Radau tables (" #tu ")");                        \
            if (rc) return rc;                                                                 \
        }                                                                                      \
        if (e)                                                                                 \
            return cuda_check(cudaMemcpyToSymbol(c_eph, e, sizeof(EphemConst)),                \
                              "upload ephemeris table (" #tu ")");                             \
        return 0;                                                                              \
    }

__device__ __forceinline__ void eq_to_ecl(const double v[3], double o[3]) {
    const double c = c_tab.rot_c, s = c_tab.rot_s;
    const double y = c * v[1] + s * v[2];
    const double z = -s * v[1] + c * v[2];
    o[0] = v[0];
    o[1] = y;
    o[2] = z;
}
__device__ __forceinline__ void ecl_to_eq(const double v[3], double o[3]) {
    const double c = c_tab.rot_c, s = c_tab.rot_s;
    const double y = c * v[1] - s * v[2];
    const double z = s * v[1] + c * v[2];
    o[0] = v[0];
    o[1] = y;
    o[2] = z;
}

__device__ __forceinline__ void j2_correction(const double rp[3], double radius, double j2,
                                              double mass, double o[3]) {
    const double r = norm3(rp[0], rp[1], rp[2]);
    const double zr = rp[2] / r;
    const double z_squared = 5.0 * (zr * zr);
    const double rr = radius / r;
    const double coef = 1.5 * j2 * mass * (rr * rr) * powi<-3>(r);
    o[0] = rp[0] * coef * (z_squared - 1.0);
    o[1] = rp[1] * coef * (z_squared - 1.0);
    o[2] = rp[2] * coef * (z_squared - 3.0);
}

__device__ __forceinline__ void apply_gr(double acc[3], const double rp[3], const double rv[3],
                                         double mass, double r) {
    const double r_v = 4.0 * (rp[0] * rv[0] + rp[1] * rv[1] + rp[2] * rv[2]);
    const double rel_v2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
    const double gr_const = mass * C_AU_PER_DAY_INV_SQUARED * powi<-3>(r);
    const double c = 4. * mass / r - rel_v2;
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[i] += gr_const * (c * rp[i] + r_v * rv[i]);
}

// Per-object non-gravitational model row: kind (0 none, 1 JPL comet, 2 dust) then
// a1 a2 a3 alpha r0 m n k dt (JPL) or beta (dust).  Stored column-major (10 x n).
struct NonGrav {
    const double* __restrict__ base;
    int64_t stride;
    int kind;
    __device__ __forceinline__ double p(int k) const { return __ldg(base + (int64_t)k * stride); }
};

// The non-gravitational acceleration (NonGravModel::add_acceleration, nongrav.rs:114-157)
// at the Sun-relative position rp and velocity rv, returned for the caller to add.  DT =
// false: the JPL comet model's delay dt is known to be 0 (no two-body back-propagation).
template <bool DT>
__device__ __forceinline__ double3 nongrav_terms(const NonGrav ng, const double3 rp, const double3 rv) {
    const double pos_in[3] = {rp.x, rp.y, rp.z};
    const double vel[3] = {rv.x, rv.y, rv.z};
    double acc[3] = {0.0, 0.0, 0.0};
    if (ng.kind == 2) {
        const double beta = ng.p(1);
        const double n = norm3(pos_in[0], pos_in[1], pos_in[2]);
        const double pn[3] = {pos_in[0] / n, pos_in[1] / n, pos_in[2] / n};
        const double r_dot = pn[0] * vel[0] + pn[1] * vel[1] + pn[2] * vel[2];
        const double norm2_inv =
            1.0 / (pos_in[0] * pos_in[0] + pos_in[1] * pos_in[1] + pos_in[2] * pos_in[2]);
        const double scaling = GMS * beta * norm2_inv;
#pragma unroll
        for (int i = 0; i < 3; ++i)
            acc[i] += scaling * ((1.0 - r_dot * C_AU_PER_DAY_INV_SQUARED) * pn[i] -
                                 vel[i] * C_AU_PER_DAY_INV_SQUARED);
        return make_double3(acc[0], acc[1], acc[2]);
    }
    const double a1 = ng.p(1), a2 = ng.p(2), a3 = ng.p(3), alpha = ng.p(4), r_0 = ng.p(5);
    const double m = ng.p(6), nn = ng.p(7), k = ng.p(8), dt = ng.p(9);
    double pos[3] = {pos_in[0], pos_in[1], pos_in[2]};
    const double pnorm = norm3(pos[0], pos[1], pos[2]);
    const double pn[3] = {pos[0] / pnorm, pos[1] / pnorm, pos[2] / pnorm};
    const double vdp = vel[0] * pn[0] + vel[1] * pn[1] + vel[2] * pn[2];
    double tv[3] = {vel[0] - pn[0] * vdp, vel[1] - pn[1] * vdp, vel[2] - pn[2] * vdp};
    const double tn = norm3(tv[0], tv[1], tv[2]);
    const double t_vec[3] = {tv[0] / tn, tv[1] / tn, tv[2] / tn};
    double nv[3] = {t_vec[1] * pn[2] - t_vec[2] * pn[1], t_vec[2] * pn[0] - t_vec[0] * pn[2],
                    t_vec[0] * pn[1] - t_vec[1] * pn[0]};
    const double nnrm = norm3(nv[0], nv[1], nv[2]);
    const double n_vec[3] = {nv[0] / nnrm, nv[1] / nnrm, nv[2] / nnrm};
    if (DT && dt != 0.0) {
        double p2[3] = {pos[0], pos[1], pos[2]}, v2[3] = {vel[0], vel[1], vel[2]};
        if (analytic_2_body(-dt, p2, v2) == ST_OK) {
            pos[0] = p2[0];
            pos[1] = p2[1];
            pos[2] = p2[2];
        }
    }
    const double rr0 = norm3(pos[0], pos[1], pos[2]) / r_0;
    const double scale = alpha * pow(rr0, -m) * pow(1.0 + pow(rr0, nn), -k);
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[i] += pn[i] * (scale * a1);
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[i] += t_vec[i] * (scale * a2);
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[i] += n_vec[i] * (scale * a3);
    return make_double3(acc[0], acc[1], acc[2]);
}

// nongrav_terms out of line: its arrays are its own, and the force loops that call it do not
// carry its registers.
static __device__ __noinline__ double3 nongrav_accel(const NonGrav ng, const double3 rp, const double3 rv) {
    return nongrav_terms<true>(ng, rp, rv);
}

// -------------------------------------------------------------------------------------------
// centre / frame changes around the integration (kete_core/propagation/mod.rs:76-80,
// 107-116 with SpkCollection::try_change_center, spk.rs:99-126, and State::try_change_center,
// state.rs:242-281): the SPK states are expressed in the object's frame before they are
// added, then the sum is rotated into the integration frame (equatorial).
// -------------------------------------------------------------------------------------------
__device__ __forceinline__ int to_ssb_equatorial(double t, int frame, const CenterChain& ch,
                                                 double p[3], double v[3]) {
    for (int k = 0; k < ch.len; ++k) {
        double sp[3], sv[3];
        if (eph_raw(c_eph, ch.slot[k], t, sp, sv) != ST_OK) return ST_DAF_LIMITS;
        if (frame == FRAME_ECLIPTIC) {
            double q[3];
            eq_to_ecl(sp, q);
            sp[0] = q[0]; sp[1] = q[1]; sp[2] = q[2];
            eq_to_ecl(sv, q);
            sv[0] = q[0]; sv[1] = q[1]; sv[2] = q[2];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            p[i] += sp[i];
            v[i] += sv[i];
        }
    }
    if (frame == FRAME_ECLIPTIC) {
        double q[3];
        ecl_to_eq(p, q);
        p[0] = q[0]; p[1] = q[1]; p[2] = q[2];
        ecl_to_eq(v, q);
        v[0] = q[0]; v[1] = q[1]; v[2] = q[2];
    }
    return ST_OK;
}

__device__ __forceinline__ int from_ssb_equatorial(double t, int frame, const CenterChain& ch,
                                                   double p[3], double v[3]) {
    for (int k = ch.len - 1; k >= 0; --k) {
        double sp[3], sv[3];
        if (eph_raw(c_eph, ch.slot[k], t, sp, sv) != ST_OK) return ST_DAF_LIMITS;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            p[i] += -sp[i];
            v[i] += -sv[i];
        }
    }
    if (frame == FRAME_ECLIPTIC) {
        double q[3];
        eq_to_ecl(p, q);
        p[0] = q[0]; p[1] = q[1]; p[2] = q[2];
        eq_to_ecl(v, q);
        v[0] = q[0]; v[1] = q[1]; v[2] = q[2];
    }
    return ST_OK;
}

// Per-lane cache of the bodies' positions at one time (the fast plan's layout, see
// SpkForceT::fast_positions) in shared memory: slot k of a lane at p[k * stride].
struct EphCache {
    double* p;
    int stride;
    bool on;   // the plan fits and the cache is in use
    double t;  // time of the cached positions (NaN: none)
};

// Acceleration from the SPK perturbers (spk_accel, acceleration.rs:121-168).  KU: the
// Chebyshev loops' unrolling (cheb_pair); SpkForce is the lane-parallel kernels' compact form.
// NGI: the JPL comet model without delay inline in the Sun's term (the other models stay a
// call).  The inline code pays where every object carries the model (the differentiation
// kernels on 4,096 comets: checkpointed forward 12.7 -> 12.0 ms, adjoint 15.0 -> 14.8 ms,
// sensitivities 61.7 -> 59.8 ms) and costs where few do (the node and thread kernels on the
// 1M mix with 5% comets: 5% slower).
template <int KU, bool NGI = false>
struct SpkForceT {
    int n_force;
    NonGrav ng;
    // outputs of exact evaluations
    int32_t impact_id;
    double min_dist;  // smallest distance to a non-Sun body seen at exact evals
    int32_t min_id;

    // One body's contribution (GravParams::add_acceleration, gravity.rs:171-216, plus the
    // non-gravitational term relative to the Sun, acceleration.rs:161-165), given the relative
    // position rp and velocity rv, r2 = |rp|^2 and ir = rsqrt(r2).  VEL = false serves the
    // bodies whose velocity does not enter the force (no relativistic or non-gravitational
    // term): rv is then not read.  NG = false leaves the non-gravitational term to the caller.
    // Callers that evaluate several bodies compute their reciprocal square roots together
    // (independent chains) before summing the terms in the reference's order.
    template <bool VEL = true, bool NG = true>
    __device__ __forceinline__ int body_terms(const ForceEntry& fe, bool exact, const double rp[3],
                                              const double rv[3], double r2, double ir,
                                              double& acc0, double& acc1, double& acc2) {
        const double r = r2 * ir;
        const double ir3 = ir * ir * ir;
        // exact evaluations only: impacts and the closest approach to a non-Sun body (as
        // selects, not branches: the flag differs between the lanes of a warp)
        if (exact && r <= fe.radius) {
            impact_id = fe.naif_id;
            return ST_IMPACT;
        }
        const bool closer = exact && fe.kind != FK_SUN && r < min_dist;
        min_dist = closer ? r : min_dist;
        min_id = closer ? fe.naif_id : min_id;
        const double mass = fe.mass;
        const double kk = mass * ir3;
        acc0 -= rp[0] * kk;
        acc1 -= rp[1] * kk;
        acc2 -= rp[2] * kk;
        if (VEL && (fe.kind == FK_SUN || fe.kind == FK_JUPITER)) {
            // apply_gr_correction (gravity.rs:239-253)
            const double r_v = 4.0 * (rp[0] * rv[0] + rp[1] * rv[1] + rp[2] * rv[2]);
            const double rel_v2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
            const double gr_const = mass * C_AU_PER_DAY_INV_SQUARED * ir3;
            const double c = 4. * mass * ir - rel_v2;
            acc0 += gr_const * (c * rp[0] + r_v * rv[0]);
            acc1 += gr_const * (c * rp[1] + r_v * rv[1]);
            acc2 += gr_const * (c * rp[2] + r_v * rv[2]);
            // J2 in the ecliptic frame (gravity.rs:188-211, 223-235)
            const double rc = c_tab.rot_c, rs = c_tab.rot_s;
            const double ez = -rs * rp[1] + rc * rp[2];
            const double zr = ez * ir;
            const double z_squared = 5.0 * (zr * zr);
            const double rr = fe.radius * ir;
            const double coef =
                1.5 * (fe.kind == FK_JUPITER ? JUPITER_J2 : SUN_J2) * mass * (rr * rr) * ir3;
            const double ey = rc * rp[1] + rs * rp[2];
            const double jx = rp[0] * coef * (z_squared - 1.0);
            const double jy = ey * coef * (z_squared - 1.0);
            const double jz = ez * coef * (z_squared - 3.0);
            acc0 += jx;
            acc1 += rc * jy - rs * jz;
            acc2 += rs * jy + rc * jz;
            if (NG && fe.kind == FK_SUN && ng.kind != 0) {
                const double3 prel = make_double3(rp[0], rp[1], rp[2]);
                const double3 vrel = make_double3(rv[0], rv[1], rv[2]);
                const double3 na = (NGI && ng.kind == 1 && ng.p(9) == 0.0)
                                       ? nongrav_terms<false>(ng, prel, vrel)
                                       : nongrav_accel(ng, prel, vrel);
                acc0 += na.x;
                acc1 += na.y;
                acc2 += na.z;
            }
        } else if (fe.kind == FK_EARTH) {
            const double zr = rp[2] * ir;
            const double z_squared = 5.0 * (zr * zr);
            const double rr = fe.radius * ir;
            const double coef = 1.5 * EARTH_J2 * mass * (rr * rr) * ir3;
            acc0 += rp[0] * coef * (z_squared - 1.0);
            acc1 += rp[1] * coef * (z_squared - 1.0);
            acc2 += rp[2] * coef * (z_squared - 3.0);
        }
        return ST_OK;
    }

    // body_terms for the body at bp (velocity bv) seen from (x, v).  Distances use one
    // reciprocal square root per body: r = r2 * rsqrt(r2) and r^-3 = rsqrt(r2)^3 replace the
    // reference's sqrt and 1/(r*r*r) (a few ulp apart).
    template <bool VEL = true, bool NG = true>
    __device__ __forceinline__ int body(const ForceEntry& fe, bool exact, const double x[3],
                                        const double v[3], const double bp[3], const double bv[3],
                                        double& acc0, double& acc1, double& acc2) {
        const double rp[3] = {x[0] - bp[0], x[1] - bp[1], x[2] - bp[2]};
        double rv[3] = {0.0, 0.0, 0.0};
        if (VEL) {
            rv[0] = v[0] - bv[0];
            rv[1] = v[1] - bv[1];
            rv[2] = v[2] - bv[2];
        }
        const double r2 = rp[0] * rp[0] + rp[1] * rp[1] + rp[2] * rp[2];
        return body_terms<VEL, NG>(fe, exact, rp, rv, r2, rsqrt(r2), acc0, acc1, acc2);
    }

    // Fast path: the host-verified window where every body's first segment covers t and all
    // records have FAST_NC coefficients.  The Sun and Jupiter, whose velocities enter the
    // force, are evaluated first, two records at a time with velocities; the other bodies
    // (and the Earth-Moon barycentre they are chained through) follow in the reference's
    // order, three records at a time, positions only.  The accelerations are therefore
    // summed Sun, Jupiter, Mercury, Venus, Earth, Moon, Mars, Saturn, Uranus, Neptune.
    __device__ __forceinline__ int eval_fast(const FastPlan& P, bool exact, double t,
                                             const double x[3], const double v[3], double out[3]) {
        const double jds = __dmul_rn(t - 2451545.0, 86400.0);
        const double* pool = c_eph.pool;
        double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
        const int n_vel = P.n_vel;
#pragma unroll 1
        for (int it = 0; it < n_vel; it += 2) {
            const bool has_b = it + 1 < n_vel;
            const FastItem& A = P.item[it];
            const FastItem& B = P.item[has_b ? it + 1 : it];
            const double* ra = fast_record(pool, A, jds);
            const double* rb = fast_record(pool, B, jds);
            double pa[3], va[3], pb[3], vb[3];
            cheb_pair<FAST_NC, KU>(ra, rb, jds, pa, va, pb, vb);
            {
                const ForceEntry fe{A.mass, A.radius, 0, A.kind, A.naif_id, 0};
                const int rc = body<true>(fe, exact, x, v, pa, va, acc0, acc1, acc2);
                if (rc != ST_OK) return rc;
            }
            if (has_b) {
                const ForceEntry fe{B.mass, B.radius, 0, B.kind, B.naif_id, 0};
                const int rc = body<true>(fe, exact, x, v, pb, vb, acc0, acc1, acc2);
                if (rc != ST_OK) return rc;
            }
        }
        double cp[3] = {0.0, 0.0, 0.0};
        const double zero[3] = {0.0, 0.0, 0.0};
        const int n_items = P.n_items;
#pragma unroll 1
        for (int it = n_vel; it < n_items; it += 3) {
            const double* r0 = fast_record(pool, P.item[it], jds);
            const double* r1 = fast_record(pool, P.item[it + 1], jds);
            const double* r2 = fast_record(pool, P.item[it + 2], jds);
            double p3[3][3];
            cheb_pos3<FAST_NC, KU>(r0, r1, r2, jds, p3[0], p3[1], p3[2]);
#pragma unroll
            for (int h = 0; h < 3; ++h) {
                const FastItem& I = P.item[it + h];
                double* bp = p3[h];
                if (I.role == -2) continue;  // padding
                if (I.role < 0) {            // a centre kept for the bodies after it
                    cp[0] = bp[0]; cp[1] = bp[1]; cp[2] = bp[2];
                    continue;
                }
                if (I.chained) {
                    bp[0] += cp[0]; bp[1] += cp[1]; bp[2] += cp[2];
                }
                const ForceEntry fe{I.mass, I.radius, 0, I.kind, I.naif_id, 0};
                const int rc = body<false>(fe, exact, x, v, bp, zero, acc0, acc1, acc2);
                if (rc != ST_OK) return rc;
            }
        }
        out[0] = acc0;
        out[1] = acc1;
        out[2] = acc2;
        return ST_OK;
    }

    // eval_fast in two halves, for callers that evaluate the force at the same time more than
    // once (the corrector iterations of one Radau step share their node times):
    // fast_positions writes the bodies' positions at t (and the Sun's and Jupiter's
    // velocities) to cache[k * stride], k = 0 .. cached_doubles(P) - 1; fast_forces sums the
    // accelerations from them in eval_fast's order.
    __device__ __forceinline__ static int cached_doubles(const FastPlan& P) {
        return fast_plan_cache_doubles(P);
    }

    __device__ __forceinline__ static void fast_positions(const FastPlan& P, double t,
                                                          double* cache, int stride) {
        const double jds = __dmul_rn(t - 2451545.0, 86400.0);
        const double* pool = c_eph.pool;
        const int n_vel = P.n_vel;
        int k = 0;
#pragma unroll 1
        for (int it = 0; it < n_vel; it += 2) {
            const bool has_b = it + 1 < n_vel;
            const double* ra = fast_record(pool, P.item[it], jds);
            const double* rb = fast_record(pool, P.item[has_b ? it + 1 : it], jds);
            double pa[3], va[3], pb[3], vb[3];
            cheb_pair<FAST_NC, KU>(ra, rb, jds, pa, va, pb, vb);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                cache[(k + c) * stride] = pa[c];
                cache[(k + 3 + c) * stride] = va[c];
            }
            k += 6;
            if (has_b) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    cache[(k + c) * stride] = pb[c];
                    cache[(k + 3 + c) * stride] = vb[c];
                }
                k += 6;
            }
        }
        double cp[3] = {0.0, 0.0, 0.0};
        const int n_items = P.n_items;
#pragma unroll 1
        for (int it = n_vel; it < n_items; it += 3) {
            const double* r0 = fast_record(pool, P.item[it], jds);
            const double* r1 = fast_record(pool, P.item[it + 1], jds);
            const double* r2 = fast_record(pool, P.item[it + 2], jds);
            double p3[3][3];
            cheb_pos3<FAST_NC, KU>(r0, r1, r2, jds, p3[0], p3[1], p3[2]);
#pragma unroll
            for (int h = 0; h < 3; ++h) {
                const FastItem& I = P.item[it + h];
                double* bp = p3[h];
                if (I.role == -2) continue;
                if (I.role < 0) {
                    cp[0] = bp[0]; cp[1] = bp[1]; cp[2] = bp[2];
                    continue;
                }
                if (I.chained) {
                    bp[0] += cp[0]; bp[1] += cp[1]; bp[2] += cp[2];
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) cache[(k + c) * stride] = bp[c];
                k += 3;
            }
        }
    }

    __device__ __forceinline__ int fast_forces(const FastPlan& P, bool exact, const double x[3],
                                               const double v[3], const double* cache, int stride,
                                               double out[3]) {
        double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
        const int n_vel = P.n_vel;
        int k = 0;
#pragma unroll 1
        for (int it = 0; it < n_vel; ++it, k += 6) {
            const FastItem& A = P.item[it];
            const double bp[3] = {cache[k * stride], cache[(k + 1) * stride], cache[(k + 2) * stride]};
            const double bv[3] = {cache[(k + 3) * stride], cache[(k + 4) * stride],
                                  cache[(k + 5) * stride]};
            const ForceEntry fe{A.mass, A.radius, 0, A.kind, A.naif_id, 0};
            const int rc = body<true>(fe, exact, x, v, bp, bv, acc0, acc1, acc2);
            if (rc != ST_OK) return rc;
        }
        const double zero[3] = {0.0, 0.0, 0.0};
        const int n_items = P.n_items;
#pragma unroll 1
        for (int it = n_vel; it < n_items; ++it) {
            const FastItem& I = P.item[it];
            if (I.role < 0) continue;
            const double bp[3] = {cache[k * stride], cache[(k + 1) * stride], cache[(k + 2) * stride]};
            k += 3;
            const ForceEntry fe{I.mass, I.radius, 0, I.kind, I.naif_id, 0};
            const int rc = body<false>(fe, exact, x, v, bp, zero, acc0, acc1, acc2);
            if (rc != ST_OK) return rc;
        }
        out[0] = acc0;
        out[1] = acc1;
        out[2] = acc2;
        return ST_OK;
    }

    // `exact` marks the evaluations at the integrator's accepted states: only those check
    // for impacts (r <= body radius, acceleration.rs:147-158) and update the closest-approach
    // record.  The flag is a runtime value so one copy of the force code serves every call
    // site.  Distances use one reciprocal square root per body: r = r2 * rsqrt(r2) and
    // r^-3 = rsqrt(r2)^3 replace the reference's sqrt and 1/(r*r*r) (a few ulp apart).
    __device__ __forceinline__ int eval(bool exact, double t, const double x[3], const double v[3],
                                        double out[3]) {
        const FastPlan& P = n_force == c_eph.n_force_planets ? c_eph.fast_planets : c_eph.fast_all;
        if (P.ok && t >= P.lo && t <= P.hi) return eval_fast(P, exact, t, x, v, out);
        double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
        int cache_slot = -1;
        double cp[3] = {0.0, 0.0, 0.0}, cv[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
        for (int b = 0; b < n_force; ++b) {
            const ForceEntry fe = c_eph.force[b];
            const int slot = fe.slot;
            double bp[3], bv[3];
            if (eph_raw(c_eph, slot, t, bp, bv) != ST_OK) return ST_DAF_LIMITS;
            const int parent = c_eph.slot[slot].parent_slot;
            if (parent >= 0) {
                if (parent != cache_slot) {
                    if (eph_raw(c_eph, parent, t, cp, cv) != ST_OK) return ST_DAF_LIMITS;
                    cache_slot = parent;
                }
                bp[0] += cp[0]; bp[1] += cp[1]; bp[2] += cp[2];
                bv[0] += cv[0]; bv[1] += cv[1]; bv[2] += cv[2];
            }
            const int rc = body(fe, exact, x, v, bp, bv, acc0, acc1, acc2);
            if (rc != ST_OK) return rc;
        }
        out[0] = acc0;
        out[1] = acc1;
        out[2] = acc2;
        return ST_OK;
    }
};

// lane-parallel kernels: compact loops; a translation unit that defines KB_FORCE_NG_INLINE
// before including this header (the differentiation kernels) gets the inline comet model
#ifdef KB_FORCE_NG_INLINE
using SpkForce = SpkForceT<1, true>;
#else
using SpkForce = SpkForceT<1>;
#endif
using SpkForceUnrolled = SpkForceT<FAST_NC>;  // one object per thread

// central_accel (acceleration.rs:66-80): the Sun at the origin only.
struct CentralForce {
    int32_t impact_id;
    double min_dist;
    int32_t min_id;
    __device__ __forceinline__ int eval(bool, double, const double x[3], const double[3],
                                        double out[3]) {
        const double k = powi<-3>(norm3(x[0], x[1], x[2]));
        out[0] = -x[0] * k * GMS;
        out[1] = -x[1] * k * GMS;
        out[2] = -x[2] * k * GMS;
        return ST_OK;
    }
};

}  // namespace kb
