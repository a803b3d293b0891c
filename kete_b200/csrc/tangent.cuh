// tangent.cuh -- forward sensitivities (state-transition matrix) of the N-body propagation.
//
// The force of every perturber (GravParams::add_acceleration, gravity.rs:171-216, and the
// JPL comet non-gravitational term, nongrav.rs:131-155) is evaluated with dual numbers
// carrying the partial derivatives with respect to the object's position and velocity, so
// the 3x6 Jacobian of the acceleration comes out of the same arithmetic as the value.  The
// Radau corrector iterations (radau.rs:231-344) are then differentiated exactly as they are
// executed: every predictor, divided difference and b update has a tangent counterpart for
// each of the 8 directions (initial position, initial velocity, A1, A2), with the step
// sizes held fixed.  Columns 6 and 7 differentiate with respect to A1 and A2 of the JPL
// comet model (dt = 0).
#pragma once
#include "common.cuh"
#include "forces.cuh"

namespace kb {

constexpr int TAN_DIRS = 8;  // d/dx0 (3), d/dv0 (3), d/dA1, d/dA2

struct D6 {
    double v;
    double d[6];
};

__device__ __forceinline__ D6 dconst(double v) {
    D6 r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.d[i] = 0.0;
    return r;
}
__device__ __forceinline__ D6 operator+(const D6& a, const D6& b) {
    D6 r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
__device__ __forceinline__ D6 operator-(const D6& a, const D6& b) {
    D6 r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
__device__ __forceinline__ D6 operator-(const D6& a) {
    D6 r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.d[i] = -a.d[i];
    return r;
}
__device__ __forceinline__ D6 operator*(const D6& a, const D6& b) {
    D6 r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
__device__ __forceinline__ D6 operator*(const D6& a, double s) {
    D6 r;
    r.v = a.v * s;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] * s;
    return r;
}
__device__ __forceinline__ D6 operator*(double s, const D6& a) { return a * s; }
__device__ __forceinline__ D6 operator+(const D6& a, double s) {
    D6 r = a;
    r.v += s;
    return r;
}
__device__ __forceinline__ D6 operator-(double s, const D6& a) {
    D6 r = -a;
    r.v += s;
    return r;
}
__device__ __forceinline__ D6 drecip(const D6& a) {
    const double iv = 1.0 / a.v;
    D6 r;
    r.v = iv;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.d[i] = -a.d[i] * iv * iv;
    return r;
}
__device__ __forceinline__ D6 operator/(const D6& a, const D6& b) { return a * drecip(b); }
__device__ __forceinline__ D6 drsqrt(const D6& a) {
    const double ir = rsqrt(a.v);
    const double k = -0.5 * ir * ir * ir;
    D6 r;
    r.v = ir;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] * k;
    return r;
}
__device__ __forceinline__ D6 dpow(const D6& a, double e) {
    const double pv = pow(a.v, e);
    const double k = e * pow(a.v, e - 1.0);
    D6 r;
    r.v = pv;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.d[i] = a.d[i] * k;
    return r;
}
__device__ __forceinline__ D6 ddot(const D6 a[3], const D6 b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Non-gravitational JPL comet term in dual arithmetic; dpar receives d(accel)/dA1 and
// d(accel)/dA2 (the unit directions scaled by g(r)).
__device__ __forceinline__ void nongrav_dual(const NonGrav& ng, const D6 rp[3], const D6 rv[3],
                                             D6 acc[3], double dpar[3][2]) {
    if (ng.kind == 2) {  // dust: beta is not a differentiated parameter
        const double beta = ng.p(1);
        const D6 n2 = ddot(rp, rp);
        const D6 inv = drsqrt(n2);
        D6 pn[3] = {rp[0] * inv, rp[1] * inv, rp[2] * inv};
        const D6 r_dot = ddot(pn, rv);
        const D6 scaling = drecip(n2) * (GMS * beta);
#pragma unroll
        for (int i = 0; i < 3; ++i)
            acc[i] = acc[i] + scaling * ((1.0 - r_dot * C_AU_PER_DAY_INV_SQUARED) * pn[i] -
                                         rv[i] * C_AU_PER_DAY_INV_SQUARED);
        return;
    }
    const double a1 = ng.p(1), a2 = ng.p(2), a3 = ng.p(3), alpha = ng.p(4), r_0 = ng.p(5);
    const double m = ng.p(6), nn = ng.p(7), k = ng.p(8);
    const D6 inv = drsqrt(ddot(rp, rp));
    const D6 r = drecip(inv);
    D6 pn[3] = {rp[0] * inv, rp[1] * inv, rp[2] * inv};
    const D6 vdp = ddot(rv, pn);
    D6 tv[3] = {rv[0] - pn[0] * vdp, rv[1] - pn[1] * vdp, rv[2] - pn[2] * vdp};
    const D6 tinv = drsqrt(ddot(tv, tv));
    D6 t_vec[3] = {tv[0] * tinv, tv[1] * tinv, tv[2] * tinv};
    D6 nv[3] = {t_vec[1] * pn[2] - t_vec[2] * pn[1], t_vec[2] * pn[0] - t_vec[0] * pn[2],
                t_vec[0] * pn[1] - t_vec[1] * pn[0]};
    const D6 ninv = drsqrt(ddot(nv, nv));
    D6 n_vec[3] = {nv[0] * ninv, nv[1] * ninv, nv[2] * ninv};
    const D6 rr0 = r * (1.0 / r_0);
    // g(r) = alpha (r/r0)^-m (1 + (r/r0)^n)^-k
    const D6 gfac = dpow(rr0, -m) * dpow(dpow(rr0, nn) + 1.0, -k) * alpha;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        acc[i] = acc[i] + pn[i] * gfac * a1 + t_vec[i] * gfac * a2 + n_vec[i] * gfac * a3;
        dpar[i][0] = pn[i].v * gfac.v;
        dpar[i][1] = t_vec[i].v * gfac.v;
    }
}

// One perturber's acceleration and its Jacobian.  bp/bv: perturber state (constants).
__device__ __forceinline__ void body_dual(const ForceEntry& fe, const NonGrav& ng, const double x[3],
                                          const double v[3], const double bp[3], const double bv[3],
                                          D6 acc[3], double dpar[3][2]) {
    D6 rp[3], rv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        rp[i] = dconst(x[i] - bp[i]);
        rp[i].d[i] = 1.0;
        rv[i] = dconst(v[i] - bv[i]);
        rv[i].d[3 + i] = 1.0;
    }
    const D6 r2 = ddot(rp, rp);
    const D6 ir = drsqrt(r2);
    const D6 ir3 = ir * ir * ir;
    const double mass = fe.mass;
    const D6 kk = ir3 * mass;
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[i] = acc[i] - rp[i] * kk;
    if (fe.kind == FK_SUN || fe.kind == FK_JUPITER) {
        const D6 r_v = ddot(rp, rv) * 4.0;
        const D6 rel_v2 = ddot(rv, rv);
        const D6 gr_const = ir3 * (mass * C_AU_PER_DAY_INV_SQUARED);
        const D6 c = ir * (4. * mass) - rel_v2;
#pragma unroll
        for (int i = 0; i < 3; ++i) acc[i] = acc[i] + gr_const * (c * rp[i] + r_v * rv[i]);
        const double rc = c_tab.rot_c, rs = c_tab.rot_s;
        const D6 ez = rs * (-rp[1]) + rp[2] * rc;
        const D6 ey = rp[1] * rc + rp[2] * rs;
        const D6 zr = ez * ir;
        const D6 z_squared = zr * zr * 5.0;
        const D6 rr = ir * fe.radius;
        const D6 coef = rr * rr * ir3 * (1.5 * (fe.kind == FK_JUPITER ? JUPITER_J2 : SUN_J2) * mass);
        const D6 jx = rp[0] * coef * (z_squared + (-1.0));
        const D6 jy = ey * coef * (z_squared + (-1.0));
        const D6 jz = ez * coef * (z_squared + (-3.0));
        acc[0] = acc[0] + jx;
        acc[1] = acc[1] + jy * rc - jz * rs;
        acc[2] = acc[2] + jy * rs + jz * rc;
        if (fe.kind == FK_SUN && ng.kind != 0) nongrav_dual(ng, rp, rv, acc, dpar);
    } else if (fe.kind == FK_EARTH) {
        const D6 zr = rp[2] * ir;
        const D6 z_squared = zr * zr * 5.0;
        const D6 rr = ir * fe.radius;
        const D6 coef = rr * rr * ir3 * (1.5 * EARTH_J2 * mass);
        acc[0] = acc[0] + rp[0] * coef * (z_squared + (-1.0));
        acc[1] = acc[1] + rp[1] * coef * (z_squared + (-1.0));
        acc[2] = acc[2] + rp[2] * coef * (z_squared + (-3.0));
    }
}

// Acceleration (out), its Jacobian J (3 x 6: d/dx, d/dv) and the parameter columns
// jp (3 x 2: d/dA1, d/dA2).  Impacts are checked on exact evaluations as in SpkForce.
struct TangentForce {
    int n_force;
    NonGrav ng;
    int32_t impact_id;
    double min_dist;

    __device__ int eval(bool exact, double t, const double x[3], const double v[3], double out[3],
                        double J[3][6], double jp[3][2]) {
        D6 acc[3] = {dconst(0.0), dconst(0.0), dconst(0.0)};
        double dpar[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        int cache_slot = -1;
        double cp[3] = {0.0, 0.0, 0.0}, cv[3] = {0.0, 0.0, 0.0};
        for (int b = 0; b < n_force; ++b) {
            const ForceEntry fe = c_eph.force[b];
            double bp[3], bv[3];
            if (eph_raw(c_eph, fe.slot, t, bp, bv) != ST_OK) return ST_DAF_LIMITS;
            const int parent = c_eph.slot[fe.slot].parent_slot;
            if (parent >= 0) {
                if (parent != cache_slot) {
                    if (eph_raw(c_eph, parent, t, cp, cv) != ST_OK) return ST_DAF_LIMITS;
                    cache_slot = parent;
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    bp[i] += cp[i];
                    bv[i] += cv[i];
                }
            }
            if (exact) {
                const double r = norm3(x[0] - bp[0], x[1] - bp[1], x[2] - bp[2]);
                if (r <= fe.radius) {
                    impact_id = fe.naif_id;
                    return ST_IMPACT;
                }
                if (fe.kind != FK_SUN && r < min_dist) min_dist = r;
            }
            body_dual(fe, ng, x, v, bp, bv, acc, dpar);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            out[i] = acc[i].v;
#pragma unroll
            for (int j = 0; j < 6; ++j) J[i][j] = acc[i].d[j];
            jp[i][0] = dpar[i][0];
            jp[i][1] = dpar[i][1];
        }
        return ST_OK;
    }

    // The same (exact = false) from the fast plan's body positions in the lane's cache,
    // evaluated at t if the cache holds another time: the bodies are summed in the fast
    // plan's order (Sun, Jupiter, then the reference's order), a rounding-level change.
    __device__ int eval_cached(const FastPlan& P, EphCache& C, double t, const double x[3],
                               const double v[3], double out[3], double J[3][6],
                               double jp[3][2]) {
        if (t != C.t) {
            SpkForce::fast_positions(P, t, C.p, C.stride);
            C.t = t;
        }
        D6 acc[3] = {dconst(0.0), dconst(0.0), dconst(0.0)};
        double dpar[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        const double zero[3] = {0.0, 0.0, 0.0};
        const int s = C.stride;
        int k = 0;
        for (int it = 0; it < P.n_items; ++it) {
            const FastItem& I = P.item[it];
            if (it >= P.n_vel && I.role < 0) continue;
            const double bp[3] = {C.p[k * s], C.p[(k + 1) * s], C.p[(k + 2) * s]};
            double bv[3] = {0.0, 0.0, 0.0};
            if (it < P.n_vel) {
                bv[0] = C.p[(k + 3) * s];
                bv[1] = C.p[(k + 4) * s];
                bv[2] = C.p[(k + 5) * s];
                k += 6;
            } else {
                k += 3;
            }
            const ForceEntry fe{I.mass, I.radius, 0, I.kind, I.naif_id, 0};
            body_dual(fe, ng, x, v, bp, it < P.n_vel ? bv : zero, acc, dpar);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            out[i] = acc[i].v;
#pragma unroll
            for (int j = 0; j < 6; ++j) J[i][j] = acc[i].d[j];
            jp[i][0] = dpar[i][0];
            jp[i][1] = dpar[i][1];
        }
        return ST_OK;
    }
};

}  // namespace kb
