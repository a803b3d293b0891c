/*
 * kete_oracle.c -- CPU restatement of kete_core's FP64 hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the correctness oracle and the timed CPU baseline.
 * The kete_b200 product never links, loads or calls this file.
 *
 * Each function follows the reference source in operation order; citations are
 * "kete_core/<file>:<lines>" relative to src/kete_core/src/ of the kete repository and
 * "py/<file>:<lines>" relative to src/kete/rust/.  Rust's f64 methods call the platform
 * libm (glibc), as this file does; LLVM's powi expansion with constant exponents is
 * reproduced by ko_powi.  Build with -ffp-contract=off (no fused multiply-add).
 */
#include "kete_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------------------------
 * constants: kete_core/constants/gravity.rs:9-153, kete_core/constants/universal.rs:2-36
 * ---------------------------------------------------------------------------------------- */
#define GMS 0.00029591220828411956
#define GMS_SQRT 0.01720209894996
#define SUN_J2 2.2e-7
#define EARTH_J2 0.00108262998905
#define JUPITER_J2 0.014696572
#define C_AU_PER_DAY 173.14463267424034
#define C_AU_PER_DAY_INV 0.005775518331436995
#define C_AU_PER_DAY_INV_SQUARED 3.33566119967647e-05
#define AU_KM 149597870.7
#define SUN_TEMP 5778.0
#define SUN_DIAMETER 1.3914e6
#define SOLAR_FLUX 1360.8
#define STEFAN_BOLTZMANN 5.670374419e-8
#define GOLDEN_RATIO 1.618033988749894
#define V_MAG_ZERO 3597.28
#define C_V 1329.0
#define OBLIQUITY 0.40909280422232897 /* kete_core/frames/definitions.rs:135 */
#define TAU 6.283185307179586
#define PI 3.141592653589793

typedef struct {
    int64_t naif_id;
    double mass;
    double radius;
} grav_params;

/* MASSES (kete_core/constants/gravity.rs:43-134); PLANETS is the first 10 entries
 * (gravity.rs:145-148). */
static const grav_params MASSES[15] = {
    {10, GMS, 0.004654758765894654},
    {1, 1.66012082548908e-07 * GMS, 1.63139354095098e-05},
    {2, 2.44783828779694e-06 * GMS, 4.04537843465442e-05},
    {399, 3.00348961546514e-06 * GMS, 4.33036684926559e-05},
    {301, 3.69430335010988e-08 * GMS, 1.16138016662292e-05},
    {4, 3.22715608291416e-07 * GMS, 2.27021279387769e-05},
    {5, 0.0009547919099414246 * GMS, 0.00047789450254521576},
    {6, 0.00028588567002459455 * GMS, 0.0004028666966848747},
    {7, 4.36624961322212e-05 * GMS, 0.0001708513622580592},
    {8, 5.15138377265457e-05 * GMS, 0.0001655371154958558},
    {20000001, 4.7191659919436e-10 * GMS, 6.276827e-6},
    {20000002, 1.0259143964958e-10 * GMS, 3.415824e-6},
    {20000004, 1.3026452498655e-10 * GMS, 3.512082e-6},
    {20000010, 4.3953391300849e-11 * GMS, 2.894426e-6},
    {20000704, 1.911e-11 * GMS, 2.219283e-6},
};

/* LLVM's constant-exponent powi expansion (repeated squaring, reciprocal for n < 0),
 * which is what f64::powi compiles to for the literal exponents kete uses. */
static double ko_powi(double x, int n) {
    unsigned v = (unsigned)(n < 0 ? -n : n);
    double res = 1.0;
    int have = 0;
    double sq = x;
    while (v) {
        if (v & 1u) {
            if (have)
                res = res * sq;
            else {
                res = sq;
                have = 1;
            }
        }
        v >>= 1;
        if (v) sq = sq * sq;
    }
    if (!have) res = 1.0;
    if (n < 0) res = 1.0 / res;
    return res;
}

static inline double norm3(const double v[3]) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
static inline double dot3(const double a[3], const double b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline double rem_euclid(double a, double b) {
    double r = fmod(a, b);
    return r < 0.0 ? r + fabs(b) : r;
}
/* f64::max / nalgebra max(): NaN-ignoring */
static inline double fmax3(const double v[3]) { return fmax(fmax(v[0], v[1]), v[2]); }
/* f64::clamp keeps NaN */
static inline double clampd(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

/* ------------------------------------------------------------------------------------------
 * frames: ecliptic <-> equatorial by the fixed obliquity (kete_core/frames/definitions.rs:
 * 135,154-158,224-237).  Rotation3::from_axis_angle about x gives [[1,0,0],[0,c,-s],[0,s,c]].
 * ---------------------------------------------------------------------------------------- */
static double ROT_C, ROT_S;
static int rot_init_done = 0;
static void rot_init(void) {
    if (!rot_init_done) {
        ROT_S = sin(OBLIQUITY);
        ROT_C = cos(OBLIQUITY);
        rot_init_done = 1;
    }
}
static void ecl_to_eq(const double v[3], double o[3]) {
    rot_init();
    double y = ROT_C * v[1] + -ROT_S * v[2];
    double z = ROT_S * v[1] + ROT_C * v[2];
    o[0] = v[0];
    o[1] = y;
    o[2] = z;
}
static void eq_to_ecl(const double v[3], double o[3]) {
    rot_init();
    double y = ROT_C * v[1] + ROT_S * v[2];
    double z = -ROT_S * v[1] + ROT_C * v[2];
    o[0] = v[0];
    o[1] = y;
    o[2] = z;
}

/* ------------------------------------------------------------------------------------------
 * newton_raphson (kete_core/fitting/newton.rs:18-65)
 * ---------------------------------------------------------------------------------------- */
typedef double (*scalar_fn)(double, const void *);

static int newton_raphson(scalar_fn func, scalar_fn der, const void *ctx, double start,
                          double atol, double *out) {
    double x = start;
    if (fabs(der(x, ctx)) < 1e-12) x += 0.1;
    double f_eval, d_eval;
    for (int it = 0; it < 100; ++it) {
        f_eval = func(x, ctx);
        if (fabs(f_eval) < atol) {
            *out = x;
            return KO_OK;
        }
        d_eval = der(x, ctx);
        if (fabs(d_eval) < 1e-12) return KO_CONVERGENCE;
        if (!isfinite(d_eval) || !isfinite(f_eval)) return KO_CONVERGENCE;
        x -= 0.5 * f_eval / d_eval;
        d_eval = der(x, ctx);
        if (fabs(d_eval) < 1e-3) f_eval = func(x, ctx);
        x -= 0.5 * f_eval / d_eval;
    }
    return KO_CONVERGENCE;
}

static double nt_f(double x, const void *c) { (void)c; return 1.0 * x * x - 1.0; }
static double nt_d(double x, const void *c) { (void)c; return 2.0 * x; }
int ko_newton_test(double start, double atol, double *root) {
    return newton_raphson(nt_f, nt_d, NULL, start, atol, root);
}

/* ------------------------------------------------------------------------------------------
 * universal Kepler solver (kete_core/propagation/kepler.rs:119-297)
 * ---------------------------------------------------------------------------------------- */
#define PARABOLIC_BETA 1e-10
#define PARABOLIC_ECC_LIMIT 1e-3

static double g_1(double s, double beta) {
    if (fabs(beta) < PARABOLIC_BETA) return s;
    double beta_sqrt = sqrt(fabs(beta));
    if (beta >= 0.0) return sin(beta_sqrt * s) / beta_sqrt;
    return sinh(beta_sqrt * s) / beta_sqrt;
}

static double g_2(double s, double beta) {
    if (fabs(beta) < PARABOLIC_BETA) return ko_powi(s, 2) / 2.0;
    double beta_sqrt = sqrt(fabs(beta)) * s;
    if (beta >= 0.0) return 2.0 * pow(sin(beta_sqrt / 2.0), 2.0) / beta;
    return (1.0 - cosh(beta_sqrt)) / beta;
}

typedef struct {
    double r0, rv0, beta, b_sqrt, dt;
} kep_ctx;

static double kep_f_ell(double x, const void *p) {
    const kep_ctx *c = (const kep_ctx *)p;
    double g1 = sin(c->b_sqrt * x) / c->b_sqrt;
    double g2 = 2.0 * pow(sin(c->b_sqrt * x / 2.0), 2.0) / c->beta;
    double g3 = (x - g1) / c->beta;
    return c->r0 * g1 + c->rv0 * g2 + GMS * g3 - c->dt;
}
static double kep_d_ell(double x, const void *p) {
    const kep_ctx *c = (const kep_ctx *)p;
    double g2d = sin(c->b_sqrt * x), g1d = cos(c->b_sqrt * x);
    double g3d = (1.0 - g1d) / c->beta;
    return c->r0 * g1d + c->rv0 * g2d + GMS * g3d;
}
static double kep_f_hyp(double x, const void *p) {
    const kep_ctx *c = (const kep_ctx *)p;
    double g1 = sinh(c->b_sqrt * x) / c->b_sqrt;
    double g2 = (1.0 - cosh(c->b_sqrt * x)) / c->beta;
    double g3 = (x - g1) / c->beta;
    return c->r0 * g1 + c->rv0 * g2 + GMS * g3 - c->dt;
}
static double kep_d_hyp(double x, const void *p) {
    const kep_ctx *c = (const kep_ctx *)p;
    double g2d = sinh(c->b_sqrt * x), g1d = cosh(c->b_sqrt * x);
    double g3d = (1.0 - g1d) / c->beta;
    return c->r0 * g1d + c->rv0 * g2d + GMS * g3d;
}

static int solve_kepler_universal(double dt, double r0, double v0, double rv0, double *s_out,
                                  double *beta_out) {
    double beta = 2.0 * GMS / r0 - ko_powi(v0, 2);
    double b_sqrt = sqrt(fabs(beta));
    kep_ctx c = {r0, rv0, beta, b_sqrt, dt};
    int rc;
    double res = 0.0;
    if (beta >= PARABOLIC_BETA) {
        double period = GMS * ko_powi(b_sqrt, -3);
        c.dt = fmod(c.dt, period * TAU);
        double guess = (1.0 / b_sqrt) * c.dt / period;
        rc = newton_raphson(kep_f_ell, kep_d_ell, &c, guess, 1e-11, &res);
    } else if (fabs(beta) < PARABOLIC_BETA) {
        double a0 = -6.0 * dt / GMS;
        double a1 = 6.0 * r0 / GMS;
        double a2 = 3.0 * rv0 / GMS;
        double p = (3.0 * a1 - ko_powi(a2, 2)) / 3.0;
        double q = (9.0 * a1 * a2 - 27.0 * a0 - 2.0 * ko_powi(a2, 3)) / 27.0;
        double w = pow(q / 2.0 + sqrt(ko_powi(q, 2) / 4.0 + ko_powi(p, 3) / 27.0), 1.0 / 3.0);
        res = w - p / (3.0 * w) - a2 / 3.0;
        rc = KO_OK;
    } else {
        rc = newton_raphson(kep_f_hyp, kep_d_hyp, &c, GMS_SQRT * fabs(beta) * dt, 1e-11, &res);
    }
    if (rc != KO_OK) return KO_CONVERGENCE;
    *s_out = res;
    *beta_out = beta;
    return KO_OK;
}

static int analytic_2_body_d(double time, const double pos[3], const double vel[3], int depth,
                             double op[3], double ov[3]) {
    if (depth >= 10) return KO_CONVERGENCE;
    depth += 1;
    if (fabs(time) < 1e-10) {
        memcpy(op, pos, 3 * sizeof(double));
        memcpy(ov, vel, 3 * sizeof(double));
        return KO_OK;
    }
    double r0 = norm3(pos), v0 = norm3(vel), rv0 = dot3(pos, vel);
    if (isnan(rv0) || isinf(rv0)) return KO_CONVERGENCE;
    double s, beta;
    if (solve_kepler_universal(time, r0, v0, rv0, &s, &beta) == KO_OK) {
        double g1 = g_1(s, beta), g2 = g_2(s, beta);
        double f = 1.0 - GMS / r0 * g2;
        double g = r0 * g1 + rv0 * g2;
        double np[3];
        for (int i = 0; i < 3; ++i) np[i] = pos[i] * f + vel[i] * g;
        double nr0 = norm3(np);
        double f_dot = -GMS / (nr0 * r0) * g1;
        double g_dot = 1.0 - (GMS / nr0) * g2;
        for (int i = 0; i < 3; ++i) {
            op[i] = np[i];
            ov[i] = pos[i] * f_dot + vel[i] * g_dot;
        }
        return KO_OK;
    }
    double ip[3], iv[3];
    int rc = analytic_2_body_d(0.5 * time, pos, vel, depth, ip, iv);
    if (rc != KO_OK) return rc;
    return analytic_2_body_d(time * 0.5, ip, iv, depth, op, ov);
}

int ko_analytic_2_body(double time, const double pos[3], const double vel[3], double op[3],
                       double ov[3]) {
    return analytic_2_body_d(time, pos, vel, 0, op, ov);
}

/* compute_eccentric_anomaly (kete_core/propagation/kepler.rs:27-60) */
typedef struct {
    double ecc, m;
} ecc_ctx;
static double ea_f_ell(double e, const void *p) {
    const ecc_ctx *c = (const ecc_ctx *)p;
    return -c->ecc * sin(e) + e - rem_euclid(c->m, TAU);
}
static double ea_d_ell(double e, const void *p) {
    const ecc_ctx *c = (const ecc_ctx *)p;
    return 1.0 - 1.0 * c->ecc * cos(e);
}
static double ea_f_hyp(double e, const void *p) {
    const ecc_ctx *c = (const ecc_ctx *)p;
    return c->ecc * sinh(e) - e - c->m;
}
static double ea_d_hyp(double e, const void *p) {
    const ecc_ctx *c = (const ecc_ctx *)p;
    return -1.0 + c->ecc * cosh(e);
}
int ko_compute_eccentric_anomaly(double ecc, double mean_anom, double peri_dist, double *out) {
    if (!isfinite(ecc)) return KO_VALUE_ERROR;
    if (ecc < 0.0) return KO_VALUE_ERROR;
    if (ecc < 1e-6) {
        *out = mean_anom;
        return KO_OK;
    }
    ecc_ctx c = {ecc, mean_anom};
    if (ecc < 1.0 - PARABOLIC_ECC_LIMIT) {
        double r;
        int rc = newton_raphson(ea_f_ell, ea_d_ell, &c, rem_euclid(mean_anom, TAU), 1e-11, &r);
        if (rc) return rc;
        *out = rem_euclid(r, TAU);
        return KO_OK;
    }
    if (ecc < 1.0 + PARABOLIC_ECC_LIMIT) {
        double p = 2.0 * peri_dist, q = 6.0 * mean_anom;
        double w = cbrt(0.5 * (q + sqrt(ko_powi(q, 2) + 4.0 * ko_powi(p, 3))));
        *out = w - p / w;
        return KO_OK;
    }
    return newton_raphson(ea_f_hyp, ea_d_hyp, &c, asinh(mean_anom / ecc), 1e-11, out);
}

/* CometElements::to_pos_vel (kete_core/elements.rs:190-264) */
int ko_elements_to_pos_vel(double epoch, double ecc, double incl, double lon_asc,
                           double peri_time, double peri_arg, double peri_dist, double pos[3],
                           double vel[3]) {
    int elliptical = ecc < 1.0 - PARABOLIC_ECC_LIMIT;
    int hyperbolic = ecc > 1.0 + PARABOLIC_ECC_LIMIT;
    int parabolic = !elliptical && !hyperbolic;
    double semi_major = parabolic ? 0.0 : peri_dist / (1.0 - ecc);
    double mean_motion = parabolic ? GMS_SQRT : pow(fabs(semi_major), -1.5) * GMS_SQRT;
    double mean_anom = mean_motion * (epoch - peri_time);
    double ea;
    int rc = ko_compute_eccentric_anomaly(ecc, mean_anom, peri_dist, &ea);
    if (rc) return rc;
    double x, y, xd, yd;
    if (elliptical) {
        double se = sin(ea), ce = cos(ea);
        double e_dot = pow(semi_major, 1.5) * (1.0 - ecc * ce);
        double b = semi_major * sqrt(1.0 - ko_powi(ecc, 2));
        x = semi_major * (ce - ecc);
        y = b * se;
        xd = -semi_major / e_dot * se * GMS_SQRT;
        yd = b / e_dot * ce * GMS_SQRT;
    } else if (hyperbolic) {
        double sh = sinh(ea), ch = cosh(ea);
        double b = -semi_major * sqrt(ko_powi(ecc, 2) - 1.0);
        double h_dot = pow(fabs(semi_major), 1.5) * (1.0 - ecc * ch);
        x = semi_major * (ch - ecc);
        y = b * sh;
        xd = -semi_major / h_dot * sh * GMS_SQRT;
        yd = -b / h_dot * ch * GMS_SQRT;
    } else {
        double d_dot = peri_dist + ko_powi(ea, 2) / 2.0;
        x = peri_dist - ko_powi(ea, 2) / 2.0;
        y = sqrt(2.0 * peri_dist) * ea;
        xd = -ea / d_dot * GMS_SQRT;
        yd = sqrt(2.0 * peri_dist) / d_dot * GMS_SQRT;
    }
    double s_w = sin(peri_arg), c_w = cos(peri_arg);
    double s_o = sin(lon_asc), c_o = cos(lon_asc);
    double s_i = sin(incl), c_i = cos(incl);
    double px = c_w * c_o - s_w * s_o * c_i;
    double py = c_w * s_o + s_w * c_o * c_i;
    double pz = s_w * s_i;
    double qx = -s_w * c_o - c_w * s_o * c_i;
    double qy = -s_w * s_o + c_w * c_o * c_i;
    double qz = c_w * s_i;
    pos[0] = x * px + y * qx;
    pos[1] = x * py + y * qy;
    pos[2] = x * pz + y * qz;
    vel[0] = xd * px + yd * qx;
    vel[1] = xd * py + yd * qy;
    vel[2] = xd * pz + yd * qz;
    return KO_OK;
}

/* propagate_two_body with light delay, as the PyO3 binding does it
 * (py/kepler.rs:68-108; kete_core/propagation/kepler.rs:306-322).  States are already
 * Sun-centred here (the binding's change_center(10) is the caller's job). */
static int two_body_one(const double p[3], const double v[3], double jd0, double jd1,
                        const double *obs, double op[3], double ov[3], double *ojd) {
    int rc = analytic_2_body_d(jd1 - jd0, p, v, 0, op, ov);
    if (rc) return rc;
    *ojd = jd1;
    if (obs) {
        double d[3] = {op[0] - obs[0], op[1] - obs[1], op[2] - obs[2]};
        double delay = -norm3(d) / C_AU_PER_DAY;
        double p2[3], v2[3];
        double t2 = *ojd + delay;
        rc = analytic_2_body_d(t2 - *ojd, op, ov, 0, p2, v2);
        if (rc) return rc;
        memcpy(op, p2, sizeof p2);
        memcpy(ov, v2, sizeof v2);
        *ojd = t2;
    }
    return KO_OK;
}

static int g_threads = 0;
void ko_set_threads(int n) { g_threads = n; }

void ko_propagate_two_body_batch(int64_t n, const double *pos, const double *vel,
                                 const double *jd0, const double *jd1,
                                 const double *observer_pos, double *out_pos, double *out_vel,
                                 double *out_jd, int32_t *status, int n_threads) {
#pragma omp parallel for schedule(dynamic, 1000) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
    for (int64_t i = 0; i < n; ++i) {
        double p[3] = {pos[i], pos[n + i], pos[2 * n + i]};
        double v[3] = {vel[i], vel[n + i], vel[2 * n + i]};
        double op[3], ov[3], ojd;
        int rc = two_body_one(p, v, jd0[i], jd1[i], observer_pos, op, ov, &ojd);
        if (rc) {
            op[0] = op[1] = op[2] = ov[0] = ov[1] = ov[2] = NAN;
            ojd = jd1[i];
        }
        for (int c = 0; c < 3; ++c) {
            out_pos[c * n + i] = op[c];
            out_vel[c * n + i] = ov[c];
        }
        if (out_jd) out_jd[i] = ojd;
        status[i] = rc;
    }
}

/* ------------------------------------------------------------------------------------------
 * Gauss-Radau 15 (kete_core/propagation/radau.rs:24-346)
 * ---------------------------------------------------------------------------------------- */
static const double GR_SPACING[8] = {
    0.0, 0.05626256053692215, 0.18024069173689236, 0.3526247171131696,
    0.5471536263305554, 0.7342101772154105, 0.8853209468390958, 0.9775206135612875,
};
static double W_VEC[7], U_VEC[7], C_MAT[7][7];
static double W_POW[8][7], U_POW[8][7], FRAC2[8];
static int radau_init_done = 0;

static void radau_init(void) {
    if (radau_init_done) return;
    for (int i = 0; i < 7; ++i) {
        W_VEC[i] = 1.0 / (double)((i + 2) * (i + 3));
        U_VEC[i] = 1.0 / (double)(i + 2);
    }
    for (int i = 0; i < 7; ++i)
        for (int j = 0; j < 7; ++j) C_MAT[i][j] = (i == j) ? 1.0 : 0.0;
    for (int idx = 0; idx < 7; ++idx) {
        if (idx > 0) C_MAT[idx][0] = -GR_SPACING[idx] * C_MAT[idx - 1][0];
        for (int idy = 1; idy < idx; ++idy)
            C_MAT[idx][idy] = C_MAT[idx - 1][idy - 1] - GR_SPACING[idx] * C_MAT[idx - 1][idy];
    }
    for (int j = 1; j < 8; ++j) {
        double f = GR_SPACING[j];
        for (int k = 0; k < 7; ++k) {
            W_POW[j][k] = ko_powi(f, 1 + k) * W_VEC[k];
            U_POW[j][k] = ko_powi(f, 1 + k) * U_VEC[k];
        }
        FRAC2[j] = ko_powi(f, 2);
    }
    radau_init_done = 1;
}

/* force callback: returns error code, writes acceleration */
typedef int (*accel_fn)(double t, const double x[3], const double v[3], void *meta, int exact,
                        double out[3]);

typedef struct {
    double t, tf;
    double x[3], v[3], a[3];
    double b[3][7];
    int64_t n_steps, n_evals;
} radau_state;

static int radau_step(radau_state *s, accel_fn F, void *meta, double h, double *next_h) {
    double g[3][7];
    double xs[3], vs[3], ev[3];
    memset(g, 0, sizeof g);
    memcpy(ev, s->a, sizeof ev);
    for (int iter = 0; iter < 10; ++iter) {
        double b6_old[3] = {s->b[0][6], s->b[1][6], s->b[2][6]};
        for (int j = 1; j < 8; ++j) {
            double f = GR_SPACING[j];
            for (int c = 0; c < 3; ++c) {
                double bw = 0.0, bu = 0.0;
                for (int k = 0; k < 7; ++k) bw = W_POW[j][k] * s->b[c][k] + bw;
                for (int k = 0; k < 7; ++k) bu = U_POW[j][k] * s->b[c][k] + bu;
                xs[c] = s->x[c] + f * s->v[c] * h + FRAC2[j] * ko_powi(h, 2) * (s->a[c] / 2.0 + bw);
                vs[c] = s->v[c] + f * h * (s->a[c] + bu);
            }
            int rc = F(s->t + f * h, xs, vs, meta, 0, ev);
            s->n_evals++;
            if (rc) return rc;
            for (int c = 0; c < 3; ++c) {
                double gk = (ev[c] - s->a[c]) / f;
                for (int z = 1; z < j; ++z) gk = (gk - g[c][z - 1]) / (f - GR_SPACING[z]);
                g[c][j - 1] = gk;
            }
        }
        /* cur_b = g * C  (radau.rs:313) */
        for (int c = 0; c < 3; ++c)
            for (int jj = 0; jj < 7; ++jj) {
                double acc = 0.0;
                int first = 1;
                for (int k = 0; k < 7; ++k) {
                    double t = C_MAT[k][jj] * g[c][k];
                    if (first) {
                        acc = t;
                        first = 0;
                    } else
                        acc = t + acc;
                }
                s->b[c][jj] = acc;
            }
        double ratio[3], fem[3];
        for (int c = 0; c < 3; ++c) {
            fem[c] = fabs(ev[c]) + 1e-6;
            ratio[c] = fabs(s->b[c][6] - b6_old[c]) / fem[c];
        }
        if (fmax3(ratio) < 1e-14) {
            for (int c = 0; c < 3; ++c) {
                double dw = 0.0, du = 0.0;
                for (int k = 0; k < 7; ++k) dw = dw + s->b[c][k] * W_VEC[k];
                for (int k = 0; k < 7; ++k) du = du + s->b[c][k] * U_VEC[k];
                s->x[c] += s->v[c] * h + ko_powi(h, 2) * (s->a[c] * 0.5 + dw);
                s->v[c] += h * (s->a[c] + du);
            }
            s->t += h;
            int rc = F(s->t, s->x, s->v, meta, 1, s->a);
            s->n_evals++;
            if (rc) return rc;
            double ab6[3] = {fabs(s->b[0][6]), fabs(s->b[1][6]), fabs(s->b[2][6])};
            double r = pow(1e-6 * fmax3(fem) / fmax3(ab6), 1.0 / 7.0);
            *next_h = h * clampd(r, 0.25, 4.0);
            s->n_steps++;
            return KO_OK;
        }
    }
    return KO_CONVERGENCE;
}

static int radau_integrate(accel_fn F, void *meta, const double x0[3], const double v0[3],
                           double t0, double tf, double xo[3], double vo[3], int64_t *n_steps,
                           int64_t *n_evals) {
    radau_init();
    radau_state s;
    memset(&s, 0, sizeof s);
    s.t = t0;
    s.tf = tf;
    memcpy(s.x, x0, sizeof s.x);
    memcpy(s.v, v0, sizeof s.v);
    int rc = F(t0, s.x, s.v, meta, 1, s.a);
    s.n_evals++;
    if (rc) goto done;
    if (fabs(tf - t0) < 1e-10) goto ok;
    double h = copysign(0.1, tf - s.t);
    int failures = 0;
    for (;;) {
        if (fabs(s.t - tf) <= fabs(h)) h = tf - s.t;
        double nh;
        rc = radau_step(&s, F, meta, h, &nh);
        if (rc == KO_OK) {
            h = nh;
            if (fabs(s.t - tf) < 1e-12) goto ok;
            failures = 0;
        } else if (rc == KO_IMPACT || rc == KO_DAF_LIMITS) {
            goto done;
        } else {
            failures += 1;
            h *= 0.7;
            if (failures > 10) {
                rc = KO_CONVERGENCE;
                goto done;
            }
        }
        if (fabs(h) < 0.005) h = copysign(0.005, h);
    }
ok:
    rc = KO_OK;
    memcpy(xo, s.x, sizeof s.x);
    memcpy(vo, s.v, sizeof s.v);
done:
    if (n_steps) *n_steps = s.n_steps;
    if (n_evals) *n_evals = s.n_evals;
    return rc;
}

/* central_accel (kete_core/propagation/acceleration.rs:66-80) */
static int central_accel(double t, const double x[3], const double v[3], void *meta, int exact,
                         double out[3]) {
    (void)t; (void)v; (void)meta; (void)exact;
    double k = ko_powi(norm3(x), -3);
    for (int c = 0; c < 3; ++c) out[c] = -x[c] * k * GMS;
    return KO_OK;
}

int ko_radau_central(const double pos[3], const double vel[3], double t0, double t1,
                     double out_pos[3], double out_vel[3]) {
    return radau_integrate(central_accel, NULL, pos, vel, t0, t1, out_pos, out_vel, NULL, NULL);
}

/* ------------------------------------------------------------------------------------------
 * DAF / SPK types 2, 3, 1 and 21 (kete_core/spice/daf.rs:148-351, spk.rs:37-126,210-329,
 * spk_segments.rs:105-177,185-310 (type 1),316-397 (type 2),404-480 (type 3),
 * 964-1105 (type 21), interpolation.rs:25-130, spice/mod.rs:25-34)
 * ---------------------------------------------------------------------------------------- */
typedef struct {
    int64_t obj_id, center_id;
    int frame; /* KO_FRAME_* or -(raw frame code) */
    int seg_type;
    double jd_start, jd_end;
    double *data;
    int64_t n_data;
    double jd_step;              /* types 2, 3 */
    int64_t n_coef, record_len;  /* types 2, 3: coefficients per coordinate; 1, 21: MAXDIM */
    int64_t n_rec;               /* types 1, 21 */
} spk_segment;

static spk_segment *g_planet = NULL, *g_other = NULL;
static int g_n_planet = 0, g_n_other = 0, g_cap_planet = 0, g_cap_other = 0;

static double spice_jds_to_jd(double s) { return s / 86400.0 + 2451545.0; }
static double jd_to_spice_jd(double jd) { return (jd - 2451545.0) * 86400.0; }

int ko_spk_reset(void) {
    for (int i = 0; i < g_n_planet; ++i) free(g_planet[i].data);
    for (int i = 0; i < g_n_other; ++i) free(g_other[i].data);
    free(g_planet);
    free(g_other);
    g_planet = g_other = NULL;
    g_n_planet = g_n_other = g_cap_planet = g_cap_other = 0;
    return KO_OK;
}

static int32_t rd_i32(const uint8_t *p, int le) {
    uint32_t v;
    if (le)
        v = (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
    else
        v = (uint32_t)p[3] | ((uint32_t)p[2] << 8) | ((uint32_t)p[1] << 16) | ((uint32_t)p[0] << 24);
    return (int32_t)v;
}
static double rd_f64(const uint8_t *p, int le) {
    uint8_t b[8];
    for (int i = 0; i < 8; ++i) b[i] = le ? p[i] : p[7 - i];
    double d;
    memcpy(&d, b, 8);
    return d;
}

static int push_segment(spk_segment *s) {
    if (s->obj_id >= 0 && s->obj_id <= 1000) {
        if (g_n_planet == g_cap_planet) {
            g_cap_planet = g_cap_planet ? 2 * g_cap_planet : 16;
            g_planet = (spk_segment *)realloc(g_planet, (size_t)g_cap_planet * sizeof *s);
        }
        g_planet[g_n_planet++] = *s;
    } else {
        if (g_n_other == g_cap_other) {
            g_cap_other = g_cap_other ? 2 * g_cap_other : 16;
            g_other = (spk_segment *)realloc(g_other, (size_t)g_cap_other * sizeof *s);
        }
        g_other[g_n_other++] = *s;
    }
    return KO_OK;
}

int ko_spk_load_buffer(const uint8_t *buf, int64_t n_bytes) {
    if (n_bytes < 1024) return KO_IO_ERROR;
    char magic[9] = {0};
    memcpy(magic, buf, 8);
    if (strncmp(magic + 4, "SPK", 3) != 0 && strncmp(magic + 4, "spk", 3) != 0) return KO_IO_ERROR;
    int le;
    if (strncmp((const char *)buf + 88, "LTL-IEEE", 8) == 0)
        le = 1;
    else if (strncmp((const char *)buf + 88, "BIG-IEEE", 8) == 0)
        le = 0;
    else
        return KO_IO_ERROR;
    int nd = rd_i32(buf + 8, le), ni = rd_i32(buf + 12, le);
    int fward = rd_i32(buf + 76, le);
    if (nd != 2 || ni != 6) return KO_IO_ERROR;
    int summary_size = nd + (ni + 1) / 2;
    int next = fward;
    while (next != 0) {
        int64_t off = 1024LL * (next - 1);
        if (off + 1024 > n_bytes) return KO_IO_ERROR;
        const uint8_t *rec = buf + off;
        next = (int)rd_f64(rec, le);
        int n_sum = (int)rd_f64(rec + 16, le);
        for (int k = 0; k < n_sum; ++k) {
            const uint8_t *s = rec + 24 + (int64_t)k * summary_size * 8;
            double f0 = rd_f64(s, le), f1 = rd_f64(s + 8, le);
            int32_t iv[6];
            for (int q = 0; q < 6; ++q) iv[q] = rd_i32(s + 16 + 4 * q, le);
            int64_t a0 = iv[4], a1 = iv[5];
            int64_t nf = a1 - a0 + 1;
            if (nf <= 0 || 8 * (a0 - 1) + 8 * nf > n_bytes) return KO_IO_ERROR;
            spk_segment seg;
            memset(&seg, 0, sizeof seg);
            seg.jd_start = spice_jds_to_jd(f0);
            seg.jd_end = spice_jds_to_jd(f1);
            seg.obj_id = iv[0];
            seg.center_id = iv[1];
            seg.frame = iv[2] == 1 ? KO_FRAME_EQUATORIAL : (iv[2] == 17 ? KO_FRAME_ECLIPTIC : -iv[2]);
            seg.seg_type = iv[3];
            seg.n_data = nf;
            seg.data = (double *)malloc((size_t)nf * sizeof(double));
            for (int64_t q = 0; q < nf; ++q) seg.data[q] = rd_f64(buf + 8 * (a0 - 1) + 8 * q, le);
            int bad = 0;
            if (seg.seg_type == 2 || seg.seg_type == 3) {
                /* From<DafArray> for SpkSegmentType2 / 3 (spk_segments.rs:379-397, 482-498) */
                const int per = seg.seg_type == 2 ? 3 : 6;
                seg.record_len = (int64_t)seg.data[nf - 2];
                seg.jd_step = seg.data[nf - 3];
                seg.n_coef = (seg.record_len - 2) / per;
                bad = nf < 4 || per * seg.n_coef + 2 != seg.record_len || seg.n_coef < 2;
            } else if (seg.seg_type == 1 || seg.seg_type == 21) {
                /* From<DafArray> for SpkSegmentType1 / 21 (spk_segments.rs:302-308, 971-984) */
                seg.n_rec = (int64_t)seg.data[nf - 1];
                seg.n_coef = seg.seg_type == 1 ? 15 : (int64_t)seg.data[nf - 2];
                seg.record_len = 4 * seg.n_coef + 11;
                bad = seg.n_rec < 1 || seg.n_coef < 1 || seg.n_coef > 25 ||
                      seg.n_rec * (seg.record_len + 1) > nf;
            } else {
                bad = 1; /* types 2, 3, 1 and 21 are restated */
            }
            if (bad) {
                free(seg.data);
                return KO_IO_ERROR;
            }
            push_segment(&seg);
        }
    }
    return KO_OK;
}

/* chebyshev_evaluate_both (kete_core/spice/interpolation.rs:25-77) */
static void cheb_both(double x, const double *cx, const double *cy, const double *cz, int64_t n,
                      double val[3], double der[3]) {
    double x2 = 2.0 * x;
    val[0] = cx[0] + cx[1] * x;
    val[1] = cy[0] + cy[1] * x;
    val[2] = cz[0] + cz[1] * x;
    double second_t = 1.0, last_t = x, next_t;
    double second_u = 1.0, last_u = x2, next_u;
    der[0] = cx[1];
    der[1] = cy[1];
    der[2] = cz[1];
    for (int64_t idx = 2; idx < n; ++idx) {
        next_t = x2 * last_t - second_t;
        val[0] += cx[idx] * next_t;
        val[1] += cy[idx] * next_t;
        val[2] += cz[idx] * next_t;
        second_t = last_t;
        last_t = next_t;
        next_u = x2 * last_u - second_u;
        der[0] += cx[idx] * last_u * (double)idx;
        der[1] += cy[idx] * last_u * (double)idx;
        der[2] += cz[idx] * last_u * (double)idx;
        second_u = last_u;
        last_u = next_u;
    }
}

typedef struct {
    int64_t id, center;
    int frame;
    double pos[3], vel[3];
} ko_state;

/* chebyshev_evaluate (interpolation.rs:96-130): values only */
static void cheb_val(double x, const double *cx, const double *cy, const double *cz, int64_t n,
                     double val[3]) {
    double x2 = 2.0 * x;
    val[0] = cx[0] + cx[1] * x;
    val[1] = cy[0] + cy[1] * x;
    val[2] = cz[0] + cz[1] * x;
    double second_t = 1.0, last_t = x, next_t;
    for (int64_t idx = 2; idx < n; ++idx) {
        next_t = x2 * last_t - second_t;
        val[0] += cx[idx] * next_t;
        val[1] += cy[idx] * next_t;
        val[2] += cz[idx] * next_t;
        second_t = last_t;
        last_t = next_t;
    }
}

/* SpkSegmentType3::try_get_pos_vel (spk_segments.rs:446-480): Chebyshev position and
 * velocity polynomials, values only.  The record index is clamped to the segment. */
static void type3_state(const spk_segment *s, double jds, double p[3], double v[3]) {
    double start = jd_to_spice_jd(s->jd_start);
    double fidx = floor((jds - start) / s->jd_step);
    int64_t idx = fidx < 0 ? 0 : (int64_t)fidx;
    int64_t n_rec = (s->n_data - 4) / s->record_len;
    if (idx >= n_rec) idx = n_rec - 1;
    const double *rec = s->data + idx * s->record_len;
    const int64_t n = s->n_coef;
    double t = (jds - rec[0]) / rec[1];
    double pp[3], vv[3];
    cheb_val(t, rec + 2, rec + 2 + n, rec + 2 + 2 * n, n, pp);
    cheb_val(t, rec + 2 + 3 * n, rec + 2 + 4 * n, rec + 2 + 5 * n, n, vv);
    double t_scaled = 86400.0 / AU_KM;
    for (int c = 0; c < 3; ++c) {
        p[c] = pp[c] / AU_KM;
        v[c] = vv[c] * t_scaled;
    }
}

/* SpkSegmentType1 / 21::try_get_pos_vel (spk_segments.rs:207-290, 1008-1090): the modified
 * difference array of the first record whose final epoch is at or after t (SPICE's
 * SPKE21 interpolation).  Returns KO_IO_ERROR for a zero step-size entry. */
static int mda_state(const spk_segment *s, double jds, double p[3], double v[3]) {
    const int64_t nr = s->n_rec, md = s->n_coef, rl = s->record_len;
    const double *epochs = s->data + nr * rl;
    int64_t lo = 0, hi = nr; /* first index with epochs[idx] >= jds */
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (epochs[mid] < jds) lo = mid + 1;
        else hi = mid;
    }
    if (lo >= nr) lo = nr - 1; /* the reference reads past the records here */
    const double *rec = s->data + lo * rl;
    const double tl = rec[0];
    const double *g = rec + 1, *ref = rec + 1 + md, *dt_arr = rec + 7 + md;
    const int64_t kqmax1 = (int64_t)rec[4 * md + 7];
    const double *kq = rec + 4 * md + 8;
    if (kqmax1 < 2 || kqmax1 > md + 1 || kqmax1 > 26) return KO_IO_ERROR;
    for (int c = 0; c < 3; ++c)
        if (kq[c] < 0 || kq[c] > (double)(kqmax1 - 1)) return KO_IO_ERROR;
    const double delta = jds - tl;
    double fc[25], wc[25], w[27];
    double tp = delta;
    const int64_t mq2 = kqmax1 - 2;
    for (int64_t j = 0; j < mq2; ++j) {
        if (g[j] == 0.0) return KO_IO_ERROR;
        fc[j] = tp / g[j];
        wc[j] = delta / g[j];
        tp = delta + g[j];
    }
    for (int64_t j = 0; j < kqmax1; ++j) w[j] = 1.0 / (double)(j + 1);
    int64_t ks = kqmax1 - 1, ks1 = ks - 1, jx = 0;
    while (ks >= 2) {
        jx += 1;
        for (int64_t j = 0; j < jx; ++j) w[j + ks] = fc[j] * w[j + ks1] - wc[j] * w[j + ks];
        ks = ks1;
        ks1 -= 1;
    }
    for (int c = 0; c < 3; ++c) {
        double sum = 0.0;
        for (int64_t j = (int64_t)kq[c]; j >= 1; --j) sum += dt_arr[c * md + j - 1] * w[j + ks - 1];
        p[c] = (ref[2 * c] + delta * (sum * delta + ref[2 * c + 1])) / AU_KM;
    }
    for (int64_t j = 0; j < jx; ++j) w[j + ks] = fc[j] * w[j + ks1] - wc[j] * w[j + ks];
    ks -= 1;
    for (int c = 0; c < 3; ++c) {
        double sum = 0.0;
        for (int64_t j = (int64_t)kq[c]; j >= 1; --j) sum += dt_arr[c * md + j - 1] * w[j + ks - 1];
        v[c] = (ref[2 * c + 1] + delta * sum) / AU_KM * 86400.0;
    }
    return KO_OK;
}

/* SpkSegment::try_get_state + SpkSegmentType2::try_get_pos_vel */
static int seg_state(const spk_segment *s, double jd, ko_state *out) {
    if (jd < s->jd_start || jd > s->jd_end) return KO_DAF_LIMITS;
    if (s->seg_type != 2) {
        double jds3 = jd_to_spice_jd(jd), p[3], v[3];
        if (s->seg_type == 3) {
            type3_state(s, jds3, p, v);
        } else {
            int rc = mda_state(s, jds3, p, v);
            if (rc != KO_OK) return rc;
        }
        out->id = s->obj_id;
        out->center = s->center_id;
        out->frame = s->frame;
        for (int c = 0; c < 3; ++c) {
            out->pos[c] = p[c];
            out->vel[c] = v[c];
        }
        return KO_OK;
    }
    double jds = jd_to_spice_jd(jd);
    double start = jd_to_spice_jd(s->jd_start);
    double fidx = floor((jds - start) / s->jd_step);
    int64_t idx = fidx < 0 ? 0 : (int64_t)fidx;
    int64_t n_rec = (s->n_data - 4) / s->record_len;
    if (idx >= n_rec) idx = n_rec - 1; /* the reference reads past the records here */
    const double *rec = s->data + idx * s->record_len;
    double t_mid = rec[0], t_step = rec[1];
    double t = (jds - t_mid) / t_step;
    double tss = 86400.0 / t_step / AU_KM;
    double p[3], v[3];
    cheb_both(t, rec + 2, rec + 2 + s->n_coef, rec + 2 + 2 * s->n_coef, s->n_coef, p, v);
    out->id = s->obj_id;
    out->center = s->center_id;
    out->frame = s->frame;
    for (int c = 0; c < 3; ++c) {
        out->pos[c] = p[c] / AU_KM;
        out->vel[c] = v[c] * tss;
    }
    return KO_OK;
}

/* SpkCollection::try_get_raw_state (spk.rs:65-82) */
static int raw_state(int64_t id, double jd, ko_state *out) {
    for (int i = 0; i < g_n_planet; ++i) {
        const spk_segment *s = &g_planet[i];
        if (s->obj_id == id && jd >= s->jd_start && jd <= s->jd_end) return seg_state(s, jd, out);
    }
    for (int i = 0; i < g_n_other; ++i) {
        const spk_segment *s = &g_other[i];
        if (s->obj_id == id && jd >= s->jd_start && jd <= s->jd_end) return seg_state(s, jd, out);
    }
    return KO_DAF_LIMITS;
}

static void state_change_frame(ko_state *s, int target) {
    if (s->frame == target) return;
    double p[3], v[3];
    if (s->frame == KO_FRAME_EQUATORIAL) {
        eq_to_ecl(s->pos, p);
        eq_to_ecl(s->vel, v);
    } else {
        memcpy(p, s->pos, sizeof p);
        memcpy(v, s->vel, sizeof v);
    }
    if (target == KO_FRAME_EQUATORIAL) {
        ecl_to_eq(p, s->pos);
        ecl_to_eq(v, s->vel);
    } else {
        memcpy(s->pos, p, sizeof p);
        memcpy(s->vel, v, sizeof v);
    }
    s->frame = target;
}

/* State::try_change_center (kete_core/state.rs:242-281) */
static int state_apply_center(ko_state *self, ko_state other) {
    if (self->center != other.center && self->center != other.id) return KO_VALUE_ERROR;
    if (self->center == other.center) {
        int64_t t = other.id;
        other.id = other.center;
        other.center = t;
        for (int c = 0; c < 3; ++c) {
            other.pos[c] = -other.pos[c];
            other.vel[c] = -other.vel[c];
        }
    }
    if (self->frame != other.frame) state_change_frame(&other, self->frame);
    self->center = other.center;
    for (int c = 0; c < 3; ++c) {
        self->pos[c] += other.pos[c];
        self->vel[c] += other.vel[c];
    }
    return KO_OK;
}

/* find_path (spk.rs:210-234) as a breadth-first search over segment links */
static int find_path(int64_t start, int64_t goal, int64_t *path, int *n_path) {
    enum { MAXN = 256 };
    int64_t node[MAXN], via[MAXN];
    int parent[MAXN];
    int head = 0, tail = 0;
    node[tail] = start;
    via[tail] = INT64_MIN;
    parent[tail] = -1;
    tail++;
    while (head < tail) {
        int cur = head++;
        if (node[cur] == goal) {
            int64_t rev[MAXN];
            int m = 0;
            for (int k = cur; parent[k] >= 0; k = parent[k]) rev[m++] = via[k];
            for (int k = 0; k < m; ++k) path[k] = rev[m - 1 - k];
            *n_path = m;
            return KO_OK;
        }
        for (int pass = 0; pass < 2; ++pass) {
            int n = pass == 0 ? g_n_planet : g_n_other;
            spk_segment *arr = pass == 0 ? g_planet : g_other;
            for (int i = 0; i < n; ++i) {
                int64_t nb = -1, v = 0;
                if (arr[i].obj_id == node[cur]) {
                    nb = arr[i].center_id;
                    v = arr[i].obj_id;
                } else if (arr[i].center_id == node[cur]) {
                    nb = arr[i].obj_id;
                    v = arr[i].obj_id;
                } else
                    continue;
                int seen = 0;
                for (int k = 0; k < tail; ++k)
                    if (node[k] == nb) seen = 1;
                if (!seen && tail < MAXN) {
                    node[tail] = nb;
                    via[tail] = v;
                    parent[tail] = cur;
                    tail++;
                }
            }
        }
    }
    return KO_DAF_LIMITS;
}

/* SpkCollection::try_change_center (spk.rs:99-126) */
static int change_center(ko_state *s, int64_t new_center, double jd) {
    int64_t c = s->center;
    ko_state r;
    int rc;
    if (c == new_center) return KO_OK;
    if (new_center == 0 && c <= 10) {
        if ((rc = raw_state(c, jd, &r))) return rc;
        return state_apply_center(s, r);
    }
    if (c == 0 && new_center == 10) {
        if ((rc = raw_state(10, jd, &r))) return rc;
        return state_apply_center(s, r);
    }
    if (new_center == 10 && c < 10) {
        if ((rc = raw_state(c, jd, &r))) return rc;
        if ((rc = state_apply_center(s, r))) return rc;
        if ((rc = raw_state(10, jd, &r))) return rc;
        return state_apply_center(s, r);
    }
    if (c == 10 && new_center > 1 && new_center < 10) {
        if ((rc = raw_state(10, jd, &r))) return rc;
        if ((rc = state_apply_center(s, r))) return rc;
        if ((rc = raw_state(new_center, jd, &r))) return rc;
        return state_apply_center(s, r);
    }
    int64_t path[64];
    int np = 0;
    if ((rc = find_path(c, new_center, path, &np))) return rc;
    for (int k = 0; k < np; ++k) {
        if ((rc = raw_state(path[k], jd, &r))) return rc;
        if ((rc = state_apply_center(s, r))) return rc;
    }
    return KO_OK;
}

/* SpkCollection::try_get_state (spk.rs:87-96) */
static int get_state(int64_t id, double jd, int64_t center, int frame, ko_state *out) {
    int rc = raw_state(id, jd, out);
    if (rc) return rc;
    if (out->center != center)
        if ((rc = change_center(out, center, jd))) return rc;
    if (out->frame != frame) state_change_frame(out, frame);
    return KO_OK;
}

int ko_spk_get_state(int64_t id, double jd, int64_t center, int frame, double out6[6]) {
    ko_state s;
    int rc = get_state(id, jd, center, frame, &s);
    if (rc) return rc;
    memcpy(out6, s.pos, 3 * sizeof(double));
    memcpy(out6 + 3, s.vel, 3 * sizeof(double));
    return KO_OK;
}

/* SpkCollection::try_get_state for many epochs (the batch form of the call above), OpenMP
 * over the epochs; out6 is 6 x n (SoA). */
int ko_spk_get_states(int64_t n, int64_t id, const double *jd, int64_t center, int frame,
                      double *out6, int32_t *status, int threads) {
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < n; ++i) {
        double o[6] = {0, 0, 0, 0, 0, 0};
        int rc = ko_spk_get_state(id, jd[i], center, frame, o);
        status[i] = rc;
        for (int c = 0; c < 6; ++c) out6[c * n + i] = rc == KO_OK ? o[c] : NAN;
    }
    return KO_OK;
}

/* ------------------------------------------------------------------------------------------
 * forces (kete_core/constants/gravity.rs:171-253, propagation/nongrav.rs:114-157,
 * propagation/acceleration.rs:121-168)
 * ---------------------------------------------------------------------------------------- */
static void j2_correction(const double rp[3], double radius, double j2, double mass, double o[3]) {
    double r = norm3(rp);
    double z_squared = 5.0 * ko_powi(rp[2] / r, 2);
    double coef = 1.5 * j2 * mass * ko_powi(radius / r, 2) * ko_powi(r, -3);
    o[0] = rp[0] * coef * (z_squared - 1.0);
    o[1] = rp[1] * coef * (z_squared - 1.0);
    o[2] = rp[2] * coef * (z_squared - 3.0);
}

static void apply_gr(double acc[3], const double rp[3], const double rv[3], double mass) {
    double r_v = 4.0 * dot3(rp, rv);
    double rel_v2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
    double r = norm3(rp);
    double gr_const = mass * C_AU_PER_DAY_INV_SQUARED * ko_powi(r, -3);
    double c = 4. * mass / r - rel_v2;
    for (int i = 0; i < 3; ++i) acc[i] += gr_const * (c * rp[i] + r_v * rv[i]);
}

static void grav_add(const grav_params *gp, double acc[3], const double rp[3], const double rv[3]) {
    double mass = gp->mass;
    double k = mass * ko_powi(norm3(rp), -3);
    for (int i = 0; i < 3; ++i) acc[i] -= rp[i] * k;
    if (gp->naif_id == 5 || gp->naif_id == 10) {
        apply_gr(acc, rp, rv, mass);
        double re[3], j2[3], j2q[3];
        eq_to_ecl(rp, re);
        j2_correction(re, gp->radius, gp->naif_id == 5 ? JUPITER_J2 : SUN_J2, mass, j2);
        ecl_to_eq(j2, j2q);
        for (int i = 0; i < 3; ++i) acc[i] += j2q[i];
    } else if (gp->naif_id == 399) {
        double j2[3];
        j2_correction(rp, gp->radius, EARTH_J2, mass, j2);
        for (int i = 0; i < 3; ++i) acc[i] += j2[i];
    }
}

static void normalize3(const double v[3], double o[3]) {
    double n = norm3(v);
    for (int i = 0; i < 3; ++i) o[i] = v[i] / n;
}

static void nongrav_add(const double *ng, double acc[3], const double pos_in[3], const double vel[3]) {
    int kind = (int)ng[0];
    if (kind == 2) {
        double beta = ng[1];
        double pn[3];
        normalize3(pos_in, pn);
        double r_dot = dot3(pn, vel);
        double norm2_inv = 1.0 / (pos_in[0] * pos_in[0] + pos_in[1] * pos_in[1] + pos_in[2] * pos_in[2]);
        double scaling = GMS * beta * norm2_inv;
        for (int i = 0; i < 3; ++i)
            acc[i] += scaling * ((1.0 - r_dot * C_AU_PER_DAY_INV_SQUARED) * pn[i] - vel[i] * C_AU_PER_DAY_INV_SQUARED);
    } else if (kind == 1) {
        double a1 = ng[1], a2 = ng[2], a3 = ng[3], alpha = ng[4], r_0 = ng[5], m = ng[6], n = ng[7],
               k = ng[8], dt = ng[9];
        double pos[3] = {pos_in[0], pos_in[1], pos_in[2]};
        double pn[3], tv[3], t_vec[3], nv[3], n_vec[3];
        normalize3(pos, pn);
        double vdp = dot3(vel, pn);
        for (int i = 0; i < 3; ++i) tv[i] = vel[i] - pn[i] * vdp;
        normalize3(tv, t_vec);
        nv[0] = t_vec[1] * pn[2] - t_vec[2] * pn[1];
        nv[1] = t_vec[2] * pn[0] - t_vec[0] * pn[2];
        nv[2] = t_vec[0] * pn[1] - t_vec[1] * pn[0];
        normalize3(nv, n_vec);
        if (dt != 0.0) {
            double p2[3], v2[3];
            if (analytic_2_body_d(-dt, pos, vel, 0, p2, v2) == KO_OK) memcpy(pos, p2, sizeof p2);
        }
        double rr0 = norm3(pos) / r_0;
        double scale = alpha * pow(rr0, -m) * pow(1.0 + pow(rr0, n), -k);
        for (int i = 0; i < 3; ++i) acc[i] += pn[i] * (scale * a1);
        for (int i = 0; i < 3; ++i) acc[i] += t_vec[i] * (scale * a2);
        for (int i = 0; i < 3; ++i) acc[i] += n_vec[i] * (scale * a3);
    }
}

typedef struct {
    int include_extended;
    const double *ng;
    int64_t impact_id;
    double impact_jd;
} spk_meta;

int ko_spk_accel(double t, const double pos[3], const double vel[3], int include_extended,
                 const double *ng, int exact, double out[3], int64_t *impact_id) {
    int n_bodies = include_extended ? 15 : 10;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < n_bodies; ++b) {
        const grav_params *gp = &MASSES[b];
        ko_state st;
        int rc = get_state(gp->naif_id, t, 0, KO_FRAME_EQUATORIAL, &st);
        if (rc) return rc;
        double rp[3], rv[3];
        for (int i = 0; i < 3; ++i) {
            rp[i] = pos[i] - st.pos[i];
            rv[i] = vel[i] - st.vel[i];
        }
        if (exact) {
            double r = norm3(rp);
            if (r <= gp->radius) {
                if (impact_id) *impact_id = gp->naif_id;
                return KO_IMPACT;
            }
        }
        grav_add(gp, acc, rp, rv);
        if (gp->naif_id == 10 && ng) nongrav_add(ng, acc, rp, rv);
    }
    memcpy(out, acc, sizeof acc);
    return KO_OK;
}

static int spk_accel_cb(double t, const double x[3], const double v[3], void *meta, int exact,
                        double out[3]) {
    spk_meta *m = (spk_meta *)meta;
    int64_t id = 0;
    int rc = ko_spk_accel(t, x, v, m->include_extended, m->ng, exact, out, &id);
    if (rc == KO_IMPACT) {
        m->impact_id = id;
        m->impact_jd = t;
    }
    return rc;
}

/* propagate_n_body_spk (kete_core/propagation/mod.rs:70-118) */
int ko_propagate_n_body_spk(const double pos[3], const double vel[3], double jd0, int frame,
                            int64_t center, double jd1, int include_extended, const double *ng,
                            double out_pos[3], double out_vel[3], int64_t *impact_id,
                            double *impact_jd, int64_t *n_steps, int64_t *n_evals) {
    ko_state s;
    s.id = -1;
    s.center = center;
    s.frame = frame;
    memcpy(s.pos, pos, sizeof s.pos);
    memcpy(s.vel, vel, sizeof s.vel);
    int rc = change_center(&s, 0, jd0);
    if (rc) return rc;
    state_change_frame(&s, KO_FRAME_EQUATORIAL);
    spk_meta meta = {include_extended, (ng && ng[0] != 0.0) ? ng : NULL, 0, 0.0};
    double xo[3], vo[3];
    rc = radau_integrate(spk_accel_cb, &meta, s.pos, s.vel, jd0, jd1, xo, vo, n_steps, n_evals);
    if (rc) {
        if (rc == KO_IMPACT) {
            if (impact_id) *impact_id = meta.impact_id;
            if (impact_jd) *impact_jd = meta.impact_jd;
        }
        return rc;
    }
    ko_state ns;
    ns.id = -1;
    ns.center = 0;
    ns.frame = KO_FRAME_EQUATORIAL;
    memcpy(ns.pos, xo, sizeof xo);
    memcpy(ns.vel, vo, sizeof vo);
    if ((rc = change_center(&ns, center, jd1))) return rc;
    state_change_frame(&ns, frame);
    memcpy(out_pos, ns.pos, sizeof ns.pos);
    memcpy(out_vel, ns.vel, sizeof ns.vel);
    return KO_OK;
}

void ko_propagate_n_body_batch(int64_t n, const double *pos, const double *vel,
                               const double *jd0, const double *jd1, int frame, int64_t center,
                               int include_extended, const double *ng, double *out_pos,
                               double *out_vel, int32_t *status, int64_t *n_steps,
                               int64_t *n_evals, int n_threads) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
    for (int64_t i = 0; i < n; ++i) {
        double p[3] = {pos[i], pos[n + i], pos[2 * n + i]};
        double v[3] = {vel[i], vel[n + i], vel[2 * n + i]};
        double op[3], ov[3];
        double ngrow[KO_NG_STRIDE];
        const double *ngp = NULL;
        if (ng) {
            for (int q = 0; q < KO_NG_STRIDE; ++q) ngrow[q] = ng[(int64_t)q * n + i];
            ngp = ngrow;
        }
        int64_t ns = 0, ne = 0, iid = 0;
        double ijd = 0.0;
        int rc = KO_VALUE_ERROR;
        if (isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]) && isfinite(v[0]) && isfinite(v[1]) &&
            isfinite(v[2]) && isfinite(jd0[i]))
            rc = ko_propagate_n_body_spk(p, v, jd0[i], frame, center, jd1[i], include_extended, ngp,
                                         op, ov, &iid, &ijd, &ns, &ne);
        if (rc) op[0] = op[1] = op[2] = ov[0] = ov[1] = ov[2] = NAN;
        for (int c = 0; c < 3; ++c) {
            out_pos[c * n + i] = op[c];
            out_vel[c * n + i] = ov[c];
        }
        status[i] = rc;
        if (n_steps) n_steps[i] = ns;
        if (n_evals) n_evals[i] = ne;
    }
}

/* ------------------------------------------------------------------------------------------
 * FOV (kete_core/fov/patches.rs:122-155,214-234, fov/fov_like.rs:43-192,
 * frames/definitions.rs:356-363)
 * ---------------------------------------------------------------------------------------- */
/* Rotation3::from_axis_angle(UnitVector3::new_normalize(axis), angle) * v */
static void rotate_around(const double v[3], const double axis_in[3], double angle, double o[3]) {
    if (angle == 0.0) { /* from_axis_angle returns the identity for a zero angle */
        o[0] = v[0];
        o[1] = v[1];
        o[2] = v[2];
        return;
    }
    double ax[3];
    normalize3(axis_in, ax);
    double ux = ax[0], uy = ax[1], uz = ax[2];
    double sqx = ux * ux, sqy = uy * uy, sqz = uz * uz;
    double s = sin(angle), c = cos(angle);
    double omc = 1.0 - c;
    double m[3][3] = {
        {sqx + (1.0 - sqx) * c, ux * uy * omc - uz * s, ux * uz * omc + uy * s},
        {ux * uy * omc + uz * s, sqy + (1.0 - sqy) * c, uy * uz * omc - ux * s},
        {ux * uz * omc - uy * s, uy * uz * omc + ux * s, sqz + (1.0 - sqz) * c},
    };
    for (int i = 0; i < 3; ++i) o[i] = (v[0] * m[i][0] + v[1] * m[i][1]) + v[2] * m[i][2];
}

static void cross3(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

void ko_rect_from_pointing(const double pointing[3], double rotation, double lon_width,
                           double lat_width, double nrm[12]) {
    double z[3] = {0.0, 0.0, 1.0};
    double up0[3], left[3], up[3], nl[3], nu[3];
    rotate_around(z, pointing, -rotation, up0);
    cross3(pointing, up0, left);
    cross3(pointing, left, up);
    nl[0] = -left[0]; nl[1] = -left[1]; nl[2] = -left[2];
    nu[0] = -up[0]; nu[1] = -up[1]; nu[2] = -up[2];
    rotate_around(left, up, -lon_width / 2.0, nrm + 0);
    rotate_around(up, left, lat_width / 2.0, nrm + 3);
    rotate_around(nl, up, lon_width / 2.0, nrm + 6);
    rotate_around(nu, left, -lat_width / 2.0, nrm + 9);
}

int ko_rect_contains(const double nrm[12], const double v[3], double *dist) {
    double closest = -INFINITY;
    for (int e = 0; e < 4; ++e) {
        double d = dot3(v, nrm + 3 * e);
        if (isnan(d)) {
            *dist = d;
            return 0;
        }
        if (signbit(d) && fabs(d) > closest) closest = fabs(d);
    }
    if (isfinite(closest)) {
        *dist = fmin(closest, norm3(v));
        return 0;
    }
    *dist = 0.0;
    return 1;
}

/* SphericalCone::contains (fov/patches.rs:300-337): prm = unit pointing (3), half-angle */
int ko_cone_contains(const double prm[4], const double v[3], double *dist) {
    double r = norm3(v);
    double u[3] = {v[0] / r, v[1] / r, v[2] / r};
    double d = fabs(acos(dot3(prm, u)));
    if (d <= prm[3]) {
        *dist = 0.0;
        return 1;
    }
    double min_angle = fabs(d - prm[3]);
    *dist = min_angle > 1.5707963267948966 ? r : sin(min_angle) * r;
    return 0;
}

/* One patch of a field: kind 0 rectangle (4 edge normals), 1 cone (pointing, half-angle),
 * 2 omnidirectional (OmniDirectional::contains, fov/generic.rs:123-125: always inside). */
int ko_patch_contains(const double prm[12], int kind, const double v[3], double *dist) {
    if (kind == 1) return ko_cone_contains(prm, v, dist);
    if (kind == 2) {
        *dist = 0.0;
        return 1;
    }
    return ko_rect_contains(prm, v, dist);
}

typedef struct {
    double jd, pos[3], vel[3];
} fstate;

static int check_two_body_fov(const double obs7[7], const double nrm[12], int kind,
                              const fstate *s, int *inside, double *dist, fstate *fin) {
    double op[3], ov[3];
    int rc = analytic_2_body_d(obs7[0] - s->jd, s->pos, s->vel, 0, op, ov);
    if (rc) return rc;
    double d[3] = {op[0] - obs7[1], op[1] - obs7[2], op[2] - obs7[3]};
    double dt = -norm3(d) * C_AU_PER_DAY_INV;
    double p2[3], v2[3];
    double t2 = obs7[0] + dt;
    rc = analytic_2_body_d(t2 - obs7[0], op, ov, 0, p2, v2);
    if (rc) return rc;
    double rel[3] = {p2[0] - obs7[1], p2[1] - obs7[2], p2[2] - obs7[3]};
    *inside = ko_patch_contains(nrm, kind, rel, dist);
    fin->jd = t2;
    memcpy(fin->pos, p2, sizeof p2);
    memcpy(fin->vel, v2, sizeof v2);
    return KO_OK;
}

static int check_n_body_fov(const double obs7[7], const double nrm[12], int kind,
                            const fstate *s, int include_extended, int *inside, double *dist,
                            fstate *fin) {
    double op[3], ov[3];
    /* states here are heliocentric ecliptic (center 10, frame Ecliptic) */
    int rc = ko_propagate_n_body_spk(s->pos, s->vel, s->jd, KO_FRAME_ECLIPTIC, 10, obs7[0],
                                     include_extended, NULL, op, ov, NULL, NULL, NULL, NULL);
    if (rc) return rc;
    double d[3] = {op[0] - obs7[1], op[1] - obs7[2], op[2] - obs7[3]};
    double dt = -norm3(d) * C_AU_PER_DAY_INV;
    double p2[3], v2[3];
    double t2 = obs7[0] + dt;
    rc = analytic_2_body_d(t2 - obs7[0], op, ov, 0, p2, v2);
    if (rc) return rc;
    double rel[3] = {p2[0] - obs7[1], p2[1] - obs7[2], p2[2] - obs7[3]};
    *inside = ko_patch_contains(nrm, kind, rel, dist);
    fin->jd = t2;
    memcpy(fin->pos, p2, sizeof p2);
    memcpy(fin->vel, v2, sizeof v2);
    return KO_OK;
}

void ko_fov_check_visible(const double obs7[7], const double nrm[12], int64_t n,
                          const double *pos, const double *vel, const double *jd,
                          double dt_limit, int include_extended, int32_t *flags, double *out7) {
    ko_fov_check_visible_kind(obs7, nrm, 0, n, pos, vel, jd, dt_limit, include_extended, flags,
                              out7);
}

/* check_visible for a patch of any kind (ko_patch_contains) */
void ko_fov_check_visible_kind(const double obs7[7], const double nrm[12], int kind, int64_t n,
                               const double *pos, const double *vel, const double *jd,
                               double dt_limit, int include_extended, int32_t *flags,
                               double *out7) {
#pragma omp parallel for schedule(dynamic, 1000)
    for (int64_t i = 0; i < n; ++i) {
        fstate s;
        s.jd = jd[i];
        for (int c = 0; c < 3; ++c) {
            s.pos[c] = pos[c * n + i];
            s.vel[c] = vel[c * n + i];
        }
        double dv[3] = {s.vel[0] - obs7[4], s.vel[1] - obs7[5], s.vel[2] - obs7[6]};
        double max_dist = norm3(dv) * dt_limit * 2.0;
        int vis = 0, inside = 0;
        double dist = 0.0;
        fstate fin;
        memset(&fin, 0, sizeof fin);
        if (fabs(s.jd - obs7[0]) < dt_limit) {
            /* check_linear (fov_like.rs:43-66) */
            double rel[3] = {s.pos[0] - obs7[1], s.pos[1] - obs7[2], s.pos[2] - obs7[3]};
            double dt = obs7[0] - s.jd - norm3(rel) * C_AU_PER_DAY_INV;
            double np[3], nrel[3];
            for (int c = 0; c < 3; ++c) np[c] = s.pos[c] + s.vel[c] * dt;
            for (int c = 0; c < 3; ++c) nrel[c] = np[c] - obs7[1 + c];
            int lin_in = ko_patch_contains(nrm, kind, nrel, &dist);
            if (!(!lin_in && dist > max_dist)) {
                if (check_two_body_fov(obs7, nrm, kind, &s, &inside, &dist, &fin) == KO_OK && inside) vis = 1;
            }
        } else {
            if (check_two_body_fov(obs7, nrm, kind, &s, &inside, &dist, &fin) == KO_OK) {
                if (!(!inside && dist > max_dist)) {
                    if (check_n_body_fov(obs7, nrm, kind, &s, include_extended, &inside, &dist, &fin) == KO_OK &&
                        inside)
                        vis = 1;
                }
            }
        }
        flags[i] = vis;
        if (out7) {
            out7[i] = vis ? fin.jd : NAN;
            for (int c = 0; c < 3; ++c) {
                out7[(1 + c) * n + i] = vis ? fin.pos[c] : NAN;
                out7[(4 + c) * n + i] = vis ? fin.vel[c] : NAN;
            }
        }
    }
}

/* ------------------------------------------------------------------------------------------
 * propagate_n_body_vec (kete_core/propagation/mod.rs:142-237) with vec_accel
 * (acceleration.rs:197-249): the massive bodies of SIMPLE_PLANETS (constants/gravity.rs:
 * 137-153) integrated together with a batch of test particles by one Radau integration over
 * all their coordinates (radau.rs:160-346 on a DVector).
 * ---------------------------------------------------------------------------------------- */
#define N_SIMPLE 9
static const int64_t SIMPLE_IDS[N_SIMPLE] = {10, 1, 2, 3, 4, 5, 6, 7, 8};

static void simple_params(grav_params out[N_SIMPLE]) {
    const int from_masses[N_SIMPLE] = {0, 1, 2, -1, 5, 6, 7, 8, 9};
    for (int k = 0; k < N_SIMPLE; ++k) {
        if (from_masses[k] >= 0) {
            out[k] = MASSES[from_masses[k]];
        } else { /* EM_BARY (gravity.rs:137-142) */
            out[k].naif_id = 3;
            out[k].mass = (3.00348961546514e-06 + 3.69430335010988e-08) * GMS;
            out[k].radius = 385000.0 / AU_KM;
        }
    }
}

typedef struct {
    int m;                     /* bodies: N_SIMPLE massive, then the test particles */
    const double *ng;          /* 10 rows per test particle (row-major per particle) or NULL */
    grav_params gp[N_SIMPLE];
} vec_meta;

/* vec_accel: every body feels every massive body but itself; the comet / dust model acts
 * relative to the Sun on test particles after the first of the batch (the reference's
 * `idx > n_massive`, acceleration.rs:239-240, skips the first one). */
static int vec_accel(double t, const double *x, const double *v, const vec_meta *m, int exact,
                     double *out) {
    (void)t;
    for (int i = 0; i < m->m; ++i) {
        double acc[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < N_SIMPLE; ++k) {
            if (i == k) continue;
            double rp[3], rv[3], w[3] = {0.0, 0.0, 0.0};
            for (int c = 0; c < 3; ++c) {
                rp[c] = x[3 * i + c] - x[3 * k + c];
                rv[c] = v[3 * i + c] - v[3 * k + c];
            }
            if (exact && norm3(rp) <= m->gp[k].radius) return KO_IMPACT;
            grav_add(&m->gp[k], w, rp, rv);
            if (m->gp[k].naif_id == 10 && i > N_SIMPLE && m->ng) {
                const double *ng = m->ng + 10 * (i - N_SIMPLE);
                if ((int)ng[0] != 0) nongrav_add(ng, w, rp, rv);
            }
            for (int c = 0; c < 3; ++c) acc[c] += w[c];
        }
        memcpy(out + 3 * i, acc, sizeof acc);
    }
    return KO_OK;
}

/* vec_accel (acceleration.rs:197-249) for n test particles under m massive bodies whose
 * barycentric equatorial states the caller gives (massive: 6 x m rows x, y, z, vx, vy, vz):
 * bodies 0 = PLANETS (MASSES[0..10)), 1 = MASSES, 2 = SIMPLE_PLANETS.  Every particle sums
 * add_acceleration over the massive list in order, and the non-gravitational model (ng:
 * 10 x n, column i for particle i, or NULL) relative to the Sun; exact checks r <= radius.
 * The reference's batch quirk of skipping the first particle's model belongs to the batch
 * integration (vec_accel above), not to this per-particle form. */
int ko_vec_accel(int bodies, const double *massive, int64_t n, const double *pos,
                 const double *vel, const double *ng, int exact, double *out, int32_t *status) {
    grav_params simple[N_SIMPLE];
    simple_params(simple);
    const grav_params *gp = bodies == 2 ? simple : MASSES;
    const int m = bodies == 2 ? N_SIMPLE : (bodies == 1 ? 15 : 10);
    for (int64_t i = 0; i < n; ++i) {
        double x[3], v[3], acc[3] = {0.0, 0.0, 0.0}, row[10];
        for (int c = 0; c < 3; ++c) {
            x[c] = pos[c * n + i];
            v[c] = vel[c * n + i];
        }
        if (ng)
            for (int r = 0; r < 10; ++r) row[r] = ng[r * n + i];
        int rc = KO_OK;
        for (int k = 0; k < m; ++k) {
            double rp[3], rv[3], w[3] = {0.0, 0.0, 0.0};
            for (int c = 0; c < 3; ++c) {
                rp[c] = x[c] - massive[c * m + k];
                rv[c] = v[c] - massive[(3 + c) * m + k];
            }
            if (exact && norm3(rp) <= gp[k].radius) {
                rc = KO_IMPACT;
                break;
            }
            grav_add(&gp[k], w, rp, rv);
            if (gp[k].naif_id == 10 && ng && (int)row[0] != 0) nongrav_add(row, w, rp, rv);
            for (int c = 0; c < 3; ++c) acc[c] += w[c];
        }
        for (int c = 0; c < 3; ++c) out[c * n + i] = rc == KO_OK ? acc[c] : NAN;
        status[i] = rc;
    }
    return KO_OK;
}

/* RadauIntegrator::integrate / step (radau.rs:160-346) over d coordinates */
static int radau_vec(int d, double *x, double *v, double t0, double tf, const vec_meta *m) {
    radau_init();
    double *a = calloc((size_t)d, sizeof(double)), *ev = calloc((size_t)d, sizeof(double));
    double *xs = calloc((size_t)d, sizeof(double)), *vs = calloc((size_t)d, sizeof(double));
    double *b = calloc((size_t)d * 7, sizeof(double)), *g = calloc((size_t)d * 7, sizeof(double));
    double *b6_old = calloc((size_t)d, sizeof(double));
    double t = t0;
    int rc = vec_accel(t, x, v, m, 1, a);
    if (rc) goto done;
    if (fabs(tf - t0) < 1e-10) goto done;
    double h = copysign(0.1, tf - t);
    int failures = 0;
    for (;;) {
        if (fabs(t - tf) <= fabs(h)) h = tf - t;
        /* one step */
        int converged = 0;
        double next_h = h;
        memset(g, 0, (size_t)d * 7 * sizeof(double));
        memcpy(ev, a, (size_t)d * sizeof(double));
        for (int iter = 0; iter < 10 && !converged; ++iter) {
            for (int q = 0; q < d; ++q) b6_old[q] = b[7 * q + 6];
            for (int j = 1; j < 8; ++j) {
                double f = GR_SPACING[j];
                for (int q = 0; q < d; ++q) {
                    double bw = 0.0, bu = 0.0;
                    for (int k = 0; k < 7; ++k) bw = W_POW[j][k] * b[7 * q + k] + bw;
                    for (int k = 0; k < 7; ++k) bu = U_POW[j][k] * b[7 * q + k] + bu;
                    xs[q] = x[q] + f * v[q] * h + FRAC2[j] * ko_powi(h, 2) * (a[q] / 2.0 + bw);
                    vs[q] = v[q] + f * h * (a[q] + bu);
                }
                rc = vec_accel(t + f * h, xs, vs, m, 0, ev);
                if (rc) goto done;
                for (int q = 0; q < d; ++q) {
                    double gk = (ev[q] - a[q]) / f;
                    for (int z = 1; z < j; ++z) gk = (gk - g[7 * q + z - 1]) / (f - GR_SPACING[z]);
                    g[7 * q + j - 1] = gk;
                }
            }
            for (int q = 0; q < d; ++q)
                for (int jj = 0; jj < 7; ++jj) {
                    double acc = 0.0;
                    int first = 1;
                    for (int k = 0; k < 7; ++k) {
                        double tt = C_MAT[k][jj] * g[7 * q + k];
                        if (first) {
                            acc = tt;
                            first = 0;
                        } else
                            acc = tt + acc;
                    }
                    b[7 * q + jj] = acc;
                }
            double ratio = 0.0, fem_max = 0.0, b6_max = 0.0;
            for (int q = 0; q < d; ++q) {
                double fem = fabs(ev[q]) + 1e-6;
                double r = fabs(b[7 * q + 6] - b6_old[q]) / fem;
                if (r > ratio) ratio = r;
                if (fem > fem_max) fem_max = fem;
                if (fabs(b[7 * q + 6]) > b6_max) b6_max = fabs(b[7 * q + 6]);
            }
            if (ratio < 1e-14) {
                for (int q = 0; q < d; ++q) {
                    double dw = 0.0, du = 0.0;
                    for (int k = 0; k < 7; ++k) dw = dw + b[7 * q + k] * W_VEC[k];
                    for (int k = 0; k < 7; ++k) du = du + b[7 * q + k] * U_VEC[k];
                    x[q] += v[q] * h + ko_powi(h, 2) * (a[q] * 0.5 + dw);
                    v[q] += h * (a[q] + du);
                }
                t += h;
                rc = vec_accel(t, x, v, m, 1, a);
                if (rc) goto done;
                next_h = h * clampd(pow(1e-6 * fem_max / b6_max, 1.0 / 7.0), 0.25, 4.0);
                converged = 1;
            }
        }
        if (converged) {
            h = next_h;
            if (fabs(t - tf) < 1e-12) break;
            failures = 0;
        } else {
            failures += 1;
            h *= 0.7;
            if (failures > 10) {
                rc = KO_CONVERGENCE;
                goto done;
            }
        }
        if (fabs(h) < 0.005) h = copysign(0.005, h);
    }
    rc = KO_OK;
done:
    free(a);
    free(ev);
    free(xs);
    free(vs);
    free(b);
    free(g);
    free(b6_old);
    return rc;
}

/* n objects (heliocentric equatorial, 3 x n SoA) at jd0 to jd1 in batches of batch_size,
 * each with the 9 massive bodies (planets: 9 x 6 row-major heliocentric equatorial states
 * at jd0, or NULL to read them from the loaded SPK); ng 10 x n or NULL.  out_planets
 * (9 x 6, may be NULL) receives the massive bodies of the last batch.  status[i] is the
 * failure of object i's batch. */
int ko_propagate_n_body_vec(int64_t n, const double *pos, const double *vel, double jd0,
                            double jd1, const double *planets, const double *ng, int batch_size,
                            double *out_pos, double *out_vel, double *out_planets,
                            int32_t *status, int n_threads) {
    if (batch_size < 1) return KO_VALUE_ERROR;
    double p0[N_SIMPLE * 6];
    for (int k = 0; k < N_SIMPLE; ++k) {
        if (planets) {
            memcpy(p0 + 6 * k, planets + 6 * k, 6 * sizeof(double));
        } else {
            ko_state st;
            int rc = get_state(SIMPLE_IDS[k], jd0, 10, KO_FRAME_EQUATORIAL, &st);
            if (rc) return rc;
            memcpy(p0 + 6 * k, st.pos, 3 * sizeof(double));
            memcpy(p0 + 6 * k + 3, st.vel, 3 * sizeof(double));
        }
    }
    const int64_t n_batch = (n + batch_size - 1) / batch_size;
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
    for (int64_t bi = 0; bi < n_batch; ++bi) {
        const int64_t i0 = bi * batch_size;
        const int nb = (int)((n - i0) < batch_size ? (n - i0) : batch_size);
        const int mm = N_SIMPLE + nb, d = 3 * mm;
        double *x = malloc((size_t)d * sizeof(double)), *v = malloc((size_t)d * sizeof(double));
        double *ngb = ng ? malloc((size_t)10 * nb * sizeof(double)) : NULL;
        for (int k = 0; k < N_SIMPLE; ++k)
            for (int c = 0; c < 3; ++c) {
                x[3 * k + c] = p0[6 * k + c];
                v[3 * k + c] = p0[6 * k + 3 + c];
            }
        for (int q = 0; q < nb; ++q)
            for (int c = 0; c < 3; ++c) {
                x[3 * (N_SIMPLE + q) + c] = pos[c * n + i0 + q];
                v[3 * (N_SIMPLE + q) + c] = vel[c * n + i0 + q];
            }
        if (ngb)
            for (int q = 0; q < nb; ++q)
                for (int r = 0; r < 10; ++r) ngb[10 * q + r] = ng[r * n + i0 + q];
        vec_meta m;
        m.m = mm;
        m.ng = ngb;
        simple_params(m.gp);
        int rc = radau_vec(d, x, v, jd0, jd1, &m);
        for (int q = 0; q < nb; ++q) {
            status[i0 + q] = rc;
            for (int c = 0; c < 3; ++c) {
                out_pos[c * n + i0 + q] = rc ? NAN : x[3 * (N_SIMPLE + q) + c] - x[c];
                out_vel[c * n + i0 + q] = rc ? NAN : v[3 * (N_SIMPLE + q) + c] - v[c];
            }
        }
        if (out_planets && bi == n_batch - 1)
            for (int k = 0; k < N_SIMPLE; ++k)
                for (int c = 0; c < 3; ++c) {
                    out_planets[6 * k + c] = x[3 * k + c] - x[c];
                    out_planets[6 * k + 3 + c] = v[3 * k + c] - v[c];
                }
        free(x);
        free(v);
        free(ngb);
    }
    return KO_OK;
}

/* ------------------------------------------------------------------------------------------
 * two-body state-transition matrix: compute_state_transition (kete_core/propagation/
 * state_transition.rs:6-122) on the RK4(5) Fehlberg integrator (runge_kutta.rs:33-158), with
 * its three defects corrected: the Jacobian of the central acceleration is
 * cm (3 r r^T - r^2 I) / r^5 (acceleration.rs:267-290 has a factor -1/2), the scaled-time
 * acceleration uses GM = cm (central_accel uses GMS), and the physical matrix is
 * D Phi D^-1 with D = diag(1, 1, 1, sqrt(GMS) x 3) instead of its transpose.
 * ---------------------------------------------------------------------------------------- */
#define STM_DIM 42

static void stm_ivp(const double *y, double cm, double *dy) {
    double r2 = y[0] * y[0] + y[1] * y[1] + y[2] * y[2];
    double r = sqrt(r2);
    double r3 = r2 * r, r5 = r3 * r2;
    for (int i = 0; i < 3; ++i) {
        dy[i] = y[3 + i];
        dy[3 + i] = -y[i] * cm / r3;
    }
    double G[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) G[a][b] = cm * (3.0 * y[a] * y[b] - (a == b ? r2 : 0.0)) / r5;
    /* M column-major (nalgebra reshape): M(row, col) = y[6 + col * 6 + row]; dM = A M with
     * A = [[0, I], [G, 0]] */
    for (int c = 0; c < 6; ++c) {
        const double *m = y + 6 + c * 6;
        double *dm = dy + 6 + c * 6;
        for (int row = 0; row < 3; ++row) dm[row] = m[3 + row];
        for (int row = 0; row < 3; ++row) dm[3 + row] = G[row][0] * m[0] + G[row][1] * m[1] + G[row][2] * m[2];
    }
}

static double vnorm(const double *x, int n) {
    double s2 = 0.0;
    for (int i = 0; i < n; ++i) s2 += x[i] * x[i];
    return sqrt(s2);
}

/* RK45Integrator::step (runge_kutta.rs:33-113); the recursion on a rejected step becomes a
 * loop.  Returns the next step size, or 0 on failure. */
static double rk45_step(double *t, double *y, double *der, double h, double cm, double tol) {
    double k2[STM_DIM], k3[STM_DIM], k4[STM_DIM], k5[STM_DIM], k6[STM_DIM], tmp[STM_DIM],
        e[STM_DIM];
    for (int attempt = 0; attempt < 10000; ++attempt) {
        if (h != h || fabs(h) < 1e-30) return 0.0;
        for (int i = 0; i < STM_DIM; ++i) tmp[i] = y[i] + der[i] * (h / 4.0);
        stm_ivp(tmp, cm, k2);
        for (int i = 0; i < STM_DIM; ++i) k2[i] *= h;
        for (int i = 0; i < STM_DIM; ++i) tmp[i] = y[i] + der[i] * (3.0 * h / 32.0) + k2[i] * (9.0 / 32.0);
        stm_ivp(tmp, cm, k3);
        for (int i = 0; i < STM_DIM; ++i) k3[i] *= h;
        for (int i = 0; i < STM_DIM; ++i)
            tmp[i] = y[i] + der[i] * (h * 1932.0 / 2197.0) - k2[i] * (7200.0 / 2197.0) +
                     k3[i] * (7296.0 / 2197.0);
        stm_ivp(tmp, cm, k4);
        for (int i = 0; i < STM_DIM; ++i) k4[i] *= h;
        for (int i = 0; i < STM_DIM; ++i)
            tmp[i] = y[i] + der[i] * (h * 439.0 / 216.0) - k2[i] * 8.0 + k3[i] * (3680.0 / 513.0) -
                     k4[i] * (845.0 / 4104.0);
        stm_ivp(tmp, cm, k5);
        for (int i = 0; i < STM_DIM; ++i) k5[i] *= h;
        for (int i = 0; i < STM_DIM; ++i)
            tmp[i] = y[i] - der[i] * (h * 8.0 / 27.0) + k2[i] * 2.0 - k3[i] * (3544.0 / 2565.0) +
                     k4[i] * (1859.0 / 4104.0) - k5[i] * (11.0 / 40.0);
        stm_ivp(tmp, cm, k6);
        for (int i = 0; i < STM_DIM; ++i) k6[i] *= h;
        for (int i = 0; i < STM_DIM; ++i)
            e[i] = der[i] * (h / -360.0) + k3[i] * (128.0 / 4275.0) + k4[i] * (2197.0 / 75240.0) -
                   k5[i] / 50.0 - k6[i] * (2.0 / 55.0);
        double trunc_err = vnorm(e, STM_DIM);
        double new_step;
        if (trunc_err == 0.0) {
            new_step = 2.0 * h;
        } else {
            new_step = 0.9 * h * pow(tol / trunc_err, 1.0 / 5.0);
            if (trunc_err > tol) {
                h = new_step;
                continue;
            }
        }
        for (int i = 0; i < STM_DIM; ++i)
            y[i] += der[i] * (h * 16.0 / 135.0) + k3[i] * (6656.0 / 12825.0) +
                    k4[i] * (28561.0 / 56430.0) - k5[i] * (9.0 / 50.0) + k6[i] * (2.0 / 55.0);
        *t += h;
        stm_ivp(y, cm, der);
        return new_step;
    }
    return 0.0;
}

int ko_compute_stm(const double pos[3], const double vel[3], double jd0, double jd1,
                   double central_mass, double out_pos[3], double out_vel[3], double stm[36]) {
    double y[STM_DIM], der[STM_DIM];
    memset(y, 0, sizeof y);
    for (int i = 0; i < 3; ++i) {
        y[i] = pos[i];
        y[3 + i] = vel[i] / GMS_SQRT;
    }
    for (int k = 0; k < 6; ++k) y[6 + k * 6 + k] = 1.0;
    const double tol = 1e-12;
    double t = jd0 * GMS_SQRT, tf = jd1 * GMS_SQRT;
    if (fabs(t - tf) >= 1e-30) {
        stm_ivp(y, central_mass, der);
        double h = rk45_step(&t, y, der, tf - t, central_mass, tol);
        if (h == 0.0) return KO_CONVERGENCE;
        int guard = 0;
        while (fabs(t - tf) > tol) {
            if (fabs(t - tf) < fabs(h)) h = tf - t;
            h = rk45_step(&t, y, der, h, central_mass, tol);
            if (h == 0.0 || ++guard > 10000000) return KO_CONVERGENCE;
        }
    }
    for (int i = 0; i < 3; ++i) {
        out_pos[i] = y[i];
        out_vel[i] = y[3 + i] * GMS_SQRT;
    }
    /* physical matrix (row-major): D M D^-1 */
    for (int row = 0; row < 6; ++row)
        for (int c = 0; c < 6; ++c) {
            double m = y[6 + c * 6 + row];
            double da = row >= 3 ? GMS_SQRT : 1.0, db = c >= 3 ? 1.0 / GMS_SQRT : 1.0;
            stm[row * 6 + c] = da * m * db;
        }
    return KO_OK;
}

/* ------------------------------------------------------------------------------------------
 * flux (kete_core/flux/reflected.rs:23-34,255-326, common.rs:139-256, neatm.rs:19-185,
 * frm.rs:15-185,
 * shapes.rs:42-66, sun.rs:64-75, constants/wise.rs:9-85)
 * ---------------------------------------------------------------------------------------- */
static double hg_helper(double a, double b, double c, double phase) {
    double phase_s = sin(phase);
    double theta_l = exp(-a * pow(tan(0.5 * phase), b));
    double theta_s = 1.0 - c * phase_s / (0.119 + 1.341 * phase_s - 0.754 * ko_powi(phase_s, 2));
    double w = exp(-90.56 * ko_powi(tan(0.5 * phase), 2));
    return w * theta_s + (1.0 - w) * theta_l;
}

double ko_hg_phase_curve_correction(double g, double phase) {
    return (1.0 - g) * hg_helper(3.332, 0.631, 0.986, phase) + g * hg_helper(1.862, 1.218, 0.238, phase);
}

/* nalgebra Matrix::angle: acos of the clamped normalised dot product */
static double vangle(const double a[3], const double b[3]) {
    double prod = dot3(a, b);
    double n1 = norm3(a), n2 = norm3(b);
    if (n1 == 0.0 || n2 == 0.0) return 0.0;
    double cang = prod / (n1 * n2);
    return acos(clampd(cang, -1.0, 1.0));
}

double ko_hg_apparent_mag(const double sun2obj[3], const double sun2obs[3], double h_mag,
                          double g_param) {
    double obj_r = norm3(sun2obj);
    double o2o[3] = {sun2obs[0] - sun2obj[0], sun2obs[1] - sun2obj[1], sun2obs[2] - sun2obj[2]};
    double o2o_r = norm3(o2o);
    double neg[3] = {-o2o[0], -o2o[1], -o2o[2]};
    double phase = vangle(sun2obj, neg);
    if (phase > 2.792526803190927) return NAN;
    double correction = log10(ko_hg_phase_curve_correction(g_param, phase));
    return h_mag + 5.0 * log10(obj_r * o2o_r) - 2.5 * correction;
}

double ko_black_body_flux(double temp, double wavelength) {
    if (wavelength < 10.0 || temp < 30.0) return 0.0;
    double wavelength_um = wavelength * 1e-3;
    double exponent = 1.43877688e4 / (wavelength_um * temp);
    double coef = 397.289171e17 / ko_powi(wavelength_um, 3);
    return coef / (exp(exponent) - 1.0);
}

static double solar_flux_black_body(double dist, double wavelength) {
    const double SUN_R_AU = SUN_DIAMETER / AU_KM / 2.0;
    double solar_flux = ko_black_body_flux(SUN_TEMP, wavelength);
    return PI * solar_flux * ko_powi(SUN_R_AU / dist, 2);
}

double ko_hg_apparent_flux(const double sun2obj[3], const double sun2obs[3], double h_mag,
                           double g_param, double diam, double wavelength, double albedo) {
    (void)h_mag;
    double o2o[3] = {sun2obs[0] - sun2obj[0], sun2obs[1] - sun2obj[1], sun2obs[2] - sun2obj[2]};
    double neg[3] = {-o2o[0], -o2o[1], -o2o[2]};
    double phase = vangle(sun2obj, neg);
    if (phase > 2.792526803190927) return 0.0;
    double flux_at_object = solar_flux_black_body(norm3(sun2obj), wavelength);
    double object_flux_total = flux_at_object * ko_powi(diam / 2.0, 2);
    double sc2obj_r_km = norm3(o2o) * AU_KM;
    double correction = ko_hg_phase_curve_correction(g_param, phase) * albedo;
    return correction * object_flux_total / ko_powi(sc2obj_r_km, 2);
}

double ko_sub_solar_temperature(const double obj2sun[3], double geom_albedo, double g_param,
                                double beaming, double emissivity) {
    double phase_integral = 0.29 + 0.684 * g_param;
    double bond_albedo = geom_albedo * phase_integral;
    double n2 = obj2sun[0] * obj2sun[0] + obj2sun[1] * obj2sun[1] + obj2sun[2] * obj2sun[2];
    double reflected = (1.0 - bond_albedo) * SOLAR_FLUX / n2;
    double temp = reflected / (beaming * emissivity * STEFAN_BOLTZMANN);
    if (temp <= 0.0) return 0.0;
    return sqrt(sqrt(temp));
}

void ko_fib_lattice(int64_t n_facets, double *normals, double *area) {
    const double EPS = 0.36;
    double n = (double)n_facets;
    *area = 1.0 / n;
    for (int64_t idx = 0; idx < n_facets; ++idx) {
        double theta = TAU * (double)idx / GOLDEN_RATIO;
        double phi = acos(1.0 - 2.0 * ((double)idx + EPS) / (n - 1.0 + 2.0 * EPS));
        normals[3 * idx + 0] = cos(theta) * sin(phi);
        normals[3 * idx + 1] = sin(theta) * sin(phi);
        normals[3 * idx + 2] = cos(phi);
    }
}

double ko_neatm_facet_temperature(const double normal[3], const double o2s[3], double sst) {
    double tmp = dot3(normal, o2s);
    if (tmp > 0.0) return sqrt(sqrt(tmp)) * sst;
    return 0.0;
}

static double lambertian_vis_scale(const double normal[3], const double obs2obj_u[3],
                                   double obs2obj_r, double diameter, double emissivity) {
    double scale = ko_powi(obs2obj_r * AU_KM / diameter, -2);
    double observed = -dot3(normal, obs2obj_u);
    if (observed > 0.0) return observed * emissivity * PI * scale;
    return 0.0;
}

static double wise_cc(int band, double temp) {
    double t = clampd(temp, 100.0, 400.0);
    switch (band) {
    case 0:
        return 1.0 / (-3.78226591e-01 + 3.50431748e-03 * t + 1.45866307e-05 * ko_powi(t, 2) -
                      6.67674083e-08 * ko_powi(t, 3) + 7.03651986e-11 * ko_powi(t, 4));
    case 1:
        return 1.0 / (-8.60229377e-01 + 1.54988562e-02 * t - 5.10705456e-05 * ko_powi(t, 2) +
                      7.68314436e-08 * ko_powi(t, 3) - 4.32238900e-11 * ko_powi(t, 4));
    case 2:
        return 1.0 / (-1.29814355 + 2.43268763e-02 * t - 9.05178737e-05 * ko_powi(t, 2) +
                      1.50095351e-07 * ko_powi(t, 3) - 9.35433316e-11 * ko_powi(t, 4));
    default: {
        double l = log(t);
        return 2.17247804e+01 + -1.46084733e+01 * l + 3.85364000e+00 * ko_powi(l, 2) -
               4.51512551e-01 * ko_powi(l, 3) + 1.98397252e-02 * ko_powi(l, 4);
    }
    }
}

static double *g_shape = NULL;
static double g_shape_area = 0.0;

/* All lazily built tables are built once when the library loads, before any OpenMP
 * region can race on them. */
__attribute__((constructor)) static void ko_init_tables(void) {
    rot_init();
    radau_init();
    g_shape = (double *)malloc(2048 * 3 * sizeof(double));
    ko_fib_lattice(2048, g_shape, &g_shape_area);
}

/* frm.rs:19-30: cos of the latitude difference between facet and Sun direction */
double ko_frm_facet_temperature(const double normal[3], const double o2s[3], double sst) {
    double tmp = cos(asin(normal[2]) - asin(o2s[2]));
    if (tmp > 0.0) return sqrt(sqrt(tmp)) * sst;
    return 0.0;
}

/* neatm.rs:85-185 (model 0) and frm.rs:78-185 (model 1, beaming fixed to pi) share
 * everything but the facet temperature. */
static int thermal_total_flux(int model, const double sun2obj[3], const double sun2obs[3],
                              double h_mag, double g_param, double diam, double vis_albedo,
                              double beaming, double emissivity, int n_bands,
                              const double *bands, const double *band_albedos,
                              const double *sun_correction, const double *zero_mags,
                              int wise_color_correction, double *fluxes, double *hg_fluxes,
                              double *thermal, double *mags, double *v_mag, double *v_flux) {
    if (model == 1) beaming = PI;
    double obj2sun[3] = {-sun2obj[0], -sun2obj[1], -sun2obj[2]};
    double obs2obj[3] = {sun2obj[0] - sun2obs[0], sun2obj[1] - sun2obs[1], sun2obj[2] - sun2obs[2]};
    double obs2obj_r = norm3(obs2obj);
    double ss_temp = ko_sub_solar_temperature(obj2sun, vis_albedo, g_param, beaming, emissivity);
    double o2s_u[3], o2o_u[3];
    normalize3(obj2sun, o2s_u);
    normalize3(obs2obj, o2o_u);
    for (int b = 0; b < n_bands; ++b) thermal[b] = 0.0;
    for (int f = 0; f < 2048; ++f) {
        const double *nrm = g_shape + 3 * f;
        double temp = model == 1 ? ko_frm_facet_temperature(nrm, o2s_u, ss_temp)
                                 : ko_neatm_facet_temperature(nrm, o2s_u, ss_temp);
        double sc = lambertian_vis_scale(nrm, o2o_u, obs2obj_r, diam, emissivity);
        if (temp == 0.0 || sc == 0.0) continue;
        for (int b = 0; b < n_bands; ++b) {
            double ff = ko_black_body_flux(temp, bands[b]);
            if (wise_color_correction) ff *= wise_cc(b, temp);
            ff *= g_shape_area;
            thermal[b] += sc * ff;
        }
    }
    for (int b = 0; b < n_bands; ++b) {
        double refl = ko_hg_apparent_flux(sun2obj, sun2obs, h_mag, g_param, diam, bands[b],
                                          band_albedos[b]) *
                      sun_correction[b];
        hg_fluxes[b] = refl;
        fluxes[b] = thermal[b] + refl;
    }
    *v_mag = ko_hg_apparent_mag(sun2obj, sun2obs, h_mag, g_param);
    *v_flux = -2.5 * log10(*v_mag / V_MAG_ZERO); /* flux_to_mag, as neatm.rs:167 calls it */
    if (zero_mags && mags)
        for (int b = 0; b < n_bands; ++b) mags[b] = -2.5 * log10(fluxes[b] / zero_mags[b]);
    return KO_OK;
}

int ko_neatm_total_flux(const double sun2obj[3], const double sun2obs[3], double h_mag,
                        double g_param, double diam, double vis_albedo, double beaming,
                        double emissivity, int n_bands, const double *bands,
                        const double *band_albedos, const double *sun_correction,
                        const double *zero_mags, int wise_color_correction, double *fluxes,
                        double *hg_fluxes, double *thermal, double *mags, double *v_mag,
                        double *v_flux) {
    return thermal_total_flux(0, sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, beaming,
                              emissivity, n_bands, bands, band_albedos, sun_correction,
                              zero_mags, wise_color_correction, fluxes, hg_fluxes, thermal, mags,
                              v_mag, v_flux);
}

int ko_frm_total_flux(const double sun2obj[3], const double sun2obs[3], double h_mag,
                      double g_param, double diam, double vis_albedo, double emissivity,
                      int n_bands, const double *bands, const double *band_albedos,
                      const double *sun_correction, const double *zero_mags,
                      int wise_color_correction, double *fluxes, double *hg_fluxes,
                      double *thermal, double *mags, double *v_mag, double *v_flux) {
    return thermal_total_flux(1, sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, PI,
                              emissivity, n_bands, bands, band_albedos, sun_correction,
                              zero_mags, wise_color_correction, fluxes, hg_fluxes, thermal, mags,
                              v_mag, v_flux);
}

/* Many geometries of either model, (3, n) / (n_bands, n) arrays as the device entry points
 * take them, over the host's threads (models.rs:347-365 and 663-682 evaluate in parallel). */
int ko_thermal_batch(int model, int64_t n, const double *sun2obj, const double *sun2obs,
                     const double *h_mag, const double *g_param, const double *diam,
                     const double *vis_albedo, const double *beaming, const double *emissivity,
                     int n_bands, const double *bands, const double *band_albedos,
                     const double *sun_correction, const double *zero_mags,
                     int wise_color_correction, double *fluxes, double *hg_fluxes,
                     double *thermal, double *mags, double *v_mag, double *v_flux,
                     int n_threads) {
    if (n_bands < 1 || n_bands > 8) return KO_VALUE_ERROR;
#pragma omp parallel for schedule(dynamic, 64) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
    for (int64_t i = 0; i < n; ++i) {
        double so[3] = {sun2obj[i], sun2obj[n + i], sun2obj[2 * n + i]};
        double sb[3] = {sun2obs[i], sun2obs[n + i], sun2obs[2 * n + i]};
        double alb[8], fl[8], hg[8], th[8], mg[8];
        for (int b = 0; b < n_bands; ++b) alb[b] = band_albedos[(int64_t)b * n + i];
        thermal_total_flux(model, so, sb, h_mag[i], g_param[i], diam[i], vis_albedo[i],
                           model == 1 ? PI : beaming[i], emissivity[i], n_bands, bands, alb,
                           sun_correction, zero_mags, wise_color_correction, fl, hg, th, mg,
                           v_mag + i, v_flux + i);
        for (int b = 0; b < n_bands; ++b) {
            fluxes[(int64_t)b * n + i] = fl[b];
            hg_fluxes[(int64_t)b * n + i] = hg[b];
            thermal[(int64_t)b * n + i] = th[b];
            if (zero_mags && mags) mags[(int64_t)b * n + i] = mg[b];
        }
    }
    return KO_OK;
}
