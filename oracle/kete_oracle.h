/*
 * kete_oracle.h -- CPU restatement of kete_core's FP64 orbit-propagation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the correctness oracle and the timed
 * CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may load it.  The product (kete_b200) never links or calls it.
 *
 * Every routine restates the reference algorithm in the reference's operation order
 * (file:line citations are relative to the kete repository root, "kete_core/" means
 * src/kete_core/src/).  It is compiled with -ffp-contract=off and without fast-math so
 * that, like the Rust build, no multiply-add is fused.
 *
 * Error codes mirror kete_core::errors::Error (kete_core/errors.rs:14-32).
 */
#ifndef KETE_ORACLE_H
#define KETE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    KO_OK = 0,
    KO_CONVERGENCE = 1,
    KO_VALUE_ERROR = 2,
    KO_DAF_LIMITS = 3,
    KO_UNKNOWN_FRAME = 4,
    KO_IO_ERROR = 5,
    KO_IMPACT = 6,
};

enum { KO_FRAME_EQUATORIAL = 1, KO_FRAME_ECLIPTIC = 2 };

/* ---- kepler / newton ------------------------------------------------------------ */
int ko_newton_test(double start, double atol, double *root);
int ko_analytic_2_body(double time, const double pos[3], const double vel[3],
                       double out_pos[3], double out_vel[3]);
int ko_compute_eccentric_anomaly(double ecc, double mean_anom, double peri_dist, double *out);
/* Batched two-body: per object jd0 -> jd1, optional light delay to observer_pos.
 * pos/vel are SoA (3 x n).  status[i] is the error code for object i. */
void ko_propagate_two_body_batch(int64_t n, const double *pos, const double *vel,
                                 const double *jd0, const double *jd1,
                                 const double *observer_pos, double *out_pos,
                                 double *out_vel, double *out_jd, int32_t *status,
                                 int n_threads);

/* ---- radau with the central (Sun only) force --------------------------------------- */
int ko_radau_central(const double pos[3], const double vel[3], double t0, double t1,
                     double out_pos[3], double out_vel[3]);

/* ---- SPK ---------------------------------------------------------------------------- */
int ko_propagate_n_body_vec(int64_t n, const double *pos, const double *vel, double jd0,
                            double jd1, const double *planets, const double *ng, int batch_size,
                            double *out_pos, double *out_vel, double *out_planets,
                            int32_t *status, int n_threads);
int ko_spk_reset(void);
int ko_spk_load_buffer(const uint8_t *bytes, int64_t n_bytes);
/* state of `id` wrt `center` in frame (KO_FRAME_*), like SpkCollection::try_get_state */
int ko_spk_get_state(int64_t id, double jd, int64_t center, int frame, double out6[6]);
int ko_spk_get_states(int64_t n, int64_t id, const double *jd, int64_t center, int frame,
                      double *out6, int32_t *status, int threads);

/* ---- N-body -------------------------------------------------------------------------- */
/* non-grav row layout (11 doubles): kind, then
 *   kind 1 (JplComet): a1 a2 a3 alpha r0 m n k dt
 *   kind 2 (Dust):     beta
 *   kind 0: none */
#define KO_NG_STRIDE 10
int ko_spk_accel(double t, const double pos[3], const double vel[3], int include_extended,
                 const double *ng, int exact, double out[3], int64_t *impact_id);
/* vec_accel for test particles under given massive bodies (0 PLANETS, 1 MASSES, 2 SIMPLE) */
int ko_vec_accel(int bodies, const double *massive, int64_t n, const double *pos,
                 const double *vel, const double *ng, int exact, double *out, int32_t *status);
int ko_propagate_n_body_spk(const double pos[3], const double vel[3], double jd0,
                            int frame, int64_t center, double jd1, int include_extended,
                            const double *ng, double out_pos[3], double out_vel[3],
                            int64_t *impact_id, double *impact_jd, int64_t *n_steps,
                            int64_t *n_evals);
void ko_propagate_n_body_batch(int64_t n, const double *pos, const double *vel,
                               const double *jd0, const double *jd1, int frame,
                               int64_t center, int include_extended, const double *ng,
                               double *out_pos, double *out_vel, int32_t *status,
                               int64_t *n_steps, int64_t *n_evals, int n_threads);

/* ---- FOV ------------------------------------------------------------------------------- */
void ko_rect_from_pointing(const double pointing[3], double rotation, double lon_width,
                           double lat_width, double normals12[12]);
/* returns 1 inside, 0 outside; *dist is Contains::Outside distance */
int ko_cone_contains(const double prm[4], const double v[3], double *dist);
int ko_patch_contains(const double prm[12], int kind, const double v[3], double *dist);
void ko_fov_check_visible_kind(const double obs7[7], const double prm[12], int kind, int64_t n,
                               const double *pos, const double *vel, const double *jd,
                               double dt_limit, int include_extended, int32_t *flags,
                               double *out7);
int ko_rect_contains(const double normals12[12], const double v[3], double *dist);
/* check_visible of one rectangle FOV for n heliocentric-ecliptic states at epoch jd[i].
 * obs7 = (jd, pos[3], vel[3]).  Writes flags[i] = 1 if visible and the light-time
 * corrected state (jd, pos, vel) into out7 (7 x n, SoA). */
void ko_fov_check_visible(const double obs7[7], const double normals12[12], int64_t n,
                          const double *pos, const double *vel, const double *jd,
                          double dt_limit, int include_extended, int32_t *flags,
                          double *out7);

/* ---- two-body state-transition matrix (corrected state_transition.rs) -------------------- */
int ko_compute_stm(const double pos[3], const double vel[3], double jd0, double jd1,
                   double central_mass, double out_pos[3], double out_vel[3], double stm[36]);

/* ---- flux -------------------------------------------------------------------------------- */
double ko_hg_phase_curve_correction(double g_param, double phase);
double ko_hg_apparent_mag(const double sun2obj[3], const double sun2obs[3], double h_mag,
                          double g_param);
double ko_black_body_flux(double temp, double wavelength);
double ko_sub_solar_temperature(const double obj2sun[3], double geom_albedo, double g_param,
                                double beaming, double emissivity);
void ko_fib_lattice(int64_t n, double *normals3n, double *area);
double ko_neatm_facet_temperature(const double normal[3], const double obj2sun_unit[3],
                                  double subsolar_temp);
/* NEATM with generic bands.  diam / vis_albedo as filled by HGParams::fill.
 * Outputs per band: fluxes, hg_fluxes, thermal, mags (if zero_mags != NULL); v_mag. */
int ko_neatm_total_flux(const double sun2obj[3], const double sun2obs[3], double h_mag,
                        double g_param, double diam, double vis_albedo, double beaming,
                        double emissivity, int n_bands, const double *bands,
                        const double *band_albedos, const double *sun_correction,
                        const double *zero_mags, int wise_color_correction,
                        double *fluxes, double *hg_fluxes, double *thermal, double *mags,
                        double *v_mag, double *v_flux);
double ko_hg_apparent_flux(const double sun2obj[3], const double sun2obs[3], double h_mag,
                           double g_param, double diam, double wavelength, double albedo);
/* FRM (frm.rs): latitude-only facet temperatures, beaming fixed to pi. */
double ko_frm_facet_temperature(const double normal[3], const double obj2sun_unit[3],
                                double subsolar_temp);
int ko_frm_total_flux(const double sun2obj[3], const double sun2obs[3], double h_mag,
                      double g_param, double diam, double vis_albedo, double emissivity,
                      int n_bands, const double *bands, const double *band_albedos,
                      const double *sun_correction, const double *zero_mags,
                      int wise_color_correction, double *fluxes, double *hg_fluxes,
                      double *thermal, double *mags, double *v_mag, double *v_flux);
/* Batched NEATM (model 0) / FRM (model 1) over OpenMP threads; (3, n) and (n_bands, n)
 * arrays; beaming may be NULL for the FRM. */
int ko_thermal_batch(int model, int64_t n, const double *sun2obj, const double *sun2obs,
                     const double *h_mag, const double *g_param, const double *diam,
                     const double *vis_albedo, const double *beaming, const double *emissivity,
                     int n_bands, const double *bands, const double *band_albedos,
                     const double *sun_correction, const double *zero_mags,
                     int wise_color_correction, double *fluxes, double *hg_fluxes,
                     double *thermal, double *mags, double *v_mag, double *v_flux,
                     int n_threads);

/* ---- elements -> state (population generation helper) -------------------------------- */
int ko_elements_to_pos_vel(double epoch, double ecc, double incl, double lon_asc,
                           double peri_time, double peri_arg, double peri_dist,
                           double pos[3], double vel[3]);

/* ---- instrumentation ---------------------------------------------------------------------- */
void ko_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
