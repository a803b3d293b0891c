/*
 * kete_b200.h -- C ABI of the B200-native kete orbit-propagation hot path.
 *
 * Plain pointers and sizes only.  Arrays of vectors are structure-of-arrays FP64:
 * a "3 x n" array holds all x components, then all y, then all z.  Every entry point
 * returns 0 on success or a negative KETE_B200_E_* code, with a message available from
 * kete_b200_last_error() (per calling thread).  Per-object failures never abort a call:
 * they are reported in status[i] with the codes below, which mirror
 * kete_core::errors::Error (src/kete_core/src/errors.rs:14-32), and the object's outputs
 * are NaN -- the behaviour of the reference's suppress_errors=True path
 * (src/kete/rust/propagation.rs:113-143).
 *
 * `on_device`: 0 = the array arguments are host pointers (the call copies them to the
 * GPU and back, and returns when the results are in host memory); 1 = they are device
 * pointers on the current device (the call only enqueues work on `stream`).
 * `stream` is a cudaStream_t (NULL = the legacy default stream).
 *
 * Frames: KETE_B200_FRAME_EQUATORIAL (J2000) and KETE_B200_FRAME_ECLIPTIC (J2000 ecliptic
 * with the DE obliquity, src/kete_core/src/frames/definitions.rs:135).
 */
#ifndef KETE_B200_H
#define KETE_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* per-object status codes */
#define KETE_B200_OK 0
#define KETE_B200_CONVERGENCE 1
#define KETE_B200_VALUE_ERROR 2
#define KETE_B200_DAF_LIMITS 3
#define KETE_B200_UNKNOWN_FRAME 4
#define KETE_B200_IO_ERROR 5
#define KETE_B200_IMPACT 6
#define KETE_B200_TIMEOUT 7
#define KETE_B200_CHECKPOINT_FULL 8  /* checkpoint capacity too small; ckpt_count says how many */

/* doubles per checkpoint of kete_b200_propagate_n_body_checkpointed */
#define KETE_B200_CHECKPOINT_DOUBLES 36

/* call return codes */
#define KETE_B200_E_ARGUMENT (-1)
#define KETE_B200_E_CUDA (-2)
#define KETE_B200_E_NO_EPHEMERIS (-3)
#define KETE_B200_E_IO (-4)
#define KETE_B200_E_UNSUPPORTED (-5)

/* field-of-view table: rows per patch column, and the patch kinds of its last row */
#define KETE_B200_FOV_ROWS 20
#define KETE_B200_PATCH_RECTANGLE 0
#define KETE_B200_PATCH_CONE 1
#define KETE_B200_PATCH_OMNIDIRECTIONAL 2

#define KETE_B200_FRAME_EQUATORIAL 1
#define KETE_B200_FRAME_ECLIPTIC 2

/* propagate_n_body modes */
#define KETE_B200_MODE_AUTO 0
#define KETE_B200_MODE_THREAD 1  /* one object per thread, one launch per call */
#define KETE_B200_MODE_NODES 2   /* eight lanes per object: the 7 Gauss-Radau nodes in parallel */

/* Library version (major*10000 + minor*100 + patch). */
int kete_b200_version(void);

/* Select the CUDA device for this thread and prepare it (tables, constant memory).
 * Replaces nothing in the reference (kete has no device); called once per process. */
int kete_b200_init(int device);

/* Message of the last failed call on this thread ("" if none). */
const char* kete_b200_last_error(void);

/* --- ephemeris --------------------------------------------------------------------------
 * SpkCollection::load_file (src/kete_core/src/spice/spk.rs:307-329): parse a DAF/SPK file
 * and make its type-2 segments resident on the current device.  Segments of other types
 * are skipped and counted (kete_b200_spk_skipped). */
int kete_b200_spk_load_file(const char* path);
/* Same from an in-memory copy of the file (DafFile::from_buffer, spice/daf.rs:148-203). */
int kete_b200_spk_load_buffer(const uint8_t* bytes, int64_t n_bytes);
/* SpkCollection::reset (spk.rs:332-334). */
int kete_b200_spk_reset(void);
/* Number of segments skipped because their type is not 2. */
int kete_b200_spk_skipped(void);
/* loaded_objects(false) (spk.rs:186-205): writes up to `max` NAIF ids; returns the count. */
int kete_b200_spk_loaded_ids(int64_t* ids, int max);
/* Batched SpkCollection::try_get_state (spk.rs:87-96): state of NAIF `id` at each of the
 * n epochs `jd` relative to `center`, in `frame`.  out6 is 6 x n (pos, vel). */
int kete_b200_spk_get_states(int64_t n, int64_t id, const double* jd, int64_t center,
                             int frame, double* out6, int32_t* status, int on_device,
                             void* stream);

/* --- propagation ------------------------------------------------------------------------
 * propagate_two_body (src/kete_core/src/propagation/kepler.rs:306-322) for n Sun-centred
 * states, object i from jd0[i] to jd1[i].  With observer_pos (3 doubles, same frame) each
 * result is moved back by the light time to the observer, as the PyO3 binding does
 * (src/kete/rust/kepler.rs:89-102); out_jd then holds the delayed epochs.  out_jd may be
 * NULL. */
int kete_b200_propagate_two_body(int64_t n, const double* pos, const double* vel,
                                 const double* jd0, const double* jd1,
                                 const double* observer_pos, double* out_pos, double* out_vel,
                                 double* out_jd, int32_t* status, int on_device, void* stream);

/* propagate_n_body_spk (src/kete_core/src/propagation/mod.rs:70-118) for n states that
 * share `frame` and `center` (NAIF id), object i from jd0[i] to jd1[i], under the Sun,
 * planets and Moon of the loaded SPK (plus the five large asteroids when
 * include_asteroids != 0, mod.rs:82-88).
 *   nongrav: NULL or 10 x n rows (kind, p1..p9): kind 0 none; kind 1 JPL comet
 *            (a1 a2 a3 alpha r0 m n k dt, propagation/nongrav.rs:28-48); kind 2 dust
 *            (beta, nongrav.rs:57-60).
 *   impact_id / impact_jd: NAIF id and epoch of the body hit when status is
 *            KETE_B200_IMPACT (acceleration.rs:147-158).  May be NULL.
 *   min_dist: closest distance (AU) to any non-Sun perturber at an accepted step. May be NULL.
 *   counters: NULL or 3 x n int32 (accepted steps, corrector iterations, exact evaluations).
 *   mode: KETE_B200_MODE_*. */
int kete_b200_propagate_n_body(int64_t n, const double* pos, const double* vel,
                               const double* jd0, const double* jd1, int frame, int64_t center,
                               int include_asteroids, const double* nongrav, double* out_pos,
                               double* out_vel, int32_t* status, int32_t* impact_id,
                               double* impact_jd, double* min_dist, int32_t* counters, int mode,
                               int on_device, void* stream);

/* compute_stm / propagate_covariance (src/kete/state_transition.py:8-59, backed by
 * src/kete_core/src/propagation/state_transition.rs:52-122): the two-body state-transition
 * matrix d(pos1, vel1)/d(pos0, vel0) of n Sun-centred states from jd0 to jd1 about a central
 * body of central_mass solar masses, out_stm 6 x 6 x n (row index first, object fastest).
 * The matrix is that of kete's closed-form propagation (analytic_2_body, kepler.rs:254-297),
 * whose final states out_pos / out_vel (3 x n) match kete_b200_propagate_two_body.  kete's
 * own routine integrates the variational equations with a Jacobian off by a factor -1/2,
 * the unscaled GM in scaled time, and returns the transpose; this one returns the matrix
 * that the two-body propagation has.  With covariance (6 x 6 x n) given, out_cov receives
 * Phi covariance Phi^T (6 x 6 x n).  out_stm may be NULL.  status per object as
 * kete_b200_propagate_two_body. */
int kete_b200_compute_stm(int64_t n, const double* pos, const double* vel, const double* jd0,
                          const double* jd1, double central_mass, const double* covariance,
                          double* out_pos, double* out_vel, double* out_stm, double* out_cov,
                          int32_t* status, int on_device, void* stream);

/* out_cov = Phi C Phi^T for n objects: stm rows x cols x n, covariance cols x cols x n,
 * out_cov rows x rows x n (object index fastest; rows, cols <= 16).  With the 6 x 8
 * matrices of kete_b200_propagate_n_body_stm and an 8 x 8 covariance of (pos, vel, A1, A2)
 * it propagates an orbit's uncertainty through the N-body model. */
int kete_b200_covariance_transform(int64_t n, int rows, int cols, const double* stm,
                                   const double* covariance, double* out_cov, int on_device,
                                   void* stream);

/* propagate_n_body_spk (src/kete_core/src/propagation/mod.rs:70-118) to a sequence of epochs
 * with forward sensitivities.  Object i starts at jd0[i]; each of the n_epochs epochs
 * (shared, in the order to visit) starts a fresh integration from the previous one.  For
 * every epoch k: out_state (n_epochs x 6 x n: pos, vel in `frame`/`center`) and out_stm
 * (n_epochs x 48 x n: the 6 x 8 matrix d(pos, vel)/d(pos0, vel0, A1, A2), row-major), the
 * derivative of the executed Radau steps (step sizes held fixed) with respect to the
 * initial state and the JPL comet A1/A2 parameters (nongrav kind 1, dt = 0).  status[i]
 * reports the first failure; later epochs of a failed object are NaN. */
int kete_b200_propagate_n_body_stm(int64_t n, const double* pos, const double* vel,
                                   const double* jd0, int n_epochs, const double* epochs,
                                   int frame, int64_t center, int include_asteroids,
                                   const double* nongrav, double* out_state, double* out_stm,
                                   int32_t* status, int on_device, void* stream);

/* Reverse-mode gradients of propagate_n_body_spk (src/kete_core/src/propagation/mod.rs:70-118)
 * through a sequence of epochs, in two calls.
 *
 * kete_b200_propagate_n_body_checkpointed: the forward pass.  Same integration and outputs
 * (out_state: n_epochs x 6 x n, status: n) as kete_b200_propagate_n_body_stm without the
 * matrices.  Before every 16th step attempt of each epoch segment it stores a checkpoint
 * (KETE_B200_CHECKPOINT_DOUBLES doubles: t, h, failures, x, v, a, the Radau b and the
 * predictor's previous step) in `checkpoints` (n x ckpt_capacity x
 * KETE_B200_CHECKPOINT_DOUBLES doubles); ckpt_count (n) receives how many were taken and
 * ckpt_segment (n_epochs x n) the first checkpoint of each segment.  An object that needs
 * more than ckpt_capacity gets status KETE_B200_CHECKPOINT_FULL (its states are still
 * valid): call again with ckpt_capacity >= max(ckpt_count).  Non-gravitational models must
 * have dt = 0 (status KETE_B200_VALUE_ERROR otherwise).
 *
 * kete_b200_propagate_n_body_adjoint: the adjoint pass.  Given the forward pass's
 * checkpoints and status and seed = dL/d(out_state) (n_epochs x 6 x n), writes
 * out_grad (8 x n) = dL/d(pos0, vel0, A1, A2) in the caller's frame: the transposed
 * executed Radau steps (step sizes and iteration counts held fixed), recomputed block by
 * block from the checkpoints.  Objects whose forward status is not OK get NaN; grad_status
 * (n, may be NULL) reports failures of the adjoint pass itself.  epochs, frame,
 * include_asteroids and nongrav must be those of the forward pass. */
/* KETE_B200_CHECKPOINT_DOUBLES, for callers that cannot read the macro. */
int kete_b200_checkpoint_doubles(void);
int kete_b200_propagate_n_body_checkpointed(int64_t n, const double* pos, const double* vel,
                                            const double* jd0, int n_epochs, const double* epochs,
                                            int frame, int64_t center, int include_asteroids,
                                            const double* nongrav, double* out_state,
                                            int32_t* status, int ckpt_capacity,
                                            double* checkpoints, int32_t* ckpt_count,
                                            int32_t* ckpt_segment, int on_device, void* stream);
int kete_b200_propagate_n_body_adjoint(int64_t n, int n_epochs, const double* epochs, int frame,
                                       int include_asteroids, const double* nongrav,
                                       int ckpt_capacity, const double* checkpoints,
                                       const int32_t* ckpt_count, const int32_t* ckpt_segment,
                                       const int32_t* status, const double* seed,
                                       double* out_grad, int32_t* grad_status, int on_device,
                                       void* stream);

/* propagate_n_body_vec (src/kete_core/src/propagation/mod.rs:142-237, kete's
 * propagate_n_body_long, src/kete/rust/propagation.rs:203-249): n test particles
 * (heliocentric J2000 equatorial pos / vel 3 x n, all at jd0) integrated to jd1 together
 * with the nine massive bodies of SIMPLE_PLANETS (Sun, Mercury, Venus, Earth-Moon
 * barycentre, Mars to Neptune), in batches of batch_size particles (1 to 55) that each
 * share one integration with the massive bodies, as the reference's chunks do.  planets:
 * 9 x 6 heliocentric equatorial states at jd0 (row per body, in that order), or NULL to
 * read them from the loaded SPK.  nongrav: NULL or 10 x n rows as for
 * kete_b200_propagate_n_body; as in the reference (acceleration.rs:239-240) the first
 * particle of each batch gets no non-gravitational force.  Outputs are relative to the
 * Sun's final state; out_planets (9 x 6, may be NULL) receives the massive bodies of the
 * last batch.  status[i] is the outcome of object i's batch (an impact or a failed
 * convergence fails the whole batch). */
int kete_b200_propagate_n_body_long(int64_t n, const double* pos, const double* vel, double jd0,
                                    double jd1, const double* planets, const double* nongrav,
                                    int batch_size, double* out_pos, double* out_vel,
                                    double* out_planets, int32_t* status, int on_device,
                                    void* stream);

/* spk_accel (kete_core/propagation/acceleration.rs:121-168) at n points: the acceleration of
 * a test particle at pos/vel (3 x n, relative to the solar-system barycentre, equatorial, AU
 * and AU/day) at its own epoch jd[i] from the loaded SPK's PLANETS (or MASSES with
 * include_asteroids), with the non-gravitational row nongrav (NULL or 10 x n, as for
 * kete_b200_propagate_n_body) relative to the Sun.  exact != 0 also checks for impacts
 * (status KETE_B200_IMPACT, impact_id).  out_acc: 3 x n AU/day^2, NaN where status != 0.
 * The same force code as the propagation kernels. */
int kete_b200_spk_accel(int64_t n, const double* jd, const double* pos, const double* vel,
                        int include_asteroids, const double* nongrav, int exact, double* out_acc,
                        int32_t* status, int32_t* impact_id, int on_device, void* stream);

/* vec_accel (kete_core/propagation/acceleration.rs:197-249) on n test particles: the
 * acceleration at pos/vel (3 x n, barycentric equatorial) from massive bodies whose states
 * the caller gives, massive = 6 x m (x, y, z, vx, vy, vz rows, one column per body) in the
 * order of the chosen list (constants/gravity.rs): KETE_B200_BODIES_PLANETS (m = 10: Sun,
 * Mercury and Venus barycentres, Earth, Moon, Mars to Neptune barycentres),
 * KETE_B200_BODIES_MASSES (m = 15: PLANETS, then Ceres, Pallas, Vesta, Hygiea, Interamnia) or
 * KETE_B200_BODIES_SIMPLE_PLANETS (m = 9: Sun, Mercury, Venus, Earth-Moon, Mars to Neptune
 * barycentres; the system integration's force code).  nongrav as for kete_b200_spk_accel
 * (applied to every particle).  out_acc: 3 x n; status and impact_id as above. */
#define KETE_B200_BODIES_PLANETS 0
#define KETE_B200_BODIES_MASSES 1
#define KETE_B200_BODIES_SIMPLE_PLANETS 2
int kete_b200_vec_accel(int64_t n, int bodies, const double* massive, const double* pos,
                        const double* vel, const double* nongrav, int exact, double* out_acc,
                        int32_t* status, int32_t* impact_id, int on_device, void* stream);

/* RadauIntegrator::integrate with central_accel (propagation/mod.rs:35-46,126-138): the
 * integrator alone, for checking it against kete's closed-form two-body result. */
int kete_b200_radau_central(int64_t n, const double* pos, const double* vel, const double* t0,
                            const double* t1, double* out_pos, double* out_vel,
                            int32_t* status, int on_device, void* stream);

/* --- fields of view ----------------------------------------------------------------------
 * FovLike::check_visible (src/kete_core/src/fov/fov_like.rs:134-192) of n_obj heliocentric
 * ecliptic states (each at its own epoch jd[i]; valid: NULL or n_obj flags, 0 = skip) in
 * n_fov fields at once.  fov is KETE_B200_FOV_ROWS x n_fov, one column per sky patch:
 * observer jd, observer position[3] and velocity[3] (heliocentric ecliptic), 12 patch
 * parameters, then the patch kind: KETE_B200_PATCH_RECTANGLE (the 4 edge normals of
 * OnSkyRectangle, fov/patches.rs:122-155), KETE_B200_PATCH_CONE (unit pointing[3] and the
 * half-angle in radians of SphericalCone, patches.rs:277-337) or
 * KETE_B200_PATCH_OMNIDIRECTIONAL (always inside, fov/generic.rs:97-135).  A multi-patch
 * field (NeosVisit, ZtfField) is one column per patch.  Objects within dt_limit days of a field are
 * pre-filtered by linear motion and confirmed by two-body propagation with light delay;
 * the others by two-body then N-body propagation (include_asteroids as for
 * propagate_n_body).  Each visible (field, object) pair writes out_fov, out_obj and the
 * light-time corrected state out_state (7 x capacity: jd, pos[3], vel[3]); *n_visible is
 * the total found, which may exceed capacity (the excess is not written: call again with
 * more capacity).  Order of the pairs is unspecified. */
int kete_b200_fov_check_visible(int64_t n_obj, const double* pos, const double* vel,
                                const double* jd, const uint8_t* valid, int64_t n_fov,
                                const double* fov, double dt_limit, int include_asteroids,
                                int64_t capacity, int32_t* out_fov, int32_t* out_obj,
                                double* out_state, int64_t* n_visible, int on_device,
                                void* stream);

/* FovLike::check_statics (src/kete_core/src/fov/fov_like.rs:228-250): which of the n_fov
 * patches (fov as for kete_b200_fov_check_visible) contain each of n_vec fixed directions
 * (vec: 3 x n_vec, observer to target, ecliptic).  Each contained (patch, direction) pair
 * writes out_fov / out_idx; *n_found is the total, which may exceed capacity (the excess
 * is not written).  Order of the pairs is unspecified. */
int kete_b200_fov_contains(int64_t n_vec, const double* vec, int64_t n_fov, const double* fov,
                           int64_t capacity, int32_t* out_fov, int32_t* out_idx,
                           int64_t* n_found, int on_device, void* stream);

/* --- magnitudes ---------------------------------------------------------------------------
 * hg_apparent_mag (src/kete/rust/flux/reflected.rs:120-132, HGParams::apparent_mag
 * src/kete_core/src/flux/reflected.rs:255-268) for n geometries: sun2obj and sun2obs are
 * 3 x n (AU), h_mag and g_param n each.  Phase angles above 160 degrees give NaN. */
int kete_b200_hg_apparent_mag(int64_t n, const double* sun2obj, const double* sun2obs,
                              const double* h_mag, const double* g_param, double* out_mag,
                              int on_device, void* stream);

/* NeatmParams::apparent_total_flux (src/kete_core/src/flux/neatm.rs:143-185) for n
 * geometries, each with its own filled H-G parameters (h_mag, g_param, diam km, vis_albedo;
 * HGParams::fill, reflected.rs:177-238, is the caller's job), beaming and emissivity.  Bands
 * (1..8) share band_wavelength (nm), sun_correction and zero_mags (NULL = no magnitudes);
 * band_albedos is n_bands x n.  wise_color_correction applies the WISE W1-W4 colour
 * corrections (src/kete_core/src/constants/wise.rs:24-78; 4 bands).  Outputs n_bands x n
 * (fluxes = thermal + reflected, Jy), and v_mag / v_flux (n) as ModelResults. */
int kete_b200_neatm(int64_t n, const double* sun2obj, const double* sun2obs, const double* h_mag,
                    const double* g_param, const double* diam, const double* vis_albedo,
                    const double* beaming, const double* emissivity, int n_bands,
                    const double* band_wavelength, const double* band_albedos,
                    const double* sun_correction, const double* zero_mags,
                    int wise_color_correction, double* fluxes, double* thermal_fluxes,
                    double* hg_fluxes, double* magnitudes, double* v_mag, double* v_flux,
                    int on_device, void* stream);

/* FrmParams::apparent_total_flux (src/kete_core/src/flux/frm.rs:60-130): the fast rotating
 * model, as kete_b200_neatm but with the beaming parameter fixed to pi and facet
 * temperatures that depend on the facet's latitude only (frm_facet_temperature,
 * frm.rs:15-30). */
int kete_b200_frm(int64_t n, const double* sun2obj, const double* sun2obs, const double* h_mag,
                  const double* g_param, const double* diam, const double* vis_albedo,
                  const double* emissivity, int n_bands, const double* band_wavelength,
                  const double* band_albedos, const double* sun_correction,
                  const double* zero_mags, int wise_color_correction, double* fluxes,
                  double* thermal_fluxes, double* hg_fluxes, double* magnitudes, double* v_mag,
                  double* v_flux, int on_device, void* stream);

/* --- allocation-free variant (no counterpart in the reference) ---------------------------
 * kete_b200_propagate_n_body on the persistent lane-group grid, for callers that must not
 * have device memory allocated or freed during the call: cudaMalloc/cudaFree synchronize
 * the whole device, so steady-state loops, latency-bound services and processes whose
 * device memory belongs to another allocator cannot afford them between launches.  The
 * per-call scratch (object queue, span histogram, processing order) lives in a fixed
 * device array built into the library (KETE_B200_NOALLOC_MAX_OBJECTS * 4 + 1024 bytes,
 * held on every device that loads the library until exit); n above
 * KETE_B200_NOALLOC_MAX_OBJECTS is rejected with KETE_B200_E_ARGUMENT.
 * All array arguments are device pointers on the current device; the call only enqueues
 * work on `stream`.  The loaded SPK must already be resident on the device (load it after
 * kete_b200_init, or make one regular call first).  kete_b200_init loads the library's
 * kernels and the array on the device it prepares and looks up the array's device address,
 * so calls there load and allocate nothing; on a device it has not prepared the first call
 * does that lookup (and the lazy module load it implies), so make it before any stream
 * capture.  Calls that overlap on the GPU share the array and race, and the call reads the
 * ephemeris table and launch configuration before it enqueues: serialize it with other
 * calls, SPK loads and kete_b200_set_launch_config. */
#define KETE_B200_NOALLOC_MAX_OBJECTS 1048576
int kete_b200_propagate_n_body_noalloc(int64_t n, const double* pos, const double* vel,
                                       const double* jd0, const double* jd1, int frame,
                                       int64_t center, int include_asteroids,
                                       const double* nongrav, double* out_pos, double* out_vel,
                                       int32_t* status, int32_t* impact_id, double* impact_jd,
                                       double* min_dist, int32_t* counters, void* stream);

/* --- diagnostics (no counterpart in the reference) ------------------------------------
 * Device allocations (cudaMalloc) the library has made since it was loaded: staging
 * buffers that grow to a call's size, the ephemeris pool, facet tables, probes. */
int64_t kete_b200_device_allocations(void);

/* FP64 pipe throughput of the current device, measured with independent DFMA chains
 * (the FP64 roofline denominator).  Synchronous; ms may be NULL. */
int kete_b200_fp64_probe(int64_t iters, double* tflops, float* ms);

/* Launch configuration of the N-body kernels (no counterpart in the reference; set by the
 * autotuner).  nodes_variant: register cap of the node-parallel kernel (0 none, 1 = 168
 * registers / 3 blocks per SM, 2 = 128 / 4), plus 3 for the form whose eighth lane
 * evaluates the step end during each corrector iteration, plus 6 (with the step-end lane)
 * for the form whose lane groups start their steps together and reuse the bodies' positions
 * across a step's corrector iterations; 9 and 10 (168 / 128 registers) for the form that
 * keeps that cache but lets the four objects of a warp step independently, the whole warp
 * sharing each round's ephemeris-record evaluations (objects whose span leaves the window
 * where every perturber's first segment applies are integrated by form 7 in a second
 * launch); default 7; nodes_refill: 1 = persistent grid whose
 * lane groups take objects from a queue as they finish; thread_block: block size of the
 * one-object-per-thread kernel. */
int kete_b200_set_launch_config(int nodes_variant, int nodes_refill, int thread_block);

/* Bound on each object's Radau step loop, in step attempts, for every N-body entry point
 * (propagate_n_body, the sensitivity and adjoint passes, the FOV N-body branch and
 * propagate_n_body_long).  kete's RadauIntegrator::integrate (radau.rs:160-218) loops until
 * the target epoch is reached; on the GPU every loop is bounded so that no kernel can spin
 * without end: an object that has not arrived after max_steps attempts gets status
 * KETE_B200_TIMEOUT and a NaN state, and the kernel returns normally.  0 restores the
 * defaults (2^20 attempts per object; 2^24 per batch for system integration); at most
 * KETE_B200_STEP_LIMIT_MAX.  The sensitivity and adjoint passes bound their rounds by 12 per
 * attempt instead of counting attempts. */
#define KETE_B200_STEP_LIMIT_MAX (1 << 24)
int kete_b200_set_step_limit(int64_t max_steps);

/* Form of the N-body forward sensitivities (kete_b200_propagate_n_body_stm and the N-body
 * covariance propagation built on it; no counterpart in the reference): 0 (default) = eight
 * lanes per object, each corrector node's force Jacobian taken once per step attempt at its
 * last iteration's point; 1 = one object per thread, every iteration's Jacobian at its own
 * points.  The two agree to about 1e-8 relative. */
int kete_b200_set_sensitivity_form(int form);

/* Form of the adjoint pass's replays (kete_b200_propagate_n_body_adjoint; no counterpart in the
 * reference): 0 (default) = every checkpoint block of every object re-run in one parallel
 * launch before the sweep, when their records fit a bounded library scratch (8 GiB; else as
 * 1); 1 = the sweep re-runs each block itself, just before transposing it.  Both give the same
 * gradients bit for bit. */
int kete_b200_set_adjoint_form(int form);

/* Form of the field checks (kete_b200_fov_check_visible and the schedule built on it; no
 * counterpart in the reference): 0 (default) = a first-order linear screen of every
 * (object, field) pair, then the two-body light-time solve on the pairs that pass, one
 * thread each; 1 = both in one pass, one thread per object.  Same results. */
int kete_b200_set_fov_form(int form);

/* Number of kernels this library has enqueued since it was loaded (no counterpart in the
 * reference): read it before and after a call to count the call's GPU launches. */
int64_t kete_b200_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif
