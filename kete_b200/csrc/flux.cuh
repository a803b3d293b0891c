// flux.cuh -- H-G reflected-light magnitudes and the NEATM thermal model on the device.
//
// Restates kete_core/flux/reflected.rs:23-34 (hg_phase_curve_correction), 255-268
// (HGParams::apparent_mag), 295-326 (apparent_flux); flux/common.rs:139-154 (black_body_flux),
// 192-208 (lambertian_vis_scale_factor), 220-236 (sub_solar_temperature), 254-256
// (flux_to_mag); flux/neatm.rs:19-29, 85-185 (NEATM); flux/frm.rs:15-130 (FRM); flux/sun.rs:64-75
// (solar_flux_black_body); constants/wise.rs:24-78 (WISE colour corrections).
#pragma once
#include "common.cuh"

namespace kb {

constexpr double SUN_TEMP = 5778.0;
constexpr double SUN_DIAMETER = 1.3914e6;
constexpr double SOLAR_FLUX = 1360.8;
constexpr double STEFAN_BOLTZMANN = 5.670374419e-8;
constexpr double V_MAG_ZERO = 3597.28;
constexpr double PHASE_LIMIT = 2.792526803190927;  // 160 degrees
constexpr int N_FACETS = 2048;
constexpr int MAX_BANDS = 8;

__device__ __forceinline__ double hg_helper(double a, double b, double c, double phase) {
    const double phase_s = sin(phase);
    const double th = tan(0.5 * phase);
    const double theta_l = exp(-a * pow(th, b));
    const double theta_s = 1.0 - c * phase_s / (0.119 + 1.341 * phase_s - 0.754 * (phase_s * phase_s));
    const double w = exp(-90.56 * (th * th));
    return w * theta_s + (1.0 - w) * theta_l;
}

__device__ __forceinline__ double hg_phase_curve_correction(double g, double phase) {
    return (1.0 - g) * hg_helper(3.332, 0.631, 0.986, phase) + g * hg_helper(1.862, 1.218, 0.238, phase);
}

// nalgebra's angle(): acos of the clamped normalised dot product (0 for a zero vector)
__device__ __forceinline__ double vec_angle(const double a[3], const double b[3]) {
    const double prod = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    const double n1 = norm3(a[0], a[1], a[2]), n2 = norm3(b[0], b[1], b[2]);
    if (n1 == 0.0 || n2 == 0.0) return 0.0;
    return acos(clampd(prod / (n1 * n2), -1.0, 1.0));
}

__device__ __forceinline__ double hg_apparent_mag(const double s2obj[3], const double s2obs[3],
                                                  double h, double g) {
    const double obj_r = norm3(s2obj[0], s2obj[1], s2obj[2]);
    const double o2o[3] = {s2obs[0] - s2obj[0], s2obs[1] - s2obj[1], s2obs[2] - s2obj[2]};
    const double o2o_r = norm3(o2o[0], o2o[1], o2o[2]);
    const double neg[3] = {-o2o[0], -o2o[1], -o2o[2]};
    const double phase = vec_angle(s2obj, neg);
    if (phase > PHASE_LIMIT) return __longlong_as_double(0x7ff8000000000000LL);
    const double correction = log10(hg_phase_curve_correction(g, phase));
    return h + 5.0 * log10(obj_r * o2o_r) - 2.5 * correction;
}

__device__ __forceinline__ double black_body_flux(double temp, double wavelength) {
    if (wavelength < 10.0 || temp < 30.0) return 0.0;
    const double wl_um = wavelength * 1e-3;
    const double exponent = 1.43877688e4 / (wl_um * temp);
    const double coef = 397.289171e17 / (wl_um * (wl_um * wl_um));
    return coef / (exp(exponent) - 1.0);
}

__device__ __forceinline__ double hg_apparent_flux(const double s2obj[3], const double s2obs[3],
                                                   double g, double diam, double wavelength,
                                                   double albedo) {
    const double o2o[3] = {s2obs[0] - s2obj[0], s2obs[1] - s2obj[1], s2obs[2] - s2obj[2]};
    const double neg[3] = {-o2o[0], -o2o[1], -o2o[2]};
    const double phase = vec_angle(s2obj, neg);
    if (phase > PHASE_LIMIT) return 0.0;
    constexpr double SUN_R_AU = SUN_DIAMETER / AU_KM / 2.0;
    const double dist = norm3(s2obj[0], s2obj[1], s2obj[2]);
    const double sr = SUN_R_AU / dist;
    const double flux_at_object = PI * black_body_flux(SUN_TEMP, wavelength) * (sr * sr);
    const double hd = diam / 2.0;
    const double object_flux_total = flux_at_object * (hd * hd);
    const double sc2obj_r_km = norm3(o2o[0], o2o[1], o2o[2]) * AU_KM;
    const double correction = hg_phase_curve_correction(g, phase) * albedo;
    return correction * object_flux_total / (sc2obj_r_km * sc2obj_r_km);
}

__device__ __forceinline__ double wise_color_correction(int band, double temp) {
    const double t = clampd(temp, 100.0, 400.0);
    const double t2 = t * t, t3 = t * t2, t4 = t2 * t2;
    switch (band) {
        case 0:
            return 1.0 / (-3.78226591e-01 + 3.50431748e-03 * t + 1.45866307e-05 * t2 -
                          6.67674083e-08 * t3 + 7.03651986e-11 * t4);
        case 1:
            return 1.0 / (-8.60229377e-01 + 1.54988562e-02 * t - 5.10705456e-05 * t2 +
                          7.68314436e-08 * t3 - 4.32238900e-11 * t4);
        case 2:
            return 1.0 / (-1.29814355 + 2.43268763e-02 * t - 9.05178737e-05 * t2 +
                          1.50095351e-07 * t3 - 9.35433316e-11 * t4);
        default: {
            const double l = log(t), l2 = l * l;
            return 2.17247804e+01 + -1.46084733e+01 * l + 3.85364000e+00 * l2 -
                   4.51512551e-01 * (l * l2) + 1.98397252e-02 * (l2 * l2);
        }
    }
}

struct NeatmArgs {
    int model;  // 0 NEATM (neatm.rs), 1 FRM (frm.rs: beaming pi, latitude-only temperatures)
    int64_t n;
    const double* sun2obj;  // 3 x n
    const double* sun2obs;  // 3 x n
    const double* h_mag;
    const double* g_param;
    const double* diam;
    const double* vis_albedo;
    const double* beaming;
    const double* emissivity;
    int n_bands;
    double wavelength[MAX_BANDS];
    double sun_correction[MAX_BANDS];
    double zero_mag[MAX_BANDS];
    double bb_k[MAX_BANDS];     // black body: exponent numerator 1.43877688e4 / wavelength_um
    double bb_coef[MAX_BANDS];  // 397.289171e17 / wavelength_um^3; 0 when wavelength < 10 nm
    int have_zero_mags;
    int wise_cc;
    const double* band_albedo;  // n_bands x n
    const double* facets;       // 5 x N_FACETS: unit normals x, y, z; cos and sin of the
                                // latitude asin(z)
    double facet_area;
    double* fluxes;             // n_bands x n
    double* thermal;            // n_bands x n
    double* hg_fluxes;          // n_bands x n
    double* mags;               // n_bands x n (may be null)
    double* v_mag;              // n
    double* v_flux;             // n
};

}  // namespace kb
