"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline / reference arm import this module to check or time the GPU path.  The
kete_b200 package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

KO_OK, KO_CONVERGENCE, KO_VALUE_ERROR, KO_DAF_LIMITS = 0, 1, 2, 3
KO_UNKNOWN_FRAME, KO_IO_ERROR, KO_IMPACT = 4, 5, 6
FRAME_EQUATORIAL, FRAME_ECLIPTIC = 1, 2
NG_STRIDE = 10

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


def build() -> str:
    """Compile liboracle.so from oracle/kete_oracle.c with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "kete_oracle.c")
        ):
            build()
        _lib = C.CDLL(_LIB_PATH)
        L = _lib
        L.ko_newton_test.argtypes = [C.c_double, C.c_double, _dp]
        L.ko_analytic_2_body.argtypes = [C.c_double, _dp, _dp, _dp, _dp]
        L.ko_compute_eccentric_anomaly.argtypes = [C.c_double, C.c_double, C.c_double, _dp]
        L.ko_propagate_two_body_batch.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                                  _dp, _i32p, C.c_int]
        L.ko_radau_central.argtypes = [_dp, _dp, C.c_double, C.c_double, _dp, _dp]
        L.ko_spk_load_buffer.argtypes = [C.c_char_p, C.c_int64]
        L.ko_spk_get_state.argtypes = [C.c_int64, C.c_double, C.c_int64, C.c_int, _dp]
        L.ko_spk_get_states.argtypes = [C.c_int64, C.c_int64, _dp, C.c_int64, C.c_int, _dp,
                                        C.POINTER(C.c_int32), C.c_int]
        L.ko_spk_accel.argtypes = [C.c_double, _dp, _dp, C.c_int, _dp, C.c_int, _dp, _i64p]
        L.ko_vec_accel.argtypes = [C.c_int, _dp, C.c_int64, _dp, _dp, _dp, C.c_int, _dp, _i32p]
        L.ko_propagate_n_body_spk.argtypes = [_dp, _dp, C.c_double, C.c_int, C.c_int64,
                                              C.c_double, C.c_int, _dp, _dp, _dp, _i64p, _dp,
                                              _i64p, _i64p]
        L.ko_propagate_n_body_batch.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, C.c_int,
                                                C.c_int64, C.c_int, _dp, _dp, _dp, _i32p, _i64p,
                                                _i64p, C.c_int]
        L.ko_rect_from_pointing.argtypes = [_dp, C.c_double, C.c_double, C.c_double, _dp]
        L.ko_rect_contains.argtypes = [_dp, _dp, _dp]
        L.ko_fov_check_visible.argtypes = [_dp, _dp, C.c_int64, _dp, _dp, _dp, C.c_double,
                                           C.c_int, _i32p, _dp]
        L.ko_fov_check_visible_kind.argtypes = [_dp, _dp, C.c_int, C.c_int64, _dp, _dp, _dp,
                                                C.c_double, C.c_int, _i32p, _dp]
        L.ko_patch_contains.argtypes = [_dp, C.c_int, _dp, _dp]
        L.ko_propagate_n_body_vec.argtypes = [C.c_int64, _dp, _dp, C.c_double, C.c_double, _dp,
                                              _dp, C.c_int, _dp, _dp, _dp, _i32p, C.c_int]
        L.ko_hg_phase_curve_correction.argtypes = [C.c_double, C.c_double]
        L.ko_hg_phase_curve_correction.restype = C.c_double
        L.ko_hg_apparent_mag.argtypes = [_dp, _dp, C.c_double, C.c_double]
        L.ko_hg_apparent_mag.restype = C.c_double
        L.ko_hg_apparent_flux.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_double]
        L.ko_hg_apparent_flux.restype = C.c_double
        L.ko_black_body_flux.argtypes = [C.c_double, C.c_double]
        L.ko_black_body_flux.restype = C.c_double
        L.ko_sub_solar_temperature.argtypes = [_dp, C.c_double, C.c_double, C.c_double,
                                               C.c_double]
        L.ko_sub_solar_temperature.restype = C.c_double
        L.ko_fib_lattice.argtypes = [C.c_int64, _dp, _dp]
        L.ko_neatm_facet_temperature.argtypes = [_dp, _dp, C.c_double]
        L.ko_neatm_facet_temperature.restype = C.c_double
        L.ko_neatm_total_flux.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_double, C.c_int, _dp, _dp,
                                          _dp, _dp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ko_frm_facet_temperature.argtypes = [_dp, _dp, C.c_double]
        L.ko_frm_facet_temperature.restype = C.c_double
        L.ko_frm_total_flux.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_int, _dp, _dp, _dp, _dp,
                                        C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ko_thermal_batch.argtypes = [C.c_int, C.c_int64] + [_dp] * 8 + [C.c_int, _dp, _dp,
                                                                          _dp, _dp, C.c_int] + [
            _dp] * 6 + [C.c_int]
        L.ko_compute_stm.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp]
        L.ko_elements_to_pos_vel.argtypes = [C.c_double] * 7 + [_dp, _dp]
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _v3(v):
    return np.ascontiguousarray(v, dtype=np.float64).reshape(3)


def newton_test(start, atol):
    r = C.c_double()
    rc = lib().ko_newton_test(start, atol, C.byref(r))
    return rc, r.value


def analytic_2_body(dt, pos, vel):
    p, v = _v3(pos), _v3(vel)
    op, ov = np.zeros(3), np.zeros(3)
    rc = lib().ko_analytic_2_body(dt, _p(p), _p(v), _p(op), _p(ov))
    return rc, op, ov


def eccentric_anomaly(ecc, mean_anom, peri_dist):
    r = C.c_double()
    rc = lib().ko_compute_eccentric_anomaly(ecc, mean_anom, peri_dist, C.byref(r))
    return rc, r.value


def propagate_two_body(pos, vel, jd0, jd1, observer_pos=None, threads=0):
    """pos/vel: (3, n) SoA; returns out_pos, out_vel, out_jd, status."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    n = pos.shape[1]
    jd0 = np.ascontiguousarray(np.broadcast_to(jd0, (n,)), dtype=np.float64)
    jd1 = np.ascontiguousarray(np.broadcast_to(jd1, (n,)), dtype=np.float64)
    op, ov, ojd = np.zeros((3, n)), np.zeros((3, n)), np.zeros(n)
    st = np.zeros(n, dtype=np.int32)
    obs = None if observer_pos is None else _v3(observer_pos)
    lib().ko_propagate_two_body_batch(n, _p(pos), _p(vel), _p(jd0), _p(jd1), _p(obs), _p(op),
                                      _p(ov), _p(ojd), st.ctypes.data_as(_i32p), threads)
    return op, ov, ojd, st


def radau_central(pos, vel, t0, t1):
    p, v = _v3(pos), _v3(vel)
    op, ov = np.zeros(3), np.zeros(3)
    rc = lib().ko_radau_central(_p(p), _p(v), t0, t1, _p(op), _p(ov))
    return rc, op, ov


def spk_reset():
    lib().ko_spk_reset()


def spk_load_bytes(data: bytes):
    rc = lib().ko_spk_load_buffer(data, len(data))
    if rc != 0:
        raise IOError(f"oracle could not load SPK (code {rc})")


def spk_get_state(naif_id, jd, center=0, frame=FRAME_EQUATORIAL):
    out = np.zeros(6)
    rc = lib().ko_spk_get_state(naif_id, jd, center, frame, _p(out))
    return rc, out


def spk_get_states(naif_id, jd, center=0, frame=FRAME_EQUATORIAL, threads=0):
    """Batch form: jd (n,) -> out6 (6, n), status (n,) (OpenMP over the epochs)."""
    jd = np.ascontiguousarray(jd, dtype=np.float64)
    n = jd.size
    out = np.zeros((6, n))
    st = np.zeros(n, dtype=np.int32)
    lib().ko_spk_get_states(n, naif_id, _p(jd), center, frame, _p(out), st.ctypes.data_as(_i32p),
                            threads)
    return out, st


def propagate_n_body_vec(pos, vel, jd0, jd1, planets=None, ng=None, batch_size=10, threads=0):
    """propagate_n_body_vec in batches: pos/vel (3, n) heliocentric equatorial at jd0;
    planets (9, 6) or None (from the loaded SPK).  Returns out_pos, out_vel, out_planets
    (9, 6), status."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    n = pos.shape[1]
    pl = None if planets is None else np.ascontiguousarray(planets, dtype=np.float64).reshape(9, 6)
    ngp = None if ng is None else np.ascontiguousarray(ng, dtype=np.float64)
    op, ov = np.zeros((3, n)), np.zeros((3, n))
    opl = np.zeros((9, 6))
    st = np.zeros(n, dtype=np.int32)
    rc = lib().ko_propagate_n_body_vec(n, _p(pos), _p(vel), jd0, jd1, _p(pl), _p(ngp), batch_size,
                                       _p(op), _p(ov), _p(opl), st.ctypes.data_as(_i32p), threads)
    if rc != 0:
        raise ValueError(f"oracle propagate_n_body_vec failed ({rc})")
    return op, ov, opl, st


def spk_accel(t, pos, vel, include_extended=False, ng=None, exact=False):
    p, v = _v3(pos), _v3(vel)
    out = np.zeros(3)
    iid = C.c_int64(0)
    ngp = None if ng is None else np.ascontiguousarray(ng, dtype=np.float64)
    rc = lib().ko_spk_accel(t, _p(p), _p(v), int(include_extended), _p(ngp), int(exact), _p(out),
                            C.byref(iid))
    return rc, out


def vec_accel(bodies, massive, pos, vel, ng=None, exact=False):
    """vec_accel on test particles: bodies 0 PLANETS, 1 MASSES, 2 SIMPLE_PLANETS; massive
    (6, m) barycentric equatorial; pos/vel (3, n).  Returns acc (3, n), status (n,)."""
    massive = np.ascontiguousarray(massive, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    n = pos.shape[1]
    ngp = None if ng is None else np.ascontiguousarray(ng, dtype=np.float64)
    out = np.zeros((3, n))
    st = np.zeros(n, dtype=np.int32)
    lib().ko_vec_accel(int(bodies), _p(massive), n, _p(pos), _p(vel), _p(ngp), int(exact),
                       _p(out), st.ctypes.data_as(_i32p))
    return out, st


def propagate_n_body(pos, vel, jd0, jd1, frame=FRAME_ECLIPTIC, center=10,
                     include_extended=False, ng=None, threads=0):
    """Batch N-body.  pos/vel (3, n) SoA, ng (NG_STRIDE, n) or None.
    Returns out_pos, out_vel, status, n_steps, n_evals."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    n = pos.shape[1]
    jd0 = np.ascontiguousarray(np.broadcast_to(jd0, (n,)), dtype=np.float64)
    jd1 = np.ascontiguousarray(np.broadcast_to(jd1, (n,)), dtype=np.float64)
    ngp = None if ng is None else np.ascontiguousarray(ng, dtype=np.float64)
    op, ov = np.zeros((3, n)), np.zeros((3, n))
    st = np.zeros(n, dtype=np.int32)
    ns, ne = np.zeros(n, dtype=np.int64), np.zeros(n, dtype=np.int64)
    lib().ko_propagate_n_body_batch(n, _p(pos), _p(vel), _p(jd0), _p(jd1), frame, center,
                                    int(include_extended), _p(ngp), _p(op), _p(ov),
                                    st.ctypes.data_as(_i32p), ns.ctypes.data_as(_i64p),
                                    ne.ctypes.data_as(_i64p), threads)
    return op, ov, st, ns, ne


def rect_from_pointing(pointing, rotation, lon_width, lat_width):
    out = np.zeros(12)
    lib().ko_rect_from_pointing(_p(_v3(pointing)), rotation, lon_width, lat_width, _p(out))
    return out.reshape(4, 3)


def rect_contains(normals, v):
    nrm = np.ascontiguousarray(normals, dtype=np.float64).reshape(12)
    d = C.c_double()
    inside = lib().ko_rect_contains(_p(nrm), _p(_v3(v)), C.byref(d))
    return bool(inside), d.value


def patch_contains(params, kind, v):
    """One patch: kind 0 rectangle (params = 4 normals), 1 cone (pointing, half-angle),
    2 omnidirectional.  Returns (inside, distance)."""
    prm = np.zeros(12)
    a = np.asarray(params, dtype=np.float64).ravel()
    prm[:a.size] = a
    d = C.c_double()
    inside = lib().ko_patch_contains(_p(prm), int(kind), _p(_v3(v)), C.byref(d))
    return bool(inside), d.value


def fov_check_visible(obs7, normals, pos, vel, jd, dt_limit=3.0, include_extended=False, kind=0):
    obs7 = np.ascontiguousarray(obs7, dtype=np.float64)
    nrm = np.zeros(12)
    a = np.asarray(normals, dtype=np.float64).ravel()
    nrm[:a.size] = a
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    n = pos.shape[1]
    jd = np.ascontiguousarray(np.broadcast_to(jd, (n,)), dtype=np.float64)
    flags = np.zeros(n, dtype=np.int32)
    out7 = np.zeros((7, n))
    lib().ko_fov_check_visible_kind(_p(obs7), _p(nrm), int(kind), n, _p(pos), _p(vel), _p(jd),
                                    dt_limit, int(include_extended), flags.ctypes.data_as(_i32p),
                                    _p(out7))
    return flags, out7


def hg_phase_curve_correction(g, phase):
    return lib().ko_hg_phase_curve_correction(g, phase)


def hg_apparent_mag(sun2obj, sun2obs, h, g):
    return lib().ko_hg_apparent_mag(_p(_v3(sun2obj)), _p(_v3(sun2obs)), h, g)


def hg_apparent_flux(sun2obj, sun2obs, h, g, diam, wavelength, albedo):
    return lib().ko_hg_apparent_flux(_p(_v3(sun2obj)), _p(_v3(sun2obs)), h, g, diam,
                                     wavelength, albedo)


def black_body_flux(temp, wavelength):
    return lib().ko_black_body_flux(temp, wavelength)


def sub_solar_temperature(obj2sun, geom_albedo, g_param, beaming, emissivity):
    return lib().ko_sub_solar_temperature(_p(_v3(obj2sun)), geom_albedo, g_param, beaming,
                                          emissivity)


def fib_lattice(n):
    out = np.zeros(3 * n)
    area = C.c_double()
    lib().ko_fib_lattice(n, _p(out), C.byref(area))
    return out.reshape(n, 3), area.value


def neatm_facet_temperature(normal, obj2sun, sst):
    return lib().ko_neatm_facet_temperature(_p(_v3(normal)), _p(_v3(obj2sun)), sst)


def neatm_total_flux(sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, beaming, emissivity,
                     bands, band_albedos, sun_correction=None, zero_mags=None,
                     wise_color_correction=False):
    bands = np.ascontiguousarray(bands, dtype=np.float64)
    nb = bands.size
    alb = np.ascontiguousarray(band_albedos, dtype=np.float64)
    sc = np.ones(nb) if sun_correction is None else np.ascontiguousarray(sun_correction,
                                                                         dtype=np.float64)
    zm = None if zero_mags is None else np.ascontiguousarray(zero_mags, dtype=np.float64)
    fl, hg, th, mg = np.zeros(nb), np.zeros(nb), np.zeros(nb), np.zeros(nb)
    vm, vf = C.c_double(), C.c_double()
    lib().ko_neatm_total_flux(_p(_v3(sun2obj)), _p(_v3(sun2obs)), h_mag, g_param, diam,
                              vis_albedo, beaming, emissivity, nb, _p(bands), _p(alb), _p(sc),
                              _p(zm), int(wise_color_correction), _p(fl), _p(hg), _p(th),
                              _p(mg), C.byref(vm), C.byref(vf))
    return dict(fluxes=fl, hg_fluxes=hg, thermal_fluxes=th,
                magnitudes=(mg if zm is not None else None), v_band_magnitude=vm.value,
                v_band_flux=vf.value)


def frm_facet_temperature(normal, obj2sun, sst):
    """frm_facet_temperature (flux/frm.rs:19-30)."""
    return lib().ko_frm_facet_temperature(_p(_v3(normal)), _p(_v3(obj2sun)), sst)


def frm_total_flux(sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, emissivity, bands,
                   band_albedos, sun_correction=None, zero_mags=None,
                   wise_color_correction=False):
    """FrmParams::apparent_total_flux (flux/frm.rs:137-185) on the 2048-facet sphere."""
    bands = np.ascontiguousarray(bands, dtype=np.float64)
    nb = bands.size
    alb = np.ascontiguousarray(band_albedos, dtype=np.float64)
    sc = np.ones(nb) if sun_correction is None else np.ascontiguousarray(sun_correction,
                                                                         dtype=np.float64)
    zm = None if zero_mags is None else np.ascontiguousarray(zero_mags, dtype=np.float64)
    fl, hg, th, mg = np.zeros(nb), np.zeros(nb), np.zeros(nb), np.zeros(nb)
    vm, vf = C.c_double(), C.c_double()
    lib().ko_frm_total_flux(_p(_v3(sun2obj)), _p(_v3(sun2obs)), h_mag, g_param, diam,
                            vis_albedo, emissivity, nb, _p(bands), _p(alb), _p(sc), _p(zm),
                            int(wise_color_correction), _p(fl), _p(hg), _p(th), _p(mg),
                            C.byref(vm), C.byref(vf))
    return dict(fluxes=fl, hg_fluxes=hg, thermal_fluxes=th,
                magnitudes=(mg if zm is not None else None), v_band_magnitude=vm.value,
                v_band_flux=vf.value)


def thermal_batch(model, sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, beaming,
                  emissivity, bands, band_albedos, sun_correction=None, zero_mags=None,
                  wise_color_correction=False, threads=0):
    """Many geometries of NEATM (model 0) or FRM (model 1; beaming ignored) on the host's
    threads: (3, n) geometry arrays, (n,) parameters, (n_bands, n) albedos."""
    s2obj = np.ascontiguousarray(sun2obj, dtype=np.float64)
    s2obs = np.ascontiguousarray(sun2obs, dtype=np.float64)
    n = s2obj.shape[1]
    per = lambda x: np.ascontiguousarray(np.broadcast_to(np.asarray(x, np.float64), (n,)))
    bands = np.ascontiguousarray(bands, dtype=np.float64)
    nb = bands.size
    alb = np.ascontiguousarray(np.broadcast_to(np.asarray(band_albedos, np.float64).reshape(
        nb, -1), (nb, n)))
    sc = np.ones(nb) if sun_correction is None else np.ascontiguousarray(sun_correction,
                                                                         dtype=np.float64)
    zm = None if zero_mags is None else np.ascontiguousarray(zero_mags, dtype=np.float64)
    out = {k: np.zeros((nb, n)) for k in ("fluxes", "hg_fluxes", "thermal_fluxes",
                                          "magnitudes")}
    vm, vf = np.zeros(n), np.zeros(n)
    bm = per(np.pi if beaming is None else beaming)
    rc = lib().ko_thermal_batch(int(model), n, _p(s2obj), _p(s2obs), _p(per(h_mag)),
                                _p(per(g_param)), _p(per(diam)), _p(per(vis_albedo)), _p(bm),
                                _p(per(emissivity)), nb, _p(bands), _p(alb), _p(sc), _p(zm),
                                int(wise_color_correction), _p(out["fluxes"]),
                                _p(out["hg_fluxes"]), _p(out["thermal_fluxes"]),
                                _p(out["magnitudes"]), _p(vm), _p(vf), int(threads))
    if rc != 0:
        raise ValueError("ko_thermal_batch: n_bands must be 1..8")
    if zm is None:
        out["magnitudes"] = None
    out["v_band_magnitude"] = vm
    out["v_band_flux"] = vf
    return out


def compute_stm(pos, vel, jd0, jd1, central_mass=1.0):
    """Two-body state-transition matrix by the corrected variational equations on kete's
    RK4(5) Fehlberg integrator (state_transition.rs:6-122): returns (pos, vel, stm 6x6)."""
    p, v, m = np.zeros(3), np.zeros(3), np.zeros(36)
    rc = lib().ko_compute_stm(_p(_v3(pos)), _p(_v3(vel)), float(jd0), float(jd1),
                              float(central_mass), _p(p), _p(v), _p(m))
    if rc != 0:
        raise ValueError("ko_compute_stm failed")
    return p, v, m.reshape(6, 6)


def elements_to_state(epoch, ecc, incl, lon_asc, peri_time, peri_arg, peri_dist):
    p, v = np.zeros(3), np.zeros(3)
    rc = lib().ko_elements_to_pos_vel(epoch, ecc, incl, lon_asc, peri_time, peri_arg, peri_dist,
                                      _p(p), _p(v))
    return rc, p, v
