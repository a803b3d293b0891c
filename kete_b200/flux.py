"""kete.flux on the GPU: H-G apparent magnitudes and the NEATM and FRM thermal models.

``hg_apparent_mag`` mirrors src/kete/rust/flux/reflected.rs:120-132, ``NeatmParams``
mirrors src/kete/rust/flux/models.rs:196-365 and ``FrmParams`` models.rs:512-690
(constructors, ``evaluate``).  Parameter
filling (H, diameter, albedo; HGParams::fill, kete_core/flux/reflected.rs:177-238) is host
logic; every flux and magnitude is computed by libketeb200.so.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib

C_V = 1329.0
NEOS_BANDS = [4700.0, 8000.0]           # kete_core/constants/neos.rs:2
NEOS_ZERO_MAG = [170.662, 64.13]        # neos.rs:5
WISE_BANDS_300K = [3352.6, 4602.8, 11560.8 * 0.96, 22088.3 * 1.025]   # constants/wise.rs:9
WISE_ZERO_MAG_300K = [306.681, 170.663, 29.0448 * 1.08, 8.2839 * 0.96]  # wise.rs:16
WISE_SUN_CORRECTION = [1.0049, 1.0193, 1.0024, 1.0012]                  # wise.rs:19


def _vec3n(v):
    a = np.asarray(v, dtype=np.float64)
    if a.ndim == 1:
        a = a.reshape(3, 1)
    elif a.shape[0] != 3:
        a = a.T
    return np.ascontiguousarray(a)


def hg_apparent_mag_arrays(sun2obj, sun2obs, h_mag, g_param):
    """Batched H-G apparent magnitude: sun2obj/sun2obs (3, n) AU, h/g (n,)."""
    _lib.init()
    s2obj, s2obs = _vec3n(sun2obj), _vec3n(sun2obs)
    n = s2obj.shape[1]
    h = np.ascontiguousarray(np.broadcast_to(np.asarray(h_mag, np.float64), (n,)))
    g = np.ascontiguousarray(np.broadcast_to(np.asarray(g_param, np.float64), (n,)))
    out = np.empty(n)
    a = _lib.Args()
    args = [a.ptr(s2obj), a.ptr(s2obs), a.ptr(h), a.ptr(g), a.ptr(out)]
    L = _lib.lib()
    L.kete_b200_hg_apparent_mag.argtypes = [_lib.C.c_int64] + [_lib.C.c_void_p] * 5 + [
        _lib.C.c_int, _lib.C.c_void_p]
    _lib.check(L.kete_b200_hg_apparent_mag(n, *args, a.on_device, a.stream))
    return out


def hg_apparent_mag(sun2obj, sun2obs, h_mag, g_param) -> float:
    """kete.flux.hg_apparent_mag for one geometry (NaN above 160 degrees phase)."""
    return float(hg_apparent_mag_arrays(sun2obj, sun2obs, [h_mag], [g_param])[0])


def hg_fill(h_mag=None, vis_albedo=None, diam=None, c_hg=None):
    """HGParams::fill (kete_core/flux/reflected.rs:177-238): returns (h, albedo, diam, c_hg)."""
    if h_mag is None and (vis_albedo is None or diam is None):
        raise ValueError("h_mag must be defined unless both vis_albedo and diam are provided.")
    c_hg = C_V if c_hg is None else c_hg
    if vis_albedo is None and diam is None:
        return h_mag, None, None, c_hg
    if h_mag is None:
        return -5.0 * np.log10(diam * np.sqrt(vis_albedo) / c_hg), vis_albedo, diam, c_hg
    if vis_albedo is not None:
        expected = c_hg / np.sqrt(vis_albedo) * 10.0 ** (-0.2 * h_mag)
        if diam is not None and abs(expected - diam) > 1e-8:
            raise ValueError(f"Provided diameter doesn't match with computed diameter. "
                             f"{expected} != {diam}")
        return h_mag, vis_albedo, expected, c_hg
    alb = min(max((c_hg * 10.0 ** (-0.2 * h_mag) / diam) ** 2, 0.0), 1.0)
    return h_mag, alb, diam, c_hg


@dataclass
class ModelResults:
    """ModelResults (kete_core/flux/common.rs:82-104)."""

    fluxes: np.ndarray
    hg_fluxes: np.ndarray
    thermal_fluxes: np.ndarray
    v_band_magnitude: float
    v_band_flux: float
    magnitudes: np.ndarray | None


def _thermal_arrays(entry, sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, beaming,
                    emissivity, band_wavelength, band_albedos, sun_correction, zero_mags,
                    wise_color_correction):
    _lib.init()
    s2obj, s2obs = _vec3n(sun2obj), _vec3n(sun2obs)
    n = s2obj.shape[1]
    bands = np.ascontiguousarray(band_wavelength, dtype=np.float64)
    nb = bands.size
    per = lambda x: np.ascontiguousarray(np.broadcast_to(np.asarray(x, np.float64), (n,)))
    alb = np.ascontiguousarray(np.broadcast_to(np.asarray(band_albedos, np.float64).reshape(
        nb, -1), (nb, n)))
    sc = np.ones(nb) if sun_correction is None else np.ascontiguousarray(sun_correction,
                                                                         dtype=np.float64)
    zm = None if zero_mags is None else np.ascontiguousarray(zero_mags, dtype=np.float64)
    out = {k: np.empty((nb, n)) for k in ("fluxes", "thermal_fluxes", "hg_fluxes",
                                          "magnitudes")}
    vm, vf = np.empty(n), np.empty(n)
    a = _lib.Args()
    args = [a.ptr(s2obj), a.ptr(s2obs), a.ptr(per(h_mag)), a.ptr(per(g_param)), a.ptr(per(diam)),
            a.ptr(per(vis_albedo))]
    if beaming is not None:
        args.append(a.ptr(per(beaming)))
    args.append(a.ptr(per(emissivity)))
    L = _lib.lib()
    v = _lib.C.c_void_p
    fn = getattr(L, entry)
    fn.argtypes = [_lib.C.c_int64] + [v] * len(args) + [_lib.C.c_int, v, v, v, v,
                                                         _lib.C.c_int] + [v] * 6 + [
        _lib.C.c_int, v]
    rc = fn(n, *args, nb, bands.ctypes.data, a.ptr(alb), sc.ctypes.data,
            None if zm is None else zm.ctypes.data, int(bool(wise_color_correction)),
            a.ptr(out["fluxes"]), a.ptr(out["thermal_fluxes"]), a.ptr(out["hg_fluxes"]),
            a.ptr(out["magnitudes"]), a.ptr(vm), a.ptr(vf), a.on_device, a.stream)
    _lib.check(rc)
    if zm is None:
        out["magnitudes"] = None
    out["v_band_magnitude"] = vm
    out["v_band_flux"] = vf
    return out


def neatm_arrays(sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, beaming, emissivity,
                 band_wavelength, band_albedos, sun_correction=None, zero_mags=None,
                 wise_color_correction=False):
    """Batched NEATM: per-geometry parameters (n,), band_albedos (n_bands, n).

    Returns dict of fluxes/thermal_fluxes/hg_fluxes/magnitudes (n_bands, n) and
    v_band_magnitude/v_band_flux (n,)."""
    return _thermal_arrays("kete_b200_neatm", sun2obj, sun2obs, h_mag, g_param, diam,
                           vis_albedo, beaming, emissivity, band_wavelength, band_albedos,
                           sun_correction, zero_mags, wise_color_correction)


def frm_arrays(sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, emissivity, band_wavelength,
               band_albedos, sun_correction=None, zero_mags=None, wise_color_correction=False):
    """Batched FRM (kete_core/flux/frm.rs:78-185): as ``neatm_arrays`` without beaming."""
    return _thermal_arrays("kete_b200_frm", sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo,
                           None, emissivity, band_wavelength, band_albedos, sun_correction,
                           zero_mags, wise_color_correction)


def neatm_flux(sun2obj, sun2obs, v_albedo, g_param, beaming, diameter, wavelength,
               emissivity=0.9):
    """kete.flux.neatm_flux (src/kete/rust/flux/common.rs:223-261): NEATM thermal flux in
    Jy of one object at one wavelength (nm).  Array arguments (sun2obj/sun2obs (3, n), one
    column per object, parameters scalar or (n,)) return an (n,) array, computed on the GPU.
    An (n, 3) array with n != 3 is accepted and read one row per object; a 3 x 3 array is
    always read as three columns."""
    return _single_band_thermal("neatm", sun2obj, sun2obs, v_albedo, g_param, diameter,
                                wavelength, emissivity, beaming)


def frm_flux(sun2obj, sun2obs, v_albedo, g_param, diameter, wavelength, emissivity=0.9):
    """kete.flux.frm_flux (src/kete/rust/flux/common.rs:292-327): FRM thermal flux in Jy of
    one object at one wavelength (nm); arrays as for ``neatm_flux``."""
    return _single_band_thermal("frm", sun2obj, sun2obs, v_albedo, g_param, diameter,
                                wavelength, emissivity, None)


def _as_3n(v):
    """(3,) -> (3, 1); (3, n) as given, one column per object (a 3 x 3 array included); an
    (n, 3) array with n != 3 transposed."""
    a = np.asarray(v, dtype=np.float64)
    if a.ndim == 1:
        return a.reshape(3, 1)
    return np.ascontiguousarray(a if a.shape[0] == 3 else a.T)


def _single_band_thermal(model, sun2obj, sun2obs, v_albedo, g_param, diameter, wavelength,
                         emissivity, beaming):
    scalar = np.asarray(sun2obj).ndim == 1
    s2obj = _as_3n(sun2obj)
    n = s2obj.shape[1]
    s2obs = np.ascontiguousarray(np.broadcast_to(_as_3n(sun2obs), (3, n)))
    pv = np.broadcast_to(np.asarray(v_albedo, np.float64), (n,))
    diam = np.broadcast_to(np.asarray(diameter, np.float64), (n,))
    h = -5.0 * np.log10(diam * np.sqrt(pv) / C_V)  # HGParams::try_new with C_V (reflected.rs)
    args = (s2obj, s2obs, h, g_param, diam, pv)
    if model == "neatm":
        r = neatm_arrays(*args, beaming, emissivity, [float(wavelength)], np.zeros((1, n)))
    else:
        r = frm_arrays(*args, emissivity, [float(wavelength)], np.zeros((1, n)))
    out = r["thermal_fluxes"][0]
    return float(out[0]) if scalar else out


def _results(r, n):
    return [ModelResults(r["fluxes"][:, i], r["hg_fluxes"][:, i], r["thermal_fluxes"][:, i],
                         float(r["v_band_magnitude"][i]), float(r["v_band_flux"][i]),
                         None if r["magnitudes"] is None else r["magnitudes"][:, i])
            for i in range(n)]


def _geometries(sun2obj_vecs, sun2obs_vecs):
    s2obj = np.asarray(sun2obj_vecs, dtype=np.float64).reshape(-1, 3).T
    s2obs = np.asarray(sun2obs_vecs, dtype=np.float64).reshape(-1, 3).T
    return s2obj, s2obs, s2obj.shape[1]


class NeatmParams:
    """NEATM parameters of one object (src/kete/rust/flux/models.rs:196-225)."""

    def __init__(self, desig, band_wavelength, band_albedos, h_mag=None, diam=None,
                 vis_albedo=None, beaming=1.0, g_param=0.15, c_hg=None, emissivity=0.9,
                 zero_mags=None, sun_correction=None, wise_color_correction=False):
        self.desig = desig
        self.h_mag, self.vis_albedo, self.diam, self.c_hg = hg_fill(h_mag, vis_albedo, diam, c_hg)
        self.band_wavelength = list(band_wavelength)
        self.band_albedos = list(band_albedos)
        self.beaming, self.g_param, self.emissivity = beaming, g_param, emissivity
        self.zero_mags = None if zero_mags is None else list(zero_mags)
        self.sun_correction = ([1.0] * len(self.band_wavelength) if sun_correction is None
                               else list(sun_correction))
        self.wise_color_correction = wise_color_correction

    @staticmethod
    def new_neos(desig, band_albedos, h_mag=None, diam=None, vis_albedo=None, beaming=1.0,
                 g_param=0.15, c_hg=None, emissivity=0.9):
        return NeatmParams(desig, NEOS_BANDS, band_albedos, h_mag, diam, vis_albedo, beaming,
                           g_param, c_hg, emissivity, NEOS_ZERO_MAG)

    @staticmethod
    def new_wise(desig, band_albedos, h_mag=None, diam=None, vis_albedo=None, beaming=1.0,
                 g_param=0.15, c_hg=None, emissivity=0.9):
        if len(band_albedos) != 4:
            raise ValueError("4 Albedos must be provided, one for each WISE band.")
        return NeatmParams(desig, WISE_BANDS_300K, band_albedos, h_mag, diam, vis_albedo,
                           beaming, g_param, c_hg, emissivity, WISE_ZERO_MAG_300K,
                           WISE_SUN_CORRECTION, wise_color_correction=True)

    def evaluate(self, sun2obj_vecs, sun2obs_vecs):
        """Fluxes and magnitudes at each geometry (models.rs:347-365)."""
        if self.diam is None or self.vis_albedo is None:
            raise ValueError("NEATM needs a diameter and a visible albedo")
        s2obj, s2obs, n = _geometries(sun2obj_vecs, sun2obs_vecs)
        alb = np.repeat(np.asarray(self.band_albedos, np.float64)[:, None], n, axis=1)
        r = neatm_arrays(s2obj, s2obs, self.h_mag, self.g_param, self.diam, self.vis_albedo,
                         self.beaming, self.emissivity, self.band_wavelength, alb,
                         self.sun_correction, self.zero_mags, self.wise_color_correction)
        return _results(r, n)


class FrmParams:
    """FRM parameters of one object (src/kete/rust/flux/models.rs:512-690)."""

    def __init__(self, desig, band_wavelength, band_albedos, h_mag=None, diam=None,
                 vis_albedo=None, g_param=0.15, c_hg=None, emissivity=0.9, zero_mags=None,
                 sun_correction=None, wise_color_correction=False):
        self.desig = desig
        self.h_mag, self.vis_albedo, self.diam, self.c_hg = hg_fill(h_mag, vis_albedo, diam, c_hg)
        self.band_wavelength = list(band_wavelength)
        self.band_albedos = list(band_albedos)
        self.g_param, self.emissivity = g_param, emissivity
        self.zero_mags = None if zero_mags is None else list(zero_mags)
        self.sun_correction = ([1.0] * len(self.band_wavelength) if sun_correction is None
                               else list(sun_correction))
        self.wise_color_correction = wise_color_correction

    @staticmethod
    def new_neos(desig, band_albedos, h_mag=None, diam=None, vis_albedo=None, g_param=0.15,
                 c_hg=None, emissivity=0.9):
        if len(band_albedos) != 2:
            raise ValueError("2 Albedos must be provided, one for each NEOS band.")
        return FrmParams(desig, NEOS_BANDS, band_albedos, h_mag, diam, vis_albedo, g_param,
                         c_hg, emissivity, NEOS_ZERO_MAG)

    @staticmethod
    def new_wise(desig, band_albedos, h_mag=None, diam=None, vis_albedo=None, g_param=0.15,
                 c_hg=None, emissivity=0.9):
        if len(band_albedos) != 4:
            raise ValueError("4 Albedos must be provided, one for each WISE band.")
        return FrmParams(desig, WISE_BANDS_300K, band_albedos, h_mag, diam, vis_albedo, g_param,
                         c_hg, emissivity, WISE_ZERO_MAG_300K, WISE_SUN_CORRECTION,
                         wise_color_correction=True)

    def evaluate(self, sun2obj_vecs, sun2obs_vecs):
        """Fluxes and magnitudes at each geometry (models.rs:663-682)."""
        if self.diam is None or self.vis_albedo is None:
            raise ValueError("FRM needs a diameter and a visible albedo")
        s2obj, s2obs, n = _geometries(sun2obj_vecs, sun2obs_vecs)
        alb = np.repeat(np.asarray(self.band_albedos, np.float64)[:, None], n, axis=1)
        r = frm_arrays(s2obj, s2obs, self.h_mag, self.g_param, self.diam, self.vis_albedo,
                       self.emissivity, self.band_wavelength, alb, self.sun_correction,
                       self.zero_mags, self.wise_color_correction)
        return _results(r, n)
