"""GPU magnitudes against the oracle and the reference's golden values.
Tolerances: magnitudes 1e-9 mag; NEATM and FRM fluxes 1e-12 relative (sums are reduced in a
different order on the GPU)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _geometries(n, seed):
    rng = np.random.default_rng(seed)
    r_obj = rng.uniform(0.8, 4.0, n)
    th = rng.uniform(0, 2 * np.pi, n)
    z = rng.normal(0, 0.2, n)
    s2obj = np.stack([r_obj * np.cos(th), r_obj * np.sin(th), z])
    th2 = rng.uniform(0, 2 * np.pi, n)
    s2obs = np.stack([np.cos(th2), np.sin(th2), np.zeros(n)])
    return s2obj, s2obs


def test_hg_mag_vs_oracle(gpu, oracle):
    s2obj, s2obs = _geometries(20000, 1)
    rng = np.random.default_rng(2)
    h = rng.uniform(12, 22, s2obj.shape[1])
    g = np.full(s2obj.shape[1], 0.15)
    out = gpu.flux.hg_apparent_mag_arrays(s2obj, s2obs, h, g)
    ref = np.array([oracle.hg_apparent_mag(s2obj[:, i], s2obs[:, i], h[i], g[i])
                    for i in range(0, s2obj.shape[1], 10)])
    got = out[::10]
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    ok = ~np.isnan(ref)
    assert np.abs(got[ok] - ref[ok]).max() < 1e-9


def test_hg_edge_cases(gpu):
    # zero phase and > 160 degree phase (NaN), reflected.rs:261-264
    m0 = gpu.flux.hg_apparent_mag([2, 0, 0], [1, 0, 0], 10.0, 0.15)
    assert abs(m0 - (10.0 + 5 * np.log10(2.0))) < 1e-12
    assert np.isnan(gpu.flux.hg_apparent_mag([1, 0, 0], [2, 0.01, 0], 10.0, 0.15))


def test_wise_neatm_golden_on_gpu(gpu, goldens):
    g = goldens["wise_neatm"]  # src/tests/flux/test_model.py:37-51
    model = gpu.flux.NeatmParams.new_wise("visible", g["band_albedos"], vis_albedo=g["vis_albedo"],
                                          g_param=g["g_param"], beaming=g["beaming"],
                                          diam=g["diam"])
    out = model.evaluate([g["sun2obj"]], [g["sun2obs"]])[0]
    np.testing.assert_allclose(out.fluxes, g["fluxes"], rtol=1e-12)


def test_neos_neatm_vs_oracle(gpu, oracle):
    s2obj, s2obs = _geometries(3000, 3)
    n = s2obj.shape[1]
    rng = np.random.default_rng(4)
    pv = np.exp(np.log(0.14) + 0.6 * rng.normal(size=n))
    h = rng.uniform(12, 22, n)
    diam = 1329.0 / np.sqrt(pv) * 10 ** (-h / 5)
    bands, zm = [4700.0, 8000.0], [170.662, 64.13]
    r = gpu.flux.neatm_arrays(s2obj, s2obs, h, 0.15, diam, pv, 1.0, 0.9, bands,
                              np.stack([pv, pv]), None, zm)
    for i in range(0, n, 30):
        o = oracle.neatm_total_flux(s2obj[:, i], s2obs[:, i], h[i], 0.15, diam[i], pv[i], 1.0, 0.9,
                                    bands, [pv[i], pv[i]], None, zm)
        np.testing.assert_allclose(r["fluxes"][:, i], o["fluxes"], rtol=1e-12)
        np.testing.assert_allclose(r["thermal_fluxes"][:, i], o["thermal_fluxes"], rtol=1e-12)
        assert np.abs(r["magnitudes"][:, i] - o["magnitudes"]).max() < 1e-9
        assert abs(r["v_band_magnitude"][i] - o["v_band_magnitude"]) < 1e-9


def test_neos_frm_model_on_gpu(gpu, oracle):
    # src/tests/flux/test_model.py:23-34, checked against the oracle as well
    model = gpu.flux.FrmParams.new_neos("visible", vis_albedo=0.3, band_albedos=[0.3, 0.3],
                                        g_param=0.15, diam=1.0)
    out = model.evaluate([[1, 1, 0]], [[0, 1, 0]])[0]
    assert model.desig == "visible"
    assert out.fluxes[0] >= 0.0 and out.fluxes[1] >= 0.0
    o = oracle.frm_total_flux([1, 1, 0], [0, 1, 0], model.h_mag, 0.15, 1.0, 0.3, 0.9,
                              [4700.0, 8000.0], [0.3, 0.3], None, [170.662, 64.13])
    np.testing.assert_allclose(out.fluxes, o["fluxes"], rtol=1e-12)
    assert np.abs(out.magnitudes - o["magnitudes"]).max() < 1e-9


def test_wise_frm_vs_oracle(gpu, oracle):
    # WISE bands with the polynomial colour corrections (constants/wise.rs:40-85)
    s2obj, s2obs = _geometries(2000, 5)
    s2obj[2] *= 3.0   # Sun directions well off the equator exercise the latitude terms
    n = s2obj.shape[1]
    rng = np.random.default_rng(6)
    pv = np.exp(np.log(0.14) + 0.6 * rng.normal(size=n))
    h = rng.uniform(8, 20, n)
    diam = 1329.0 / np.sqrt(pv) * 10 ** (-h / 5)
    bands = [3352.6, 4602.8, 11560.8 * 0.96, 22088.3 * 1.025]
    zm = [306.681, 170.663, 29.0448 * 1.08, 8.2839 * 0.96]
    sc = [1.0049, 1.0193, 1.0024, 1.0012]
    alb = np.stack([pv] * 4)
    r = gpu.flux.frm_arrays(s2obj, s2obs, h, 0.15, diam, pv, 0.9, bands, alb, sc, zm, True)
    for i in range(0, n, 25):
        o = oracle.frm_total_flux(s2obj[:, i], s2obs[:, i], h[i], 0.15, diam[i], pv[i], 0.9,
                                  bands, alb[:, i], sc, zm, wise_color_correction=True)
        np.testing.assert_allclose(r["fluxes"][:, i], o["fluxes"], rtol=1e-12)
        np.testing.assert_allclose(r["thermal_fluxes"][:, i], o["thermal_fluxes"], rtol=1e-12)
        np.testing.assert_allclose(r["hg_fluxes"][:, i], o["hg_fluxes"], rtol=1e-12)
        assert np.abs(r["magnitudes"][:, i] - o["magnitudes"]).max() < 1e-9
        assert abs(r["v_band_magnitude"][i] - o["v_band_magnitude"]) < 1e-9


def test_frm_differs_from_neatm(gpu):
    # FRM is not NEATM with another beaming: night-side facets radiate (frm.rs:19-30)
    s2obj, s2obs = _geometries(64, 7)
    kw = dict(h_mag=15.0, g_param=0.15, diam=2.0, vis_albedo=0.1, emissivity=0.9,
              band_wavelength=[12000.0], band_albedos=[0.1])
    f = gpu.flux.frm_arrays(s2obj, s2obs, **kw)
    m = gpu.flux.neatm_arrays(s2obj, s2obs, beaming=np.pi, **kw)
    assert (f["thermal_fluxes"] > 0).all()
    assert np.abs(f["thermal_fluxes"] / m["thermal_fluxes"] - 1).max() > 1e-3
    np.testing.assert_allclose(f["hg_fluxes"], m["hg_fluxes"], rtol=1e-15)


@pytest.mark.parametrize("model,bands", [("neatm", [1200.0, 3352.6, 4602.8, 11000.0, 22000.0]),
                                         ("frm", [4700.0, 8000.0, 12000.0]),
                                         ("frm", [5.0, 9000.0])])
def test_band_counts_vs_oracle(gpu, oracle, model, bands):
    # every compiled band-count form; a band below 10 nm has no thermal flux (common.rs:139-154)
    s2obj, s2obs = _geometries(300, 8)
    n, nb = s2obj.shape[1], len(bands)
    rng = np.random.default_rng(9)
    pv = np.exp(np.log(0.14) + 0.6 * rng.normal(size=n))
    h = rng.uniform(10, 20, n)
    diam = 1329.0 / np.sqrt(pv) * 10 ** (-h / 5)
    alb = np.stack([pv] * nb)
    if model == "neatm":
        r = gpu.flux.neatm_arrays(s2obj, s2obs, h, 0.15, diam, pv, 1.2, 0.9, bands, alb)
    else:
        r = gpu.flux.frm_arrays(s2obj, s2obs, h, 0.15, diam, pv, 0.9, bands, alb)
    for i in range(0, n, 7):
        if model == "neatm":
            o = oracle.neatm_total_flux(s2obj[:, i], s2obs[:, i], h[i], 0.15, diam[i], pv[i], 1.2,
                                        0.9, bands, alb[:, i])
        else:
            o = oracle.frm_total_flux(s2obj[:, i], s2obs[:, i], h[i], 0.15, diam[i], pv[i], 0.9,
                                      bands, alb[:, i])
        np.testing.assert_allclose(r["thermal_fluxes"][:, i], o["thermal_fluxes"], rtol=1e-12,
                                   atol=0.0)
        np.testing.assert_allclose(r["fluxes"][:, i], o["fluxes"], rtol=1e-12)


def test_single_band_thermal_functions(gpu, oracle):
    # kete.flux.neatm_flux / frm_flux (src/kete/rust/flux/common.rs:223-327): thermal flux
    # only, one wavelength, H from the diameter and albedo
    s2obj, s2obs = [1.5, 0.4, 0.1], [0.0, 1.0, 0.0]
    h = -5.0 * np.log10(2.0 * np.sqrt(0.1) / 1329.0)
    f = gpu.flux.neatm_flux(s2obj, s2obs, 0.1, 0.15, 1.2, 2.0, 12000.0)
    o = oracle.neatm_total_flux(s2obj, s2obs, h, 0.15, 2.0, 0.1, 1.2, 0.9, [12000.0], [0.0])
    assert abs(f / o["thermal_fluxes"][0] - 1) < 1e-12
    f = gpu.flux.frm_flux(s2obj, s2obs, 0.1, 0.15, 2.0, 12000.0)
    o = oracle.frm_total_flux(s2obj, s2obs, h, 0.15, 2.0, 0.1, 0.9, [12000.0], [0.0])
    assert abs(f / o["thermal_fluxes"][0] - 1) < 1e-12
    s2obj_n, s2obs_n = _geometries(50, 11)
    fa = gpu.flux.frm_flux(s2obj_n, s2obs_n, 0.1, 0.15, 2.0, 22000.0)
    assert fa.shape == (50,)
    for i in range(0, 50, 10):
        o = oracle.frm_total_flux(s2obj_n[:, i], s2obs_n[:, i], h, 0.15, 2.0, 0.1, 0.9,
                                  [22000.0], [0.0])
        assert abs(fa[i] / o["thermal_fluxes"][0] - 1) < 1e-12


def test_thermal_functions_three_objects_are_columns(gpu):
    """A 3 x 3 sun2obj / sun2obs is three objects, one column each (not three rows)."""
    s2obj_n, s2obs_n = _geometries(3, 17)
    for fn, args in ((gpu.flux.neatm_flux, (0.1, 0.15, 1.2, 2.0, 12000.0)),
                     (gpu.flux.frm_flux, (0.1, 0.15, 2.0, 12000.0))):
        batch = fn(np.ascontiguousarray(s2obj_n), np.ascontiguousarray(s2obs_n), *args)
        single = [fn(s2obj_n[:, i].copy(), s2obs_n[:, i].copy(), *args) for i in range(3)]
        assert batch.shape == (3,)
        assert np.allclose(batch, single, rtol=1e-14, atol=0.0)
