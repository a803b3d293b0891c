"""GPU magnitudes against the oracle and the reference's golden values.
Tolerances: magnitudes 1e-9 mag; NEATM fluxes 1e-12 relative (sums are reduced in a
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
