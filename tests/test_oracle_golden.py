"""The CPU oracle against the reference's own known-answer tests (no GPU needed)."""
import numpy as np
import pytest

GMS_SQRT = 0.01720209894996
TAU = 2 * np.pi


def test_newton(oracle, goldens):
    rc, root = oracle.newton_test(0.0, 1e-10)  # kete_core/fitting/newton.rs:72-78
    assert rc == 0 and abs(root - goldens["newton"]["root"]) < goldens["newton"]["tol"]


@pytest.mark.parametrize("r", [0.2, 0.5, 1.0, 2.0])
def test_kepler_circular(oracle, r):
    # kete_core/propagation/kepler.rs:416-430
    pos = np.array([0.0, r, 0.0])
    vel = np.array([-GMS_SQRT / np.sqrt(r), 0.0, 0.0])
    year = TAU / GMS_SQRT * r**1.5
    for t in (year, -year):
        rc, p, v = oracle.analytic_2_body(t, pos, vel)
        assert rc == 0
        assert np.linalg.norm(p - pos) < 1e-8 and np.linalg.norm(v - vel) < 1e-8


def test_kepler_parabolic(oracle, goldens):
    g = goldens["kepler_parabolic"]  # kepler.rs:445-459
    pos, vel = np.array([0.0, 2.0, 0.0]), np.array([GMS_SQRT, 0.0, 0.0])
    year = -TAU / GMS_SQRT
    rc, p, v = oracle.analytic_2_body(year, pos, vel)
    assert rc == 0
    assert np.linalg.norm(p - g["pos_exp"]) < 1e-8 and np.linalg.norm(v - g["vel_exp"]) < 1e-8
    rc, p2, v2 = oracle.analytic_2_body(-year, np.array(g["pos_exp"]), np.array(g["vel_exp"]))
    assert np.linalg.norm(p2 - pos) < 1e-8 and np.linalg.norm(v2 - vel) < 1e-8


def test_kepler_hyperbolic(oracle, goldens):
    g = goldens["kepler_hyperbolic"]  # kepler.rs:462-476
    pos, vel = np.array([0.0, 3.0, 0.0]), np.array([-GMS_SQRT, 0.0, 0.0])
    year = TAU / GMS_SQRT
    rc, p, v = oracle.analytic_2_body(year, pos, vel)
    assert rc == 0
    assert np.linalg.norm(p - g["pos_exp"]) < 1e-8 and np.linalg.norm(v - g["vel_exp"]) < 1e-8
    rc, p2, v2 = oracle.analytic_2_body(-year, np.array(g["pos_exp"]), np.array(g["vel_exp"]))
    assert np.linalg.norm(p2 - pos) < 1e-8 and np.linalg.norm(v2 - vel) < 1e-8


def test_eccentric_anomaly_hyperbolic(oracle):
    # kepler.rs:433-442
    for m in range(-100, 100):
        rc, _ = oracle.eccentric_anomaly(2.0, float(m), 0.1)
        assert rc == 0


def test_radau_basic_two_body(oracle, goldens):
    g = goldens["radau_basic_two_body"]  # radau.rs:356-374
    rc, p, v = oracle.radau_central(g["pos0"], g["vel0"], 0.0, g["t1"])
    assert rc == 0
    for which, idx, expected, tol in g["asserts"]:
        val = p[idx] if which == "pos" else v[idx]
        assert abs(val - expected) < tol
    assert p[2] == 0.0 and v[2] == 0.0


def test_radau_matches_kepler(oracle):
    """Radau + central force against the closed-form two-body solution."""
    from kete_b200 import synthetic

    pos, vel = synthetic.main_belt(20, seed=5)
    for i in range(20):
        rc, p, v = oracle.radau_central(pos[:, i], vel[:, i], 0.0, 365.25)
        rc2, pk, vk = oracle.analytic_2_body(365.25, pos[:, i], vel[:, i])
        assert rc == 0 and rc2 == 0
        assert np.linalg.norm(p - pk) < 1e-10


def test_rectangle_patch(oracle):
    # kete_core/fov/patches.rs:367-384
    rot = np.radians(45.0)
    inside = [1.0, 0.01, 0.01]
    outside = [1.0, 0.1, 0.0]
    ji = [1.0, np.sin(0.05) * 0.99, np.sin(0.05) * 0.99]
    jo = [1.0, np.sin(0.05) * 1.01, np.sin(0.05) * 1.01]
    fov = oracle.rect_from_pointing([1, 0, 0], 0.0, 0.1, 0.1)
    fov_rot = oracle.rect_from_pointing([1, 0, 0], rot, 0.1, 0.1)
    assert oracle.rect_contains(fov, inside)[0]
    assert oracle.rect_contains(fov, ji)[0]
    assert not oracle.rect_contains(fov, outside)[0]
    assert not oracle.rect_contains(fov, jo)[0]
    assert oracle.rect_contains(fov_rot, inside)[0]
    assert not oracle.rect_contains(fov_rot, ji)[0]


def test_black_body(oracle):
    # kete_core/flux/common.rs:265-289
    wl = 20757.16266505257
    rad = oracle.black_body_flux(1000.0, wl) / 1474.49946
    assert abs(299792458.0 / rad ** (1 / 3) - wl) < 0.25
    temp = 1000.0 * np.log(2.0) / np.log(3.0)
    rad = oracle.black_body_flux(temp, wl) / 1474.49946 * 2.0
    assert abs(299792458.0 / rad ** (1 / 3) - wl) < 0.25
    assert oracle.black_body_flux(0.0, 1000.0) == 0.0
    assert oracle.black_body_flux(1000.0, 0.0) == 0.0
    assert oracle.black_body_flux(1e-5, 1e-5) == 0.0


def test_sub_solar_temperature(oracle):
    # kete_core/flux/common.rs:291-307
    assert oracle.sub_solar_temperature([1.0, 0, 0], 1.0 / 0.29, 1.0, 1.0, 1.0) == 0.0
    for r in range(1, 10):
        t = oracle.sub_solar_temperature([float(r), 0, 0], 0.0, 0.0, 1.0, 1.0) ** 4
        expected = 1360.8 / r**2 / 5.670374419e-8
        assert abs(t - expected) < 1e-5


def test_neatm_facet_temperature(oracle):
    # kete_core/flux/neatm.rs:196-251
    o2s = [1.0, 0.0, 0.0]
    t = np.cos(np.pi / 4) ** 0.25
    assert abs(oracle.neatm_facet_temperature([1, 0, 0], o2s, 1.0) - 1.0) < 1e-8
    assert abs(oracle.neatm_facet_temperature([0, 1, 0], o2s, 1.0)) < 1e-8
    assert abs(oracle.neatm_facet_temperature([-1, 0, 0], o2s, 1.0)) < 1e-8
    n = np.array([1.0, 1.0, 0.0]) / np.sqrt(2)
    assert abs(oracle.neatm_facet_temperature(n, o2s, 1.0) - t) < 1e-8
    f1, _ = oracle.fib_lattice(2048)
    f2, _ = oracle.fib_lattice(1028)
    t1 = np.mean([oracle.neatm_facet_temperature(f, o2s, 1.0) for f in f1])
    t2 = np.mean([oracle.neatm_facet_temperature(f, o2s, 1.0) for f in f2])
    assert abs(t1 - t2) < 1e-2


def test_frm_facet_temperature(oracle):
    # kete_core/flux/frm.rs:188-258
    o2s = [1.0, 0.0, 0.0]
    t = np.cos(np.pi / 4) ** 0.25
    for n in ([1, 0, 0], [0, 1, 0], [-1, 0, 0], np.array([1.0, 1.0, 0.0]) / np.sqrt(2)):
        assert abs(oracle.frm_facet_temperature(n, o2s, 1.0) - 1.0) < 1e-8
    for n in ([1.0, 0.0, 1.0], [0.0, -1.0, 1.0]):
        n = np.array(n) / np.linalg.norm(n)
        assert abs(oracle.frm_facet_temperature(n, o2s, 1.0) - t) < 1e-8
    f1, _ = oracle.fib_lattice(2048)
    f2, _ = oracle.fib_lattice(1028)
    t1 = np.mean([oracle.frm_facet_temperature(f, o2s, 1.0) for f in f1])
    t2 = np.mean([oracle.frm_facet_temperature(f, o2s, 1.0) for f in f2])
    assert abs(t1 - t2) < 1e-2


def test_neos_frm_model(oracle):
    # src/tests/flux/test_model.py:23-34: positive fluxes in both NEOS bands
    h = -5.0 * np.log10(1.0 * np.sqrt(0.3) / 1329.0)
    res = oracle.frm_total_flux([1, 1, 0], [0, 1, 0], h, 0.15, 1.0, 0.3, 0.9, [4700.0, 8000.0],
                                [0.3, 0.3], None, [170.662, 64.13])
    assert (res["fluxes"] >= 0.0).all() and (res["thermal_fluxes"] > 0.0).all()


def _frm_thermal_numpy(oracle, sun2obj, sun2obs, diam, vis_albedo, g_param, emissivity, bands):
    """Independent vectorised restatement of FrmParams::apparent_thermal_flux
    (frm.rs:78-130) with common.rs's black body, Lambertian scale and sub-solar
    temperature, used to cross-check the C oracle."""
    normals, area = oracle.fib_lattice(2048)
    sun2obj, sun2obs = np.asarray(sun2obj, float), np.asarray(sun2obs, float)
    obj2sun = -sun2obj
    obs2obj = sun2obj - sun2obs
    r_obs = np.linalg.norm(obs2obj)
    bond = vis_albedo * (0.29 + 0.684 * g_param)
    sst = ((1 - bond) * 1360.8 / obj2sun.dot(obj2sun) / (np.pi * emissivity * 5.670374419e-8)) ** 0.25
    o2s = obj2sun / np.linalg.norm(obj2sun)
    tmp = np.cos(np.arcsin(normals[:, 2]) - np.arcsin(o2s[2]))
    temp = np.where(tmp > 0, np.sqrt(np.sqrt(np.maximum(tmp, 0))) * sst, 0.0)
    seen = -normals @ (obs2obj / r_obs)
    scale = np.where(seen > 0, seen * emissivity * np.pi * (r_obs * 149597870.7 / diam) ** -2, 0.0)
    out = []
    for wl in bands:
        um = wl * 1e-3
        with np.errstate(over="ignore", divide="ignore"):
            bb = 397.289171e17 / um**3 / (np.exp(1.43877688e4 / (um * temp)) - 1.0)
        bb = np.where((temp < 30.0) | (wl < 10.0), 0.0, bb)
        out.append(np.sum(np.where((temp != 0) & (scale != 0), scale * bb * area, 0.0)))
    return np.array(out)


@pytest.mark.parametrize("z", [0.0, 0.3, -0.7])
def test_frm_thermal_vs_numpy(oracle, z):
    s2obj, s2obs = [1.2, 0.9, z], [0.0, 1.0, 0.05]
    bands = [4700.0, 8000.0, 12000.0]
    res = oracle.frm_total_flux(s2obj, s2obs, 18.0, 0.15, 0.8, 0.12, 0.9, bands, [0.1] * 3)
    ref = _frm_thermal_numpy(oracle, s2obj, s2obs, 0.8, 0.12, 0.15, 0.9, bands)
    np.testing.assert_allclose(res["thermal_fluxes"], ref, rtol=1e-11)


def test_wise_neatm_golden(oracle, goldens):
    # src/tests/flux/test_model.py:37-51 (H from diameter and albedo, reflected.rs:198-203)
    g = goldens["wise_neatm"]
    h = -5.0 * np.log10(g["diam"] * np.sqrt(g["vis_albedo"]) / 1329.0)
    res = oracle.neatm_total_flux(g["sun2obj"], g["sun2obs"], h, g["g_param"], g["diam"],
                                  g["vis_albedo"], g["beaming"], 0.9,
                                  [3352.6, 4602.8, 11560.8 * 0.96, 22088.3 * 1.025],
                                  g["band_albedos"], [1.0049, 1.0193, 1.0024, 1.0012],
                                  [306.681, 170.663, 29.0448 * 1.08, 8.2839 * 0.96],
                                  wise_color_correction=True)
    np.testing.assert_allclose(res["fluxes"], g["fluxes"], rtol=1e-12)


@pytest.mark.parametrize("obs_y", np.arange(-0.5, 1, 0.25))
@pytest.mark.parametrize("h", [5.0, 9.5, 14.5])
def test_hg_mag_flux_consistency(oracle, obs_y, h):
    # src/tests/flux/test_common.py:62-83
    albedo, g = 0.1, 0.1
    mag = oracle.hg_apparent_mag([2, 0, 0], [0, obs_y, 0], h, g)
    diam = 1329.0 / np.sqrt(albedo) * 10 ** (-h / 5)
    flux = oracle.hg_apparent_flux([2, 0, 0], [0, obs_y, 0], h, g, diam, 562.25, albedo)
    conv = -2.5 * np.log10(flux / 3620)
    assert np.isclose(mag, conv, 1e-3)


def test_hg_zero_phase(oracle):
    for g in np.arange(-0.5, 1, 0.1):
        assert np.isclose(oracle.hg_phase_curve_correction(g, 0.0), 1.0)


def test_spk_roundtrip(oracle_spk):
    """Re-reading the written SPK returns the fitted planet states."""
    from kete_b200 import synthetic

    for body in (10, 1, 2, 3, 4, 5, 6, 7, 8, 399, 301):
        jd = np.array([2458001.3, 2460000.5, 2461777.7])
        ref = synthetic.synthetic_bodies(jd)[body]
        for k, t in enumerate(jd):
            rc, s = oracle_spk.spk_get_state(body, t, center=ref[2], frame=1)
            assert rc == 0
            tol_km = 2.0 if body == 1 else 0.01  # Mercury: 32-day records on an 88-day orbit
            assert np.abs(s[:3] * synthetic.AU_KM - ref[0][:, k]).max() < tol_km


def test_spk_limits(oracle_spk):
    rc, _ = oracle_spk.spk_get_state(5, 2400000.5, 0, 1)
    assert rc == 3  # DAFLimits


def test_oracle_thread_count_does_not_change_results(oracle_spk):
    """The CPU baseline runs under OpenMP; results must not depend on the thread count."""
    from kete_b200 import synthetic

    pos, vel = synthetic.main_belt(400, seed=17)
    a = oracle_spk.propagate_n_body(pos, vel, synthetic.EPOCH, synthetic.EPOCH + 120.0, threads=1)
    b = oracle_spk.propagate_n_body(pos, vel, synthetic.EPOCH, synthetic.EPOCH + 120.0, threads=8)
    assert (a[2] == 0).all() and np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
