"""GPU parity: the CUDA kernels through the C ABI against the CPU oracle.

Tolerances (stated per result, as the reference comparison demands):
  two-body positions 1e-12 AU, velocities 1e-14 AU/day;
  ephemeris states 5e-14 AU per AU of distance (multiply-add fusion and reciprocal
  scaling on the GPU move the Chebyshev sums by a few ulp of the ~1 AU positions);
  N-body Radau positions 1e-9 AU after one year (objects that pass within 0.01 AU of a
  planet are excluded from the bound and counted separately).
"""
import numpy as np
import pytest

from kete_b200 import synthetic

pytestmark = pytest.mark.gpu

GMS_SQRT = 0.01720209894996
TAU = 2 * np.pi
EPOCH = synthetic.EPOCH


def test_two_body_cfg0_vs_oracle(gpu, oracle):
    n = 100_000
    pos, vel = synthetic.main_belt(n, seed=11)
    rng = np.random.default_rng(12)
    jd0 = np.full(n, EPOCH)
    jd1 = EPOCH + rng.uniform(-1000, 1000, n)
    p, v, jd, st = gpu.propagate_two_body_arrays(pos, vel, jd0, jd1)
    op, ov, ojd, ost = oracle.propagate_two_body(pos, vel, jd0, jd1)
    assert (st == ost).all() and (st == 0).all()
    assert np.abs(p - op).max() < 1e-12
    assert np.abs(v - ov).max() < 1e-14
    assert (jd == jd1).all()


def test_two_body_light_delay_vs_oracle(gpu, oracle):
    n = 5000
    pos, vel = synthetic.neo(n, seed=13)
    jd0 = np.full(n, EPOCH)
    jd1 = np.full(n, EPOCH + 30.0)
    obs = np.array([0.9, -0.4, 0.0001])
    p, v, jd, st = gpu.propagate_two_body_arrays(pos, vel, jd0, jd1, obs)
    op, ov, ojd, ost = oracle.propagate_two_body(pos, vel, jd0, jd1, obs)
    assert (st == 0).all() and (ost == 0).all()
    assert np.abs(p - op).max() < 1e-12
    assert np.abs(jd - ojd).max() < 1e-9


@pytest.mark.parametrize("r", [0.2, 0.5, 1.0, 2.0])
def test_two_body_circular_golden(gpu, r):
    # kete_core/propagation/kepler.rs:416-430
    pos = np.array([[0.0, 0.0], [r, r], [0.0, 0.0]])
    vel = np.array([[-GMS_SQRT / np.sqrt(r)] * 2, [0.0, 0.0], [0.0, 0.0]])
    year = TAU / GMS_SQRT * r**1.5
    p, v, _, st = gpu.propagate_two_body_arrays(pos, vel, np.zeros(2), np.array([year, -year]))
    assert (st == 0).all()
    assert np.abs(p - pos).max() < 1e-8 and np.abs(v - vel).max() < 1e-8


def test_two_body_parabolic_hyperbolic_golden(gpu, goldens):
    par, hyp = goldens["kepler_parabolic"], goldens["kepler_hyperbolic"]
    pos = np.array([[0.0, 0.0], [2.0, 3.0], [0.0, 0.0]])
    vel = np.array([[GMS_SQRT, -GMS_SQRT], [0.0, 0.0], [0.0, 0.0]])
    jd1 = np.array([-TAU / GMS_SQRT, TAU / GMS_SQRT])
    p, v, _, st = gpu.propagate_two_body_arrays(pos, vel, np.zeros(2), jd1)
    assert (st == 0).all()
    assert np.linalg.norm(p[:, 0] - par["pos_exp"]) < 1e-8
    assert np.linalg.norm(v[:, 0] - par["vel_exp"]) < 1e-8
    assert np.linalg.norm(p[:, 1] - hyp["pos_exp"]) < 1e-8
    assert np.linalg.norm(v[:, 1] - hyp["vel_exp"]) < 1e-8


def test_two_body_edge_cases(gpu, oracle):
    pos = np.array([[1.0, np.nan, 1.0], [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]])
    vel = np.array([[0.0, 0.0, 0.0], [0.0172, 0.0172, 0.0172], [0.0, 0.0, 0.0]])
    jd0 = np.array([0.0, 0.0, 5.0])
    jd1 = np.array([10.0, 10.0, 5.0 + 1e-12])  # last one: below the 1e-10 day shortcut
    p, v, jd, st = gpu.propagate_two_body_arrays(pos, vel, jd0, jd1)
    op, ov, ojd, ost = oracle.propagate_two_body(pos, vel, jd0, jd1)
    assert st.tolist() == ost.tolist() == [0, 1, 0]
    assert np.isnan(p[:, 1]).all()
    assert (p[:, 2] == pos[:, 2]).all()
    e = gpu.propagate_two_body_arrays(np.zeros((3, 0)), np.zeros((3, 0)), np.zeros(0), np.zeros(0))
    assert e[0].shape == (3, 0)


def test_radau_central_golden(gpu, goldens):
    g = goldens["radau_basic_two_body"]  # radau.rs:356-374
    pos = np.array(g["pos0"]).reshape(3, 1)
    vel = np.array(g["vel0"]).reshape(3, 1)
    p, v, st = gpu.radau_central_arrays(pos, vel, np.zeros(1), np.array([g["t1"]]))
    assert st[0] == 0
    for which, idx, expected, tol in g["asserts"]:
        val = p[idx, 0] if which == "pos" else v[idx, 0]
        assert abs(val - expected) < tol
    assert p[2, 0] == 0.0 and v[2, 0] == 0.0


def test_spk_states_vs_oracle(gpu, oracle_spk):
    rng = np.random.default_rng(5)
    jd = rng.uniform(2457100, 2462900, 500)
    for body, center in [(10, 0), (5, 0), (399, 0), (301, 0), (3, 0), (399, 10), (5, 10), (301, 399)]:
        for frame in (1, 2):
            out6, st = gpu.spice.get_states_arrays(body, jd, center, frame)
            assert (st == 0).all()
            for k in range(0, 500, 25):
                rc, ref = oracle_spk.spk_get_state(body, jd[k], center, frame)
                assert rc == 0
                assert np.abs(out6[:3, k] - ref[:3]).max() < 1e-14
                assert np.abs(out6[3:, k] - ref[3:]).max() < 1e-15


# launch configurations: one object per thread; eight node lanes per object without a
# register cap; with a 128-register cap on a persistent grid that refills from a queue; and
# the step-end-lane forms (lane 7 supplies the exact evaluation of each accepted step); and
# the warp-synchronous forms that cache the bodies' positions across a step's iterations
CONFIGS = (dict(mode=1, variant=0, refill=0), dict(mode=2, variant=0, refill=0),
           dict(mode=2, variant=2, refill=1), dict(mode=2, variant=3, refill=1),
           dict(mode=2, variant=5, refill=0), dict(mode=2, variant=7, refill=1),
           dict(mode=2, variant=6, refill=0), dict(mode=2, variant=9, refill=1),
           dict(mode=2, variant=10, refill=0))
MODES = CONFIGS


def _set(gpu, cfg):
    from kete_b200 import tune

    tune.set_config(**cfg)
    return cfg["mode"]


def _compare_nbody(gpu, oracle, pos, vel, jd0, jd1, ng=None, frame=2, center=10, tol=1e-9):
    op, ov, ost, ons, one = oracle.propagate_n_body(pos, vel, jd0, jd1, frame, center, ng=ng)
    for cfg in CONFIGS:
        mode = _set(gpu, cfg)
        p, v, st, det = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, frame, center,
                                                    nongrav=ng, mode=mode, with_details=True)
        assert (st == ost).all(), (cfg, np.bincount(st), np.bincount(ost))
        ok = st == 0
        close = det["min_dist"] < 0.01
        far = ok & ~close
        err = np.linalg.norm(p - op, axis=0)
        if far.any():
            assert err[far].max() < tol, (cfg, err[far].max())
        # step counts agree (same adaptive sequence) for nearly all objects
        if ok.any():
            assert np.mean(det["counters"][0][ok] == ons[ok]) > 0.95, cfg
    return err, det, close


@pytest.mark.parametrize("refill", [0, 1])
def test_warp_synchronous_forms_match(gpu, refill):
    """Variants 6-8 change only when each group's next step starts and reuse the bodies'
    positions across a step's iterations; variants 9 and 10 reuse them too, with the records
    evaluated by the whole warp for whichever lanes need them.  The cached positions are rounded to doubles
    before the force terms read them, where the uncached path may fuse the last multiply
    into the difference, so results agree with the same register budget without caching to
    rounding: statuses equal, positions within the 1e-9 AU parity bar, step counts equal
    for nearly every object.  (The closest planet distance is sampled at the points the
    corrector evaluates, so it moves with the iteration count, as it does between the
    thread and node forms; it is not compared.)"""
    from kete_b200 import tune

    n = 3000
    pos, vel, ng = synthetic.mixed(n, seed=61, nongrav_frac=0.2)
    rng = np.random.default_rng(62)
    jd0 = EPOCH + rng.uniform(-30.0, 30.0, n)
    jd1 = EPOCH + rng.uniform(-400.0, 400.0, n)
    out = {}
    for variant in (3, 4, 5, 6, 7, 8, 9, 10):
        _set(gpu, dict(mode=2, variant=variant, refill=refill))
        out[variant] = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, nongrav=ng, mode=2,
                                                   with_details=True)
    tune.set_config()
    # the pooled forms (9, 10) against the uncached step-end forms of their register budgets
    for base, ws in ((3, 6), (4, 7), (5, 8), (4, 9), (5, 10)):
        p0, v0, s0, d0 = out[base]
        p1, v1, s1, d1 = out[ws]
        assert np.array_equal(s0, s1)
        ok = s0 == 0
        assert np.abs(p0[:, ok] - p1[:, ok]).max() < 1e-9
        assert np.abs(v0[:, ok] - v1[:, ok]).max() < 1e-11
        assert np.mean(d0["counters"][0][ok] == d1["counters"][0][ok]) > 0.98
        assert np.array_equal(d0["counters"][2][ok] - d0["counters"][0][ok],
                              d1["counters"][2][ok] - d1["counters"][0][ok])


def test_nbody_cfg1_vs_oracle(gpu, oracle_spk):
    """Plain N-body config: 10,000 main-belt states, +365.25 days, one target epoch."""
    n = 10_000
    pos, vel = synthetic.main_belt(n, seed=21)
    jd0 = np.full(n, EPOCH)
    jd1 = np.full(n, EPOCH + 365.25)
    err, det, close = _compare_nbody(gpu, oracle_spk, pos, vel, jd0, jd1)
    assert close.sum() == 0


def test_nbody_mixed_nongrav_vs_oracle(gpu, oracle_spk):
    n = 3000
    pos, vel, ng = synthetic.mixed(n, seed=31, nongrav_frac=0.3)
    rng = np.random.default_rng(32)
    jd0 = np.full(n, EPOCH)
    jd1 = EPOCH + rng.uniform(-365.25, 365.25, n)
    _compare_nbody(gpu, oracle_spk, pos, vel, jd0, jd1, ng=ng)


def test_nbody_dust_and_equatorial_ssb(gpu, oracle_spk):
    n = 200
    pos, vel = synthetic.main_belt(n, seed=41)
    ng = np.zeros((10, n))
    ng[0, ::2] = 2.0
    ng[1, ::2] = 0.01
    jd0 = np.full(n, EPOCH)
    jd1 = np.full(n, EPOCH + 100.0)
    _compare_nbody(gpu, oracle_spk, pos, vel, jd0, jd1, ng=ng, frame=1, center=0)


def test_nbody_edge_cases(gpu, oracle_spk):
    # NaN input, zero duration, out of SPK coverage, an impact with the Earth
    earth = oracle_spk.spk_get_state(399, EPOCH, 10, 2)[1]
    pos = np.array([[np.nan, 2.5, 2.5, earth[0] + 1e-5],
                    [0.0, 0.0, 0.0, earth[1]],
                    [0.0, 0.0, 0.0, earth[2]]])
    vel = np.array([[0.0, 0.0, 0.0, earth[3]],
                    [0.01, 0.01, 0.01, earth[4]],
                    [0.0, 0.0, 0.0, earth[5]]])
    jd0 = np.full(4, EPOCH)
    jd1 = np.array([EPOCH + 10, EPOCH, EPOCH + 5000.0, EPOCH + 10])
    op, ov, ost, _, _ = oracle_spk.propagate_n_body(pos, vel, jd0, jd1)
    for cfg in CONFIGS:
        mode = _set(gpu, cfg)
        p, v, st, det = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, mode=mode,
                                                    with_details=True)
        assert st.tolist() == ost.tolist() == [2, 0, 3, 6]
        assert det["impact_id"][3] == 399
        assert abs(det["impact_jd"][3] - EPOCH) < 1e-9
        assert np.abs(p[:, 1] - op[:, 1]).max() < 1e-15
        assert np.isnan(p[:, [0, 2, 3]]).all()


def test_nbody_backwards_and_roundtrip(gpu, oracle_spk):
    n = 500
    pos, vel = synthetic.main_belt(n, seed=51)
    jd0 = np.full(n, EPOCH)
    jd1 = np.full(n, EPOCH - 200.0)
    _compare_nbody(gpu, oracle_spk, pos, vel, jd0, jd1)
    p, v, st = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1)
    p2, v2, st2 = gpu.propagate_n_body_arrays(p, v, jd1, jd0)
    assert np.abs(p2 - pos).max() < 1e-9


def test_state_api(gpu, oracle_spk):
    """kete.propagate_n_body / propagate_two_body signatures and NaN behaviour."""
    pos, vel = synthetic.main_belt(4, seed=61)
    states = [gpu.State(f"obj{i}", EPOCH, pos[:, i], vel[:, i]) for i in range(4)]
    states.append(gpu.State("bad", EPOCH, [np.nan] * 3, [0, 0, 0]))
    out = gpu.propagate_n_body(states, EPOCH + 50.0)
    assert len(out) == 5 and not out[4].is_finite
    op, _, _, _, _ = oracle_spk.propagate_n_body(pos, vel, EPOCH, EPOCH + 50.0)
    for i in range(4):
        assert out[i].jd == EPOCH + 50.0 and out[i].desig == f"obj{i}"
        assert np.abs(out[i].pos - op[:, i]).max() < 1e-9
    with pytest.raises(ValueError):
        gpu.propagate_n_body(states, EPOCH + 50.0, suppress_errors=False)
    tb = gpu.propagate_two_body(states[:4], EPOCH + 5.0)
    kp, _, _, _ = oracle_spk.propagate_two_body(pos, vel, EPOCH, EPOCH + 5.0)
    for i in range(4):
        assert np.abs(tb[i].pos - kp[:, i]).max() < 1e-12


def test_device_arrays_torch(gpu, oracle_spk):
    torch = pytest.importorskip("torch")
    n = 256
    pos, vel = synthetic.main_belt(n, seed=71)
    jd0 = np.full(n, EPOCH)
    jd1 = np.full(n, EPOCH + 30.0)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    p, v, st = gpu.propagate_n_body_arrays(dev(pos), dev(vel), dev(jd0), dev(jd1))
    torch.cuda.synchronize()
    hp, hv, hst = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1)
    assert np.array_equal(p.cpu().numpy(), hp)


def test_autotune_installs_a_working_config(gpu, oracle_spk):
    torch = pytest.importorskip("torch")
    from kete_b200 import tune

    n = 512
    pos, vel = synthetic.main_belt(n, seed=81)
    jd0, jd1 = np.full(n, EPOCH), np.full(n, EPOCH + 20.0)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    best, times = tune.autotune(dev(pos), dev(vel), dev(jd0), dev(jd1), reps=1)
    assert len(times) == len(tune.CONFIGS) and best in tune.CONFIGS
    p, v, st = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, mode=best["mode"])
    op, _, ost, _, _ = oracle_spk.propagate_n_body(pos, vel, jd0, jd1)
    assert (st == 0).all() and np.abs(p - op).max() < 1e-9
    tune.set_config()


@pytest.fixture(scope="module")
def mixed_spk(tmp_path_factory):
    """An ephemeris with per-body coefficient counts like DE440s and the five asteroids."""
    p = tmp_path_factory.mktemp("spk_mixed") / "mixed.bsp"
    counts = {10: 11, 1: 14, 2: 10, 3: 13, 399: 13, 301: 13, 4: 11, 5: 8, 6: 7, 7: 6, 8: 6}
    synthetic.write_synthetic_spk(str(p), n_coef=counts, asteroids=True)
    return str(p)


def test_mixed_coefficients_and_asteroids_vs_oracle(gpu, oracle, mixed_spk, spk_path):
    try:
        gpu.spice.kernel_reload([mixed_spk])
        oracle.spk_reset()
        oracle.spk_load_bytes(open(mixed_spk, "rb").read())
        rng = np.random.default_rng(101)
        jd = rng.uniform(2457100, 2462900, 200)
        for body in (10, 5, 8, 399, 301, 20000001, 20000704):
            out6, st = gpu.spice.get_states_arrays(body, jd, 0, 1)
            assert (st == 0).all()
            for k in range(0, 200, 20):
                rc, ref = oracle.spk_get_state(body, jd[k], 0, 1)
                assert rc == 0
                assert np.abs(out6[:3, k] - ref[:3]).max() < 5e-14 * max(1.0, np.abs(ref[:3]).max())
        n = 600
        pos, vel = synthetic.main_belt(n, seed=102)
        jd0, jd1 = np.full(n, EPOCH), np.full(n, EPOCH + 200.0)
        for inc in (False, True):
            op, ov, ost, _, _ = oracle.propagate_n_body(pos, vel, jd0, jd1, include_extended=inc)
            for cfg in CONFIGS[:2] + CONFIGS[3:4] + CONFIGS[5:6]:
                mode = _set(gpu, cfg)
                p, v, st = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, include_asteroids=inc,
                                                       mode=mode)
                assert (st == ost).all() and (st == 0).all()
                assert np.abs(p - op).max() < 1e-9, (inc, cfg)
    finally:  # restore the session ephemeris for the tests that follow
        gpu.spice.kernel_reload([spk_path])
        oracle.spk_reset()
        oracle.spk_load_bytes(open(spk_path, "rb").read())
        from kete_b200 import tune

        tune.set_config()


def test_kernel_launch_counter(gpu):
    """kete_b200_kernel_launches counts the kernels each call enqueues."""
    import ctypes

    from kete_b200 import _lib

    count = _lib.lib().kete_b200_kernel_launches
    count.restype = ctypes.c_int64
    pos, vel = synthetic.main_belt(64, seed=91)
    jd0, jd1 = np.full(64, EPOCH), np.full(64, EPOCH + 30.0)
    c0 = count()
    gpu.propagate_two_body_arrays(pos, vel, jd0, jd1)
    c1 = count()
    gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, mode=2)
    c2 = count()
    assert c1 - c0 == 1
    # the three ordering kernels, then the node kernel (the warp-pooled forms: the centre
    # change, the pooled kernel and the change back for the objects inside the fast ephemeris
    # window, then the general form for the others)
    assert c2 - c1 in (4, 7)
