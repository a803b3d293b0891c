"""GPU side of the reference tests that need an SPK (see test_oracle_pins.py), and the batched
accelerations against the oracle.

- spk_accel on the GPU (the propagation kernels' force code, C ABI kete_b200_spk_accel)
  equals the oracle's restatement of acceleration.rs:121-168 at scattered points and epochs,
  with and without the comet model, to 1e-13 relative (FMA contraction and the reordered
  record sums are the only differences).
- check_accelerations_equal (acceleration.rs:298-347) on the GPU: vec_accel under the MASSES
  bodies' states read back from the device SPK equals spk_accel to 1e-10 AU/day^2; the system
  integration's pair term (SIMPLE_PLANETS, Earth-Moon barycentre) equals spk_accel with the
  PLANETS list to 1e-10 AU/day^2 too.
- test_check_rectangle_visible (kete_core/fov/generic.rs:199-235) through the batched field
  check: visible for offsets -10..10 days, both light-time branches, and the light-time
  identity (observer epoch - state epoch = distance / c to 1e-6 day).
"""
import numpy as np
import pytest

from kete_b200 import fov as fovmod
from kete_b200 import synthetic

pytestmark = pytest.mark.gpu

EPOCH = synthetic.EPOCH
MASSES = (10, 1, 2, 399, 301, 4, 5, 6, 7, 8, 20000001, 20000002, 20000004, 20000010, 20000704)
SIMPLE = (10, 1, 2, 3, 4, 5, 6, 7, 8)
GMS_SQRT = 0.01720209894996
C_AU_PER_DAY = 173.14463267424034


@pytest.fixture(scope="module")
def masses_spk(gpu, oracle, tmp_path_factory, spk_path):
    """GPU and oracle with the synthetic SPK that also holds MASSES' five asteroids; the
    session's planets-only SPK is restored afterwards."""
    p = str(tmp_path_factory.mktemp("spk_masses") / "masses.bsp")
    synthetic.write_synthetic_spk(p, asteroids=True)
    gpu.spice.kernel_reload([p])
    oracle.spk_reset()
    oracle.spk_load_bytes(open(p, "rb").read())
    yield gpu, oracle
    gpu.spice.kernel_reload([spk_path])
    oracle.spk_reset()
    oracle.spk_load_bytes(open(spk_path, "rb").read())


def _massive(gpu, ids, jd):
    cols = []
    for i in ids:
        out6, st = gpu.spice.get_states_arrays(i, np.array([jd]), 0, 1)
        assert (st == 0).all()
        cols.append(out6[:, 0])
    return np.ascontiguousarray(np.stack(cols, axis=1))


def test_spk_accel_vs_oracle(masses_spk):
    gpu, oracle = masses_spk
    n = 400
    rng = np.random.default_rng(5)
    jd = rng.uniform(2457200.0, 2462800.0, n)
    pos = rng.uniform(-4.0, 4.0, (3, n))
    vel = rng.uniform(-0.02, 0.02, (3, n))
    ng = np.zeros((10, n))
    ng[:, ::3] = synthetic.comet_nongrav(3e-8, -2e-9, 1e-10)[:, None]
    for inc in (False, True):
        for use_ng in (False, True):
            acc, st, _ = gpu.spk_accel_arrays(jd, pos, vel, include_asteroids=inc,
                                              nongrav=ng if use_ng else None)
            assert (st == 0).all()
            for k in range(0, n, 7):
                rc, ref = oracle.spk_accel(jd[k], pos[:, k], vel[:, k], include_extended=inc,
                                           ng=ng[:, k] if use_ng else None)
                assert rc == 0
                assert np.abs(acc[:, k] - ref).max() <= 1e-13 * np.abs(ref).max(), (inc, use_ng, k)


def test_spk_accel_impact_status(masses_spk):
    gpu, oracle = masses_spk
    earth = _massive(gpu, (399,), EPOCH)[:, 0]
    pos = np.array([[earth[0] + 1e-5, 2.0], [earth[1], 0.0], [earth[2], 0.0]])
    vel = np.zeros((3, 2))
    jd = np.full(2, EPOCH)
    acc, st, iid = gpu.spk_accel_arrays(jd, pos, vel, exact=True)
    assert st.tolist() == [6, 0] and iid[0] == 399 and np.isnan(acc[:, 0]).all()
    acc, st, _ = gpu.spk_accel_arrays(jd, pos, vel, exact=False)
    assert (st == 0).all()


@pytest.mark.parametrize("jd", [EPOCH, EPOCH - 1234.5, EPOCH + 2000.25])
def test_check_accelerations_equal(masses_spk, jd):
    gpu, oracle = masses_spk
    massive = _massive(gpu, MASSES, jd)
    pos, vel = np.array([[0.0], [0.0], [0.5]]), np.array([[0.0], [0.0], [1.0]])
    acc, st, _ = gpu.vec_accel_arrays(massive, pos, vel, bodies="masses")
    acc2, st2, _ = gpu.spk_accel_arrays(np.array([jd]), pos, vel, include_asteroids=True)
    assert st[0] == 0 and st2[0] == 0
    assert np.abs(acc - acc2).max() < 1e-10
    oacc, ost = oracle.vec_accel(1, massive, pos, vel)
    assert np.abs(acc - oacc).max() <= 1e-13 * np.abs(oacc).max()
    # the system integration's force code against the propagation kernels', and PLANETS
    rng = np.random.default_rng(int(jd) % 1000)
    pos = rng.uniform(-3.0, 3.0, (3, 64))
    vel = rng.uniform(-0.02, 0.02, (3, 64))
    jds = np.full(64, jd)
    ref, st, _ = gpu.spk_accel_arrays(jds, pos, vel)
    assert (st == 0).all()
    simple, st, _ = gpu.vec_accel_arrays(_massive(gpu, SIMPLE, jd), pos, vel,
                                         bodies="simple_planets")
    assert (st == 0).all() and np.abs(simple - ref).max() < 1e-10
    planets, st, _ = gpu.vec_accel_arrays(massive[:, :10].copy(), pos, vel, bodies="planets")
    assert (st == 0).all() and np.abs(planets - ref).max() < 1e-10
    osimple, _ = oracle.vec_accel(2, _massive(gpu, SIMPLE, jd), pos, vel)
    assert np.abs(simple - osimple).max() <= 1e-13 * np.abs(osimple).max()


@pytest.mark.parametrize("offset", [-10.0, -5.0, 0.0, 5.0, 10.0])
def test_check_rectangle_visible(gpu, oracle_spk, offset):
    jd = EPOCH
    obs_p, obs_v = np.array([0.0, 1.0, 0.0]), np.array([-GMS_SQRT, 0.0, 0.0])
    obj_p, obj_v = np.array([1.0, 0.0, 0.0]), np.array([0.0, GMS_SQRT, 0.0])
    p, v, st = gpu.propagate_n_body_arrays(obj_p[:, None].copy(), obj_v[:, None].copy(),
                                           np.array([jd]), np.array([jd - offset]), frame=2,
                                           center=0)
    assert st[0] == 0
    sun_o = oracle_spk.spk_get_state(10, jd, 0, 2)[1]
    sun_s = oracle_spk.spk_get_state(10, jd - offset, 0, 2)[1]
    normals = fovmod.rect_normals(obj_p - obs_p, 0.0001, 0.01, 0.01)
    col = np.concatenate([[jd], obs_p - sun_o[:3], obs_v - sun_o[3:], normals.ravel(),
                          [float(fovmod.PATCH_RECTANGLE)]])
    hp = np.ascontiguousarray(p - sun_s[:3, None])
    hv = np.ascontiguousarray(v - sun_s[3:, None])
    for dt_limit in (6.0, 3.0):
        ff, oo, ss = fovmod.fov_check_visible_arrays(hp, hv, np.array([jd - offset]), None,
                                                     col[:, None].copy(), dt_limit)
        assert oo.tolist() == [0], (offset, dt_limit)
        dist = np.linalg.norm(ss[1:4, 0] - col[1:4])
        assert abs(jd - ss[0, 0] - dist / C_AU_PER_DAY) < 1e-6
        flags, out7 = oracle_spk.fov_check_visible(col[:7], normals, hp, hv, jd - offset,
                                                   dt_limit)
        assert flags[0] == 1
        assert np.abs(ss[1:4, 0] - out7[1:4, 0]).max() < 1e-9
