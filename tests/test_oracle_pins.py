"""Reference tests that need an SPK, run on the oracle over the synthetic ephemeris.

- check_accelerations_equal (kete_core/propagation/acceleration.rs:298-347): vec_accel with
  the MASSES bodies' states taken from the SPK equals spk_accel for a test particle at
  (0, 0, 0.5) AU moving at (0, 0, 1) AU/day, to 1e-10 AU/day^2 per component.  The reference
  evaluates it at JD 2451545.0 on DE440s; here at epochs inside the synthetic SPK.
- test_check_rectangle_visible (kete_core/fov/generic.rs:199-235): an object on a circular
  orbit seen from an observer on another, in a 0.01 x 0.01 rad rectangle pointed at it, is
  visible when its state is given up to 10 days before or after the observation (the
  two-body and N-body light-time branches), with the light-time identity of
  generic.rs:262-263 (observer epoch - state epoch = distance / c to 1e-6 day).
"""
import numpy as np
import pytest

from kete_b200 import fov as fovmod
from kete_b200 import synthetic

EPOCH = synthetic.EPOCH
MASSES = (10, 1, 2, 399, 301, 4, 5, 6, 7, 8, 20000001, 20000002, 20000004, 20000010, 20000704)
GMS_SQRT = 0.01720209894996
C_AU_PER_DAY = 173.14463267424034


@pytest.fixture(scope="module")
def oracle_masses(oracle, tmp_path_factory, spk_path):
    """The oracle with the synthetic SPK that also holds the five asteroids of MASSES; the
    session's planets-only SPK is restored afterwards."""
    p = tmp_path_factory.mktemp("spk_masses") / "masses.bsp"
    synthetic.write_synthetic_spk(str(p), asteroids=True)
    oracle.spk_reset()
    oracle.spk_load_bytes(open(p, "rb").read())
    yield oracle
    oracle.spk_reset()
    with open(spk_path, "rb") as f:
        oracle.spk_load_bytes(f.read())


def massive_states(oracle, ids, jd):
    cols = []
    for i in ids:
        rc, s = oracle.spk_get_state(i, jd, 0, 1)  # barycentric, equatorial
        assert rc == 0
        cols.append(s)
    return np.stack(cols, axis=1)


@pytest.mark.parametrize("jd", [EPOCH, EPOCH - 1234.5, EPOCH + 2000.25])
def test_check_accelerations_equal(oracle_masses, jd):
    O = oracle_masses
    massive = massive_states(O, MASSES, jd)
    pos, vel = np.array([[0.0], [0.0], [0.5]]), np.array([[0.0], [0.0], [1.0]])
    acc, st = O.vec_accel(1, massive, pos, vel)
    rc, acc2 = O.spk_accel(jd, pos[:, 0], vel[:, 0], include_extended=True)
    assert rc == 0 and st[0] == 0
    assert np.abs(acc[:, 0] - acc2).max() < 1e-10
    # the same identity for the planets alone and at scattered points
    rng = np.random.default_rng(int(jd) % 1000)
    pos = rng.uniform(-3.0, 3.0, (3, 50))
    vel = rng.uniform(-0.02, 0.02, (3, 50))
    acc, st = O.vec_accel(0, massive[:, :10], pos, vel)
    assert (st == 0).all()
    for k in range(50):
        rc, acc2 = O.spk_accel(jd, pos[:, k], vel[:, k])
        assert rc == 0 and np.abs(acc[:, k] - acc2).max() < 1e-10


def circular_states(oracle_spk, jd, offset):
    """generic.rs:203-218: observer at (0, 1, 0) and object at (1, 0, 0) AU on circular
    orbits (barycentric ecliptic), the object's state propagated to jd - offset."""
    obs_p, obs_v = np.array([0.0, 1.0, 0.0]), np.array([-GMS_SQRT, 0.0, 0.0])
    obj_p, obj_v = np.array([1.0, 0.0, 0.0]), np.array([0.0, GMS_SQRT, 0.0])
    op, ov, st, _, _ = oracle_spk.propagate_n_body(obj_p[:, None], obj_v[:, None], jd,
                                                    jd - offset, frame=2, center=0)
    assert st[0] == 0
    pointing = obj_p - obs_p
    return obs_p, obs_v, op[:, 0], ov[:, 0], pointing


def sun_ecliptic(oracle_spk, jd):
    rc, s = oracle_spk.spk_get_state(10, jd, 0, 2)
    assert rc == 0
    return s


@pytest.mark.parametrize("offset", [-10.0, -5.0, 0.0, 5.0, 10.0])
def test_check_rectangle_visible(oracle_spk, offset):
    jd = EPOCH
    obs_p, obs_v, p, v, pointing = circular_states(oracle_spk, jd, offset)
    # the field table and the check work in heliocentric ecliptic coordinates
    sun_o, sun_s = sun_ecliptic(oracle_spk, jd), sun_ecliptic(oracle_spk, jd - offset)
    obs7 = np.concatenate([[jd], obs_p - sun_o[:3], obs_v - sun_o[3:]])
    normals = fovmod.rect_normals(pointing, 0.0001, 0.01, 0.01)
    hp, hv = (p - sun_s[:3])[:, None], (v - sun_s[3:])[:, None]
    for dt_limit in (6.0, 3.0):  # both light-time branches for |offset| in (3, 6]
        flags, out7 = oracle_spk.fov_check_visible(obs7, normals, hp, hv, jd - offset, dt_limit)
        assert flags[0] == 1, (offset, dt_limit)
        dist = np.linalg.norm(out7[1:4, 0] - obs7[1:4])
        assert abs(jd - out7[0, 0] - dist / C_AU_PER_DAY) < 1e-6
