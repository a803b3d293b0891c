"""GPU system integration (kete_b200_propagate_n_body_long) against the oracle.

Main-belt asteroids, NEOs and comets (JPL comet model) integrated for a year together with
the nine SIMPLE_PLANETS bodies, in batches of 10 (one warp per batch), 23 and 40 (two warps),
with the massive states read from the SPK on the device or given by the caller: positions
agree with the oracle's restatement to 1e-9 AU (the kernels fuse multiply-adds and use
reciprocal square roots; 1e-9 AU is the N-body bound of the other tests).
"""
import numpy as np
import pytest

from kete_b200 import synthetic

pytestmark = pytest.mark.gpu
E = synthetic.EPOCH


def _population(seed=61):
    pm, vm = synthetic.main_belt(30, seed=seed)
    pn, vn = synthetic.neo(15, seed=seed + 1)
    pos = synthetic.ecl_to_eq(np.concatenate([pm, pn], axis=1))
    vel = synthetic.ecl_to_eq(np.concatenate([vm, vn], axis=1))
    n = pos.shape[1]
    rng = np.random.default_rng(seed + 2)
    ng = np.zeros((10, n))
    for i in range(0, n, 3):
        ng[:, i] = synthetic.comet_nongrav(rng.normal(0, 1e-8), rng.normal(0, 1e-9))
    return np.ascontiguousarray(pos), np.ascontiguousarray(vel), ng


@pytest.mark.parametrize("batch", [10, 23, 40])
def test_long_vs_oracle(gpu, oracle_spk, batch):
    pos, vel, ng = _population()
    p, v, pl, st = gpu.propagate_n_body_long_arrays(pos, vel, E, E + 365.25, None, ng, batch)
    op, ov, opl, ost = oracle_spk.propagate_n_body_vec(pos, vel, E, E + 365.25, ng=ng,
                                                       batch_size=batch)
    assert (st == 0).all() and (ost == 0).all()
    assert np.abs(p - op).max() < 1e-9
    assert np.abs(v - ov).max() < 1e-11
    assert np.abs(pl - opl).max() < 1e-9


def test_long_given_planets_and_reversal(gpu, oracle_spk):
    pos, vel, _ = _population(71)
    p, v, pl, st = gpu.propagate_n_body_long_arrays(pos, vel, E, E + 200.0)
    assert (st == 0).all()
    bp, bv, _, st2 = gpu.propagate_n_body_long_arrays(p, v, E + 200.0, E, pl)
    assert (st2 == 0).all()
    assert np.abs(bp - pos).max() < 1e-10
    op, _, _, _ = oracle_spk.propagate_n_body_vec(p, v, E + 200.0, E, planets=pl)
    assert np.abs(bp - op).max() < 1e-9


def test_long_python_api(gpu):
    pos, vel, _ = _population(81)
    from kete_b200.state import equatorial_to_ecliptic as to_ecl

    states = [gpu.State(f"a{i}", E, to_ecl(pos[:, i]), to_ecl(vel[:, i]), gpu.Frames.Ecliptic, 10)
              for i in range(5)]
    out, planets = gpu.propagate_n_body_long(states, E + 50.0, batch_size=3)
    assert [s.desig for s in out] == [f"a{i}" for i in range(5)]
    assert all(s.jd == E + 50.0 and int(s.center_id) == 10 for s in out)
    assert len(planets) == 9 and np.abs(planets[0].pos).max() == 0.0  # the Sun itself
    p, _, _, _ = gpu.propagate_n_body_long_arrays(pos[:, :5].copy(), vel[:, :5].copy(), E,
                                                  E + 50.0, None, None, 3)
    assert np.abs(np.stack([s.pos for s in out], axis=1) - p).max() < 1e-12
    bad = states[:2] + [gpu.State("late", E + 1.0, [2.0, 0, 0], [0, 0.01, 0], gpu.Frames.Ecliptic, 10)]
    with pytest.raises(ValueError, match="same JD"):
        gpu.propagate_n_body_long(bad, E + 10.0)
