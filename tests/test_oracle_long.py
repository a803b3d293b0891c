"""The oracle's system integration (propagate_n_body_vec, kete_core/propagation/mod.rs:142-237).

There is no reference test of it, so it is pinned by properties: integrating forward and
back returns to the start (1e-10 AU after 200 days both ways), a test particle's result
does not depend on which batch carries it (the step sizes are set by the planets), and the
comet model is skipped for the first particle of a batch, as the reference's vec_accel does
(acceleration.rs:239-240).
"""
import os

import numpy as np
import pytest

from kete_b200 import synthetic

E = synthetic.EPOCH


@pytest.fixture(scope="module")
def loaded(oracle, tmp_path_factory):
    p = synthetic.write_synthetic_spk(str(tmp_path_factory.mktemp("spk") / "s.bsp"))
    oracle.spk_reset()
    with open(p, "rb") as f:
        oracle.spk_load_bytes(f.read())
    return oracle


def _population(n, seed):
    pos, vel = synthetic.main_belt(n, seed=seed)
    return synthetic.ecl_to_eq(pos), synthetic.ecl_to_eq(vel)


def test_time_reversal(loaded):
    pos, vel = _population(12, 5)
    op, ov, opl, st = loaded.propagate_n_body_vec(pos, vel, E, E + 200.0)
    assert (st == 0).all()
    bp, bv, _, st2 = loaded.propagate_n_body_vec(op, ov, E + 200.0, E, planets=opl)
    assert (st2 == 0).all()
    assert np.abs(bp - pos).max() < 1e-10
    assert np.abs(bv - vel).max() < 1e-12


def test_batches_do_not_change_particles(loaded):
    pos, vel = _population(23, 7)
    a = loaded.propagate_n_body_vec(pos, vel, E, E + 120.0, batch_size=10)
    b = loaded.propagate_n_body_vec(pos, vel, E, E + 120.0, batch_size=1)
    assert np.abs(a[0] - b[0]).max() < 1e-12


def test_first_particle_of_a_batch_has_no_comet_model(loaded):
    pos, vel = _population(2, 9)
    ng = np.repeat(synthetic.comet_nongrav(3e-8, 1e-9)[:, None], 2, axis=1)
    with_ng = loaded.propagate_n_body_vec(pos, vel, E, E + 300.0, ng=ng, batch_size=2)[0]
    without = loaded.propagate_n_body_vec(pos, vel, E, E + 300.0, batch_size=2)[0]
    assert np.array_equal(with_ng[:, 0], without[:, 0])
    assert np.abs(with_ng[:, 1] - without[:, 1]).max() > 1e-7
