"""Host-side logic that needs no GPU: State handling, synthetic inputs, argument checks."""
import numpy as np
import pytest


def test_state_defaults():
    from kete_b200 import Frames, State

    s = State("a", 2460000.5, [1, 2, 3], [0.1, 0.2, 0.3])
    assert s.frame == Frames.Ecliptic and s.center_id == 10 and s.is_finite
    n = State.new_nan("b", 1.0)
    assert not n.is_finite


def test_frames_roundtrip():
    from kete_b200.state import ecliptic_to_equatorial, equatorial_to_ecliptic

    v = np.array([0.3, -1.2, 0.4])
    np.testing.assert_allclose(equatorial_to_ecliptic(ecliptic_to_equatorial(v)), v, atol=1e-15)


def test_population_matches_oracle_elements(oracle):
    """The vectorised element conversion used for inputs agrees with the oracle's
    restatement of CometElements::to_pos_vel."""
    from kete_b200 import synthetic

    rng = np.random.default_rng(3)
    for _ in range(20):
        a, e, i = rng.uniform(0.8, 3.3), rng.uniform(0, 0.6), rng.uniform(0, 0.5)
        lan, argp, m = rng.uniform(0, 2 * np.pi, 3)
        q = a * (1 - e)
        tp = 2460000.5 - m / (a**-1.5 * synthetic.GMS_SQRT)
        p, v = synthetic.elements_to_state(2460000.5, e, i, lan, tp, argp, q)
        rc, po, vo = oracle.elements_to_state(2460000.5, e, i, lan, tp, argp, q)
        assert rc == 0
        np.testing.assert_allclose(p, po, atol=1e-11)
        np.testing.assert_allclose(v, vo, atol=1e-13)


def test_mixed_population_shape():
    from kete_b200 import synthetic

    pos, vel, ng = synthetic.mixed(1000, seed=1)
    assert pos.shape == (3, 1000) and ng.shape == (10, 1000)
    frac = (ng[0] == 1).mean()
    assert 0.02 < frac < 0.09


def test_host_arrays_must_be_float64():
    from kete_b200 import _lib

    a = _lib.Args()
    with pytest.raises(TypeError):
        a.ptr(np.zeros(3, dtype=np.float32))
    # non-contiguous float64 inputs are copied, not rejected
    m = np.zeros((3, 8))[:, ::2]
    assert a.ptr(m) != 0 and a.keep[-1].flags.c_contiguous


def test_fov_chunk_bounds():
    """Chunks of time-sorted fields (src/kete/rust/fovs/checks.rs:37-57): a chunk closes when
    a field is 2*dt_limit or more after the chunk's first field."""
    from kete_b200.fov import chunk_bounds

    assert chunk_bounds([], 3.0) == [0]
    assert chunk_bounds([0.0], 3.0) == [0, 1]
    assert chunk_bounds([0.0, 5.9, 6.0, 6.1, 11.99, 12.0], 3.0) == [0, 2, 5, 6]
    jds = np.sort(np.random.default_rng(1).uniform(0, 365.25, 500))
    b = chunk_bounds(jds, 3.0)
    for k0, k1 in zip(b[:-1], b[1:]):
        assert jds[k1 - 1] - jds[k0] < 6.0
        if k1 < len(jds):
            assert jds[k1] - jds[k0] >= 6.0


def test_adjoint_wrapper_checks_shapes():
    """The adjoint call refuses checkpoint or seed arrays whose extents do not match, before
    any pointer reaches the library."""
    import pytest

    from kete_b200 import autodiff as A

    ck = A.Checkpoints(4, np.zeros(3), 2, False, None, 5, np.zeros((4, 5, 7)),
                       np.zeros(4, np.int32), np.zeros((3, 4), np.int32), np.zeros(4, np.int32))
    with pytest.raises(ValueError):
        A.propagate_n_body_adjoint(ck, np.zeros((3, 6, 4)))


def test_output_arrays_are_checked():
    """propagate_n_body_arrays(out=...): a caller's arrays are used as given when their shape,
    dtype, layout and side fit, and refused otherwise (never silently copied)."""
    from kete_b200.propagation import _out_array

    tpl = np.zeros((3, 5))
    given = np.empty((3, 5))
    assert _out_array(given, tpl, (3, 5), np.float64, "out[0]") is given
    fresh = _out_array(None, tpl, (3, 5), np.float64, "out[0]")
    assert fresh.shape == (3, 5) and fresh.dtype == np.float64
    st = _out_array(np.empty(5, dtype=np.int32), tpl, (5,), np.int32, "out[2]")
    assert st.dtype == np.int32
    for bad, shape, dtype in ((np.empty((3, 4)), (3, 5), np.float64),
                              (np.empty((3, 5), dtype=np.float32), (3, 5), np.float64),
                              (np.empty((5, 3)).T, (3, 5), np.float64),
                              (np.empty(5, dtype=np.int64), (5,), np.int32),
                              ([0.0] * 5, (5,), np.float64)):
        with pytest.raises(ValueError):
            _out_array(bad, tpl, shape, dtype, "out")
