"""The oracle's two-body state-transition matrix (the corrected compute_state_transition,
kete_core/propagation/state_transition.rs:6-122 on runge_kutta.rs's RK4(5)) pinned against
finite differences of the oracle's own two-body propagation (kepler.rs:254-322), the
symplectic structure every Hamiltonian flow has, and composition; plus the host-side shape
checks of kete_b200.state_transition."""
import numpy as np
import pytest

GMS_SQRT = 0.01720209894996
SYMPLECTIC = np.block([[np.zeros((3, 3)), np.eye(3)], [-np.eye(3), np.zeros((3, 3))]])

# (pos, vel, dt): circular, main belt one year and eight years, hyperbolic, backwards NEO
CASES = [
    ([1.0, 0.0, 0.0], [0.0, GMS_SQRT, 0.0], 100.0),
    ([2.5, 0.3, 0.1], [-0.002, 0.0105, 0.001], 365.25),
    ([2.5, 0.3, 0.1], [-0.002, 0.0105, 0.001], 3000.0),
    ([1.2, 0.0, 0.0], [0.0, 0.025, 0.003], 200.0),
    ([0.9, 0.4, -0.2], [0.005, 0.015, 0.002], -500.0),
]


def fd_stm(oracle, p, v, dt, rel=1e-4):
    """Central differences with one Richardson step, of the oracle's two-body propagation."""
    x0 = np.concatenate([p, v])
    scales = np.array([1, 1, 1, 0.01, 0.01, 0.01]) * rel
    X = []
    for k in range(6):
        for h in (scales[k], scales[k] / 2):
            for sgn in (1, -1):
                x = x0.copy()
                x[k] += sgn * h
                X.append(x)
    X = np.array(X).T
    op, ov, _, st = oracle.propagate_two_body(np.ascontiguousarray(X[:3]),
                                              np.ascontiguousarray(X[3:]), 0.0, dt)
    assert (st == 0).all()
    Y = np.vstack([op, ov])
    J = np.zeros((6, 6))
    for k in range(6):
        y, h = Y[:, 4 * k:4 * k + 4], scales[k]
        J[:, k] = (4 * (y[:, 2] - y[:, 3]) / h - (y[:, 0] - y[:, 1]) / (2 * h)) / 3
    return J


@pytest.mark.parametrize("p,v,dt", CASES)
def test_oracle_stm_matches_finite_differences(oracle, p, v, dt):
    p, v = np.array(p), np.array(v)
    fp, fv, m = oracle.compute_stm(p, v, 0.0, dt)
    ref = fd_stm(oracle, p, v, dt)
    assert np.abs(m - ref).max() / np.abs(ref).max() < 2e-8
    op, ov, _, _ = oracle.propagate_two_body(p.reshape(3, 1), v.reshape(3, 1), 0.0, dt)
    assert np.abs(fp - op[:, 0]).max() < 1e-8  # RK4(5) at 1e-12 vs the closed form


@pytest.mark.parametrize("p,v,dt", CASES)
def test_oracle_stm_symplectic(oracle, p, v, dt):
    _, _, m = oracle.compute_stm(np.array(p), np.array(v), 0.0, dt)
    scale = np.abs(m).max() ** 2
    assert np.abs(m.T @ SYMPLECTIC @ m - SYMPLECTIC).max() / scale < 1e-9
    assert abs(np.linalg.det(m) - 1.0) < 1e-7


def test_oracle_stm_composes(oracle):
    p, v = np.array([2.2, -0.7, 0.2]), np.array([0.004, 0.01, -0.001])
    _, _, m02 = oracle.compute_stm(p, v, 0.0, 700.0)
    p1, v1, m01 = oracle.compute_stm(p, v, 0.0, 300.0)
    _, _, m12 = oracle.compute_stm(p1, v1, 300.0, 700.0)
    assert np.abs(m12 @ m01 - m02).max() / np.abs(m02).max() < 1e-9


def test_oracle_stm_zero_interval(oracle):
    _, _, m = oracle.compute_stm([1.5, 0, 0], [0, 0.012, 0], 10.0, 10.0)
    assert np.array_equal(m, np.eye(6))


def test_covariance_shape_checks():
    import kete_b200 as kb

    s = kb.State("a", 2460000.5, [1.5, 0, 0], [0, 0.012, 0])
    with pytest.raises(ValueError):
        kb.propagate_covariance(s, np.eye(5), 2460010.5)
    with pytest.raises(ValueError):
        kb.propagate_covariance_n_body([s], np.zeros((1, 7, 7)), 2460010.5)
    with pytest.raises(ValueError):
        kb.propagate_covariance_n_body([s, kb.State("b", 2460000.5, [2, 0, 0], [0, 0.01, 0],
                                                    center_id=0)],
                                       np.zeros((2, 6, 6)), 2460010.5)
