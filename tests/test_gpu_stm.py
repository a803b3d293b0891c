"""Two-body state-transition matrices and covariance propagation on the GPU against the
oracle (the corrected kete compute_state_transition) and finite differences.
Tolerance: STM entries 2e-8 of the matrix's largest entry (the oracle integrates with
RK4(5) at 1e-12); final states within 1e-12 AU of kete_b200_propagate_two_body; symplectic
defect 1e-10 (the closed form keeps the structure to rounding)."""
import numpy as np
import pytest

from kete_b200 import synthetic

pytestmark = pytest.mark.gpu
EPOCH = 2460000.5
SYMPLECTIC = np.block([[np.zeros((3, 3)), np.eye(3)], [-np.eye(3), np.zeros((3, 3))]])


def _population(n, seed):
    rng = np.random.default_rng(seed)
    pm, vm = synthetic.main_belt(n // 2, seed=seed)
    pn, vn = synthetic.neo(n - n // 2 - 4, seed=seed + 1)
    # hyperbolic and near-parabolic states
    ph = np.array([[1.2, 0.0, 0.0], [0.8, 0.3, 0.1], [3.0, -1.0, 0.5], [1.0, 0.0, 0.0]]).T
    vh = np.array([[0.0, 0.025, 0.003], [-0.01, 0.03, 0.0], [0.0, 0.02, 0.0],
                   [0.0, 0.02432685, 0.0]]).T
    pos = np.ascontiguousarray(np.hstack([pm, pn, ph]))
    vel = np.ascontiguousarray(np.hstack([vm, vn, vh]))
    dt = rng.uniform(-1500.0, 1500.0, pos.shape[1])
    return pos, vel, np.full(pos.shape[1], EPOCH), EPOCH + dt


def test_stm_vs_oracle(gpu, oracle):
    pos, vel, jd0, jd1 = _population(120, 3)
    p, v, m, _, st = gpu.state_transition.compute_stm_arrays(pos, vel, jd0, jd1)
    assert (st == 0).all()
    tp, tv, _, tst = gpu.propagate_two_body_arrays(pos, vel, jd0, jd1)
    # the same closed form in another kernel: rounding-level differences from where the
    # compiler fuses multiply-adds, inside the two-body tolerance
    assert np.abs(p - tp).max() < 1e-12 and np.abs(v - tv).max() < 1e-14
    for i in range(pos.shape[1]):
        _, _, ref = oracle.compute_stm(pos[:, i], vel[:, i], jd0[i], jd1[i])
        err = np.abs(m[:, :, i] - ref).max() / np.abs(ref).max()
        assert err < 2e-8, (i, err)


def test_stm_symplectic_long_spans(gpu):
    # ten-year spans: many revolutions, where the reduced-time anomaly would lose the
    # along-track term if its derivative held the reduced time fixed
    pos, vel = synthetic.main_belt(256, seed=5)
    n = pos.shape[1]
    jd0 = np.full(n, EPOCH)
    _, _, m, _, st = gpu.state_transition.compute_stm_arrays(pos, vel, jd0, jd0 + 3652.5)
    assert (st == 0).all()
    for i in range(n):
        mi = m[:, :, i]
        defect = np.abs(mi.T @ SYMPLECTIC @ mi - SYMPLECTIC).max() / np.abs(mi).max() ** 2
        assert defect < 1e-10


def test_stm_multi_rev_vs_oracle(gpu, oracle):
    pos, vel = synthetic.main_belt(8, seed=6)
    jd0 = np.full(8, EPOCH)
    _, _, m, _, _ = gpu.state_transition.compute_stm_arrays(pos, vel, jd0, jd0 + 3652.5)
    for i in range(8):
        _, _, ref = oracle.compute_stm(pos[:, i], vel[:, i], EPOCH, EPOCH + 3652.5)
        assert np.abs(m[:, :, i] - ref).max() / np.abs(ref).max() < 2e-8


def test_stm_finite_differences(gpu):
    pos, vel = synthetic.neo(4, seed=7)
    dt = 400.0
    _, _, m, _, _ = gpu.state_transition.compute_stm_arrays(pos, vel, np.full(4, EPOCH),
                                                            np.full(4, EPOCH + dt))
    for i in range(4):
        x0 = np.concatenate([pos[:, i], vel[:, i]])
        scales = np.array([1e-4] * 3 + [1e-6] * 3)
        X = []
        for k in range(6):
            for h in (scales[k], scales[k] / 2):
                for sgn in (1, -1):
                    x = x0.copy()
                    x[k] += sgn * h
                    X.append(x)
        X = np.array(X).T
        k = X.shape[1]
        op, ov, _, _ = gpu.propagate_two_body_arrays(np.ascontiguousarray(X[:3]),
                                                     np.ascontiguousarray(X[3:]),
                                                     np.full(k, EPOCH), np.full(k, EPOCH + dt))
        Y = np.vstack([op, ov])
        fd = np.zeros((6, 6))
        for c in range(6):
            y, h = Y[:, 4 * c:4 * c + 4], scales[c]
            fd[:, c] = (4 * (y[:, 2] - y[:, 3]) / h - (y[:, 0] - y[:, 1]) / (2 * h)) / 3
        assert np.abs(m[:, :, i] - fd).max() / np.abs(fd).max() < 1e-7


def test_stm_edges(gpu):
    pos = np.array([[1.5, np.nan], [0.0, 0.0], [0.0, 0.0]])
    vel = np.array([[0.0, 0.0], [0.012, 0.012], [0.0, 0.0]])
    jd0 = np.full(2, EPOCH)
    # a zero interval returns the state untouched (kepler.rs:268-270 skips |dt| < 1e-10
    # before its finiteness check) with the identity; a non-finite state fails otherwise
    p, v, m, _, st = gpu.state_transition.compute_stm_arrays(pos, vel, jd0, jd0 + [0.0, 10.0])
    assert st[0] == 0 and np.array_equal(m[:, :, 0], np.eye(6))
    assert st[1] != 0 and np.isnan(m[:, :, 1]).all() and np.isnan(p[:, 1]).all()


def test_central_mass(gpu, oracle):
    pos, vel = synthetic.main_belt(4, seed=8)
    jd0 = np.full(4, EPOCH)
    _, _, m, _, _ = gpu.state_transition.compute_stm_arrays(pos, vel, jd0, jd0 + 200.0, 2.0)
    for i in range(4):
        _, _, ref = oracle.compute_stm(pos[:, i], vel[:, i], EPOCH, EPOCH + 200.0, 2.0)
        assert np.abs(m[:, :, i] - ref).max() / np.abs(ref).max() < 2e-8


def test_propagate_covariance(gpu):
    rng = np.random.default_rng(9)
    pos, vel = synthetic.main_belt(1, seed=9)
    s = gpu.State("x", EPOCH, pos[:, 0], vel[:, 0])
    a = rng.normal(size=(6, 6)) * np.array([1e-6] * 3 + [1e-8] * 3)
    cov = a @ a.T
    phi = gpu.compute_stm(s, EPOCH + 500.0)
    out = gpu.propagate_covariance(s, cov, EPOCH + 500.0)
    np.testing.assert_allclose(out, phi @ cov @ phi.T, rtol=1e-12, atol=1e-30)
    assert np.array_equal(out, out.T)


def test_covariance_n_body(gpu):
    from kete_b200.autodiff import propagate_n_body_stm_arrays

    pos, vel, ng = synthetic.mixed(16, seed=10, nongrav_frac=0.5)
    ng = np.ascontiguousarray(ng)
    ng[9] = 0.0  # dt = 0: the sensitivities cover A1, A2 without the delay
    rng = np.random.default_rng(11)
    a = rng.normal(size=(16, 8, 8)) * 1e-7
    covs = a @ np.transpose(a, (0, 2, 1))
    states = [gpu.State(i, EPOCH, pos[:, i], vel[:, i]) for i in range(16)]
    models = [gpu.NonGravModel(tuple(ng[:, i])) if ng[0, i] != 0 else None for i in range(16)]
    out = gpu.propagate_covariance_n_body(states, covs, EPOCH + 300.0, non_gravs=models)
    _, stm, st = propagate_n_body_stm_arrays(pos, vel, np.full(16, EPOCH), [EPOCH + 300.0],
                                             nongrav=ng)
    for i in range(16):
        phi = stm[0, :, :, i]
        np.testing.assert_allclose(out[i], phi @ covs[i] @ phi.T, rtol=1e-12, atol=1e-30)
