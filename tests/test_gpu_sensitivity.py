"""GPU sensitivities of the N-body propagation (kete_b200_propagate_n_body_stm).

The 6 x 8 matrices d(pos, vel)/d(pos0, vel0, A1, A2) are checked against finite
differences of the same kernel's states.  A perturbed integration takes slightly different
steps and corrector iteration counts, which moves its result by ~1e-12 AU, so a plain
central difference carries an error ~1e-12/delta besides its delta^2 truncation.  The
steps below sit between the two (1e-4 AU, 1e-6 AU/day, 5e-8 and 5e-9 AU/day^2) and the
delta^2 term is removed by Richardson extrapolation, (4 D(delta) - D(2 delta)) / 3.  Per
object, epoch and direction, the largest difference over the six rows is at most 1e-5 of
that column's largest entry.  The states match the oracle's chained propagation to 1e-9 AU.
"""
import numpy as np
import pytest

from kete_b200 import synthetic

pytestmark = pytest.mark.gpu

EPOCH = synthetic.EPOCH
EPOCHS = EPOCH + np.array([60.0, 250.0, 730.0])


@pytest.fixture(params=[0, 1], ids=["nodes", "thread"])
def form(request, gpu):
    """Both forms of the forward sensitivities: eight lanes per object (default) and one
    object per thread."""
    from kete_b200.autodiff import set_sensitivity_form

    set_sensitivity_form(request.param)
    yield request.param
    set_sensitivity_form(0)


def _population(n_neo=6, n_comet=4, seed=77):
    pos_n, vel_n = synthetic.neo(n_neo, seed=seed)
    pos_c, vel_c = synthetic.neo(n_comet, seed=seed + 1)
    pos = np.ascontiguousarray(np.concatenate([pos_n, pos_c], axis=1))
    vel = np.ascontiguousarray(np.concatenate([vel_n, vel_c], axis=1))
    n = pos.shape[1]
    rng = np.random.default_rng(seed + 2)
    ng = np.zeros((10, n))
    for i in range(n):  # every object carries the comet model, so the A columns are defined
        a1 = rng.normal(0.0, 2e-8) if i >= n_neo else 0.0
        a2 = rng.normal(0.0, 2e-9) if i >= n_neo else 0.0
        ng[:, i] = synthetic.comet_nongrav(a1, a2)
    return pos, vel, ng


def test_stm_states_match_oracle_chain(gpu, form, oracle_spk):
    from kete_b200.autodiff import propagate_n_body_stm_arrays

    pos, vel, ng = _population()
    n = pos.shape[1]
    states, stm, st = propagate_n_body_stm_arrays(pos, vel, np.full(n, EPOCH), EPOCHS, nongrav=ng)
    assert (st == 0).all()
    assert np.isfinite(stm).all()
    p, v, t = pos, vel, EPOCH
    for k, tk in enumerate(EPOCHS):
        p, v, ost, _, _ = oracle_spk.propagate_n_body(p, v, np.full(n, t), np.full(n, tk), ng=ng)
        assert (ost == 0).all()
        assert np.abs(states[k, 0:3] - p).max() < 1e-9
        assert np.abs(states[k, 3:6] - v).max() < 1e-11
        t = tk


STEPS = [1e-4] * 3 + [1e-6] * 3 + [5e-8, 5e-9]


def _perturbed(pos, vel, ng, p, d):
    P, V, G = pos.copy(), vel.copy(), ng.copy()
    if p < 3:
        P[p] += d
    elif p < 6:
        V[p - 3] += d
    else:
        G[p - 5] += d  # rows 1, 2: A1, A2
    return P, V, G


def _richardson(f, d):
    """(4 D(d) - D(2d)) / 3 with D the central difference of f at step d."""
    D1 = (f(d) - f(-d)) / (2.0 * d)
    D2 = (f(2 * d) - f(-2 * d)) / (4.0 * d)
    return (4.0 * D1 - D2) / 3.0


def test_stm_vs_finite_differences(gpu, form):
    from kete_b200.autodiff import propagate_n_body_stm_arrays

    pos, vel, ng = _population()
    n = pos.shape[1]
    jd0 = np.full(n, EPOCH)
    _, stm, st = propagate_n_body_stm_arrays(pos, vel, jd0, EPOCHS, nongrav=ng)
    assert (st == 0).all()
    for p in range(8):
        def states_ng(d):
            P, V, G = _perturbed(pos, vel, ng, p, d)
            s, _, st2 = propagate_n_body_stm_arrays(P, V, jd0, EPOCHS, nongrav=G)
            assert (st2 == 0).all()
            return s

        fd = _richardson(states_ng, STEPS[p])  # (K, 6, n)
        col = stm[:, :, p, :]
        err = np.abs(fd - col).max(axis=1) / np.abs(col).max(axis=1)
        assert err.max() < 1e-5, (p, err.max())


def test_stm_identity_at_start_and_frames(gpu, form):
    """An epoch equal to the start gives the identity (A columns zero), in either frame."""
    from kete_b200.autodiff import propagate_n_body_stm_arrays
    from kete_b200.state import Frames

    pos, vel, ng = _population(3, 1)
    n = pos.shape[1]
    for frame in (Frames.Ecliptic, Frames.Equatorial):
        s, stm, st = propagate_n_body_stm_arrays(pos, vel, np.full(n, EPOCH), [EPOCH], frame=frame,
                                                 nongrav=ng)
        assert (st == 0).all()
        eye = np.zeros((6, 8))
        eye[:, :6] = np.eye(6)
        assert np.abs(stm[0] - eye[:, :, None]).max() < 1e-13
        assert np.abs(s[0, 0:3] - pos).max() < 1e-13


def test_stm_failure_is_nan(gpu, form):
    from kete_b200.autodiff import propagate_n_body_stm_arrays

    pos, vel, ng = _population(2, 0)
    pos[0, 1] = np.nan
    s, stm, st = propagate_n_body_stm_arrays(pos, vel, np.full(2, EPOCH), EPOCHS[:2], nongrav=ng)
    assert st[1] != 0 and st[0] == 0
    assert np.isnan(s[:, :, 1]).all() and np.isnan(stm[:, :, :, 1]).all()
    assert np.isfinite(s[:, :, 0]).all()


@pytest.mark.parametrize("method", ["adjoint", "stm"])
def test_radec_loss_gradient_through_autograd(gpu, method):
    """d(RA/Dec residual loss)/d(pos0, vel0, A1, A2) from torch.autograd against
    Richardson-extrapolated differences of the loss (relative agreement 2e-5)."""
    import torch

    from kete_b200.autodiff import ecliptic_to_equatorial_torch, nbody_positions, radec

    pos, vel, ng = _population(2, 2, seed=5)
    n = pos.shape[1]
    dev = torch.device("cuda", 0)
    T = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    obs = T(np.array([0.2, -0.95, 0.0]))[None, :, None]  # fixed observer, ecliptic AU
    epochs = T(EPOCHS)
    jd0 = T(np.full(n, EPOCH))
    rest = T(ng)
    rng = np.random.default_rng(9)
    ra_obs = None

    def loss_of(p0, v0, a1, a2):
        nonlocal ra_obs
        pos_k = nbody_positions(p0, v0, a1, a2, jd0, epochs, nongrav_rest=rest, method=method)
        ra, dec = radec(ecliptic_to_equatorial_torch(pos_k - obs))
        if ra_obs is None:
            ra_obs = (ra + T(rng.normal(0, 1e-5, tuple(ra.shape)))).detach()
        return ((ra - ra_obs) ** 2 + dec ** 2).sum()

    p0 = T(pos).requires_grad_(True)
    v0 = T(vel).requires_grad_(True)
    a1 = T(ng[1]).requires_grad_(True)
    a2 = T(ng[2]).requires_grad_(True)
    loss = loss_of(p0, v0, a1, a2)
    loss.backward()
    grads = [p0.grad.cpu().numpy(), v0.grad.cpu().numpy(), a1.grad.cpu().numpy(),
             a2.grad.cpu().numpy()]
    base = [pos, vel, ng[1], ng[2]]
    deltas = [1e-4, 1e-6, 5e-8, 5e-9]
    with torch.no_grad():
        for which in range(4):
            g = grads[which].reshape(-1)
            for j in range(g.size):
                def loss_at(d):
                    args = [b.copy() for b in base]
                    args[which].reshape(-1)[j] += d
                    return float(loss_of(*[T(a) for a in args]))

                fd = _richardson(loss_at, deltas[which])
                tol = 2e-5 * max(abs(g[j]), np.abs(g).max() * 1e-3)
                assert abs(fd - g[j]) <= tol, (which, j, fd, g[j])


def test_stm_forms_agree(gpu):
    """The node-parallel form (each node's Jacobian once per attempt, at its last corrector
    iteration's point) against the one-object-per-thread form (every iteration's Jacobian at
    its own points): per object, epoch and direction, 1e-7 of the column's largest entry."""
    from kete_b200.autodiff import propagate_n_body_stm_arrays, set_sensitivity_form

    pos, vel, ng = _population(24, 8, seed=13)
    n = pos.shape[1]
    jd0 = np.full(n, EPOCH)
    out = {}
    try:
        for f in (0, 1):
            set_sensitivity_form(f)
            out[f] = propagate_n_body_stm_arrays(pos, vel, jd0, EPOCHS, nongrav=ng)
    finally:
        set_sensitivity_form(0)
    (s0, m0, st0), (s1, m1, st1) = out[0], out[1]
    assert (st0 == 0).all() and (st1 == 0).all()
    assert np.abs(s0 - s1).max() < 1e-10  # the same trajectories, to rounding
    err = np.abs(m0 - m1).max(axis=1) / np.abs(m1).max(axis=1)  # (K, 8, n)
    assert err.max() < 1e-7, err.max()
