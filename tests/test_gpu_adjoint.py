"""GPU reverse-mode gradients (kete_b200_propagate_n_body_checkpointed / _adjoint).

The adjoint of the executed Radau steps must equal the transposed forward sensitivities:
for seeds s_k = dL/d(state at epoch k), dL/d(pos0, vel0, A1, A2) = sum_k Phi_k^T s_k with
Phi_k from kete_b200_propagate_n_body_stm.  The two kernels integrate with different
force-evaluation code (the adjoint's forward pass uses the node-parallel fast path, the
sensitivity kernel the dual-number path), so their trajectories differ by ~1e-13 AU; the
adjoint also takes each node's Jacobian at the last corrector iteration's point.  The
agreement bound is 1e-8 of the largest gradient entry of each object and parameter group.
The checkpointed states match the oracle's chained propagation to 1e-9 AU.
"""
import numpy as np
import pytest

from kete_b200 import synthetic

pytestmark = pytest.mark.gpu

EPOCH = synthetic.EPOCH


def _population(n_neo=12, n_comet=4, seed=101):
    pos_n, vel_n = synthetic.neo(n_neo, seed=seed)
    pos_c, vel_c = synthetic.neo(n_comet, seed=seed + 1)
    pos = np.ascontiguousarray(np.concatenate([pos_n, pos_c], axis=1))
    vel = np.ascontiguousarray(np.concatenate([vel_n, vel_c], axis=1))
    n = pos.shape[1]
    rng = np.random.default_rng(seed + 2)
    ng = np.zeros((10, n))
    for i in range(n):
        a1 = rng.normal(0.0, 2e-8) if i >= n_neo else 0.0
        a2 = rng.normal(0.0, 2e-9) if i >= n_neo else 0.0
        ng[:, i] = synthetic.comet_nongrav(a1, a2)
    return pos, vel, ng


def _stm_gradient(stm, seed):
    return np.einsum("kcn,kcpn->pn", seed, stm)


def _check_close(g, ref, rtol):
    for rows in (slice(0, 3), slice(3, 6), slice(6, 7), slice(7, 8)):
        scale = np.abs(ref[rows]).max(axis=0)
        err = np.abs(g[rows] - ref[rows]).max(axis=0)
        assert (err <= rtol * scale).all(), (rows, (err / scale).max())


@pytest.mark.parametrize("frame", [2, 1])
def test_adjoint_matches_transposed_stm(gpu, frame):
    from kete_b200.autodiff import (propagate_n_body_adjoint, propagate_n_body_checkpointed,
                                    propagate_n_body_stm_arrays)

    pos, vel, ng = _population()
    n = pos.shape[1]
    epochs = EPOCH + np.linspace(36.5, 730.0, 20)
    jd0 = np.full(n, EPOCH)
    states, st, ck = propagate_n_body_checkpointed(pos, vel, jd0, epochs, frame=frame, nongrav=ng)
    assert (st == 0).all()
    s_stm, stm, st2 = propagate_n_body_stm_arrays(pos, vel, jd0, epochs, frame=frame, nongrav=ng)
    assert (st2 == 0).all()
    assert np.abs(states - s_stm).max() < 1e-9
    rng = np.random.default_rng(3)
    seed = rng.normal(size=(20, 6, n))
    grad, gst = propagate_n_body_adjoint(ck, seed)
    assert (gst == 0).all()
    _check_close(grad, _stm_gradient(stm.reshape(20, 6, 8, n), seed), 1e-8)


def test_checkpointed_states_match_oracle_chain(gpu, oracle_spk):
    from kete_b200.autodiff import propagate_n_body_checkpointed

    pos, vel, ng = _population(6, 2)
    n = pos.shape[1]
    epochs = EPOCH + np.array([50.0, 300.0, 700.0])
    states, st, ck = propagate_n_body_checkpointed(pos, vel, np.full(n, EPOCH), epochs, nongrav=ng)
    assert (st == 0).all()
    p, v, t = pos, vel, EPOCH
    for k, tk in enumerate(epochs):
        p, v, ost, _, _ = oracle_spk.propagate_n_body(p, v, np.full(n, t), np.full(n, tk), ng=ng)
        assert (ost == 0).all()
        assert np.abs(states[k, 0:3] - p).max() < 1e-9
        t = tk


def test_checkpoint_capacity_retry_and_blocks(gpu):
    """A capacity of one forces the retry; the gradient does not depend on how the steps are
    blocked (a single segment spanning many blocks against many short segments)."""
    from kete_b200 import autodiff as A

    pos, vel, ng = _population(3, 1)
    n = pos.shape[1]
    jd0 = np.full(n, EPOCH)
    epochs = EPOCH + np.array([400.0])
    _, st, ck = A.propagate_n_body_checkpointed(pos, vel, jd0, epochs, nongrav=ng, capacity=1)
    assert (st == 0).all()
    assert ck.capacity == int(ck.count.max()) > 1
    seed = np.random.default_rng(5).normal(size=(1, 6, n))
    g1, _ = A.propagate_n_body_adjoint(ck, seed)
    _, stm, _ = A.propagate_n_body_stm_arrays(pos, vel, jd0, epochs, nongrav=ng)
    _check_close(g1, _stm_gradient(stm, seed), 1e-8)


def test_adjoint_zero_length_and_repeated_epochs(gpu):
    from kete_b200 import autodiff as A

    pos, vel, ng = _population(2, 1)
    n = pos.shape[1]
    jd0 = np.full(n, EPOCH)
    epochs = np.array([EPOCH, EPOCH + 20.0, EPOCH + 20.0, EPOCH - 15.0])
    states, st, ck = A.propagate_n_body_checkpointed(pos, vel, jd0, epochs, nongrav=ng)
    assert (st == 0).all()
    assert np.abs(states[0, 0:3] - pos).max() < 1e-13
    seed = np.random.default_rng(8).normal(size=(4, 6, n))
    g, gst = A.propagate_n_body_adjoint(ck, seed)
    assert (gst == 0).all()
    _, stm, _ = A.propagate_n_body_stm_arrays(pos, vel, jd0, epochs, nongrav=ng)
    _check_close(g, _stm_gradient(stm, seed), 1e-8)


def test_adjoint_failed_objects_are_nan(gpu):
    from kete_b200 import autodiff as A

    pos, vel, ng = _population(3, 0)
    pos[1, 2] = np.nan
    ng[9, 0] = 1.5  # a comet-model time delay: not differentiated, reported as a value error
    n = pos.shape[1]
    states, st, ck = A.propagate_n_body_checkpointed(pos, vel, np.full(n, EPOCH),
                                                     EPOCH + np.array([30.0, 60.0]), nongrav=ng)
    assert st.tolist() == [2, 0, 2]
    g, gst = A.propagate_n_body_adjoint(ck, np.ones((2, 6, n)))
    assert np.isnan(g[:, 0]).all() and np.isnan(g[:, 2]).all() and np.isfinite(g[:, 1]).all()
    assert np.isnan(states[:, :, 0]).all() and np.isfinite(states[:, :, 1]).all()


def test_adjoint_device_arrays_and_autograd_agree(gpu):
    """Through torch.autograd (device tensors): the adjoint route and the STM route give the
    same gradient of an RA/Dec loss."""
    import torch

    from kete_b200.autodiff import ecliptic_to_equatorial_torch, nbody_positions, radec

    pos, vel, ng = _population(8, 4, seed=7)
    n = pos.shape[1]
    dev = torch.device("cuda", 0)
    T = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    epochs = T(EPOCH + np.linspace(36.5, 730.0, 20))
    jd0 = T(np.full(n, EPOCH))
    obs = T(np.array([0.2, -0.95, 0.0]))[None, :, None]
    grads = {}
    for method in ("adjoint", "stm"):
        p0, v0 = T(pos).requires_grad_(True), T(vel).requires_grad_(True)
        a1, a2 = T(ng[1]).requires_grad_(True), T(ng[2]).requires_grad_(True)
        pk = nbody_positions(p0, v0, a1, a2, jd0, epochs, nongrav_rest=T(ng), method=method)
        ra, dec = radec(ecliptic_to_equatorial_torch(pk - obs))
        loss = (torch.sin(ra) ** 2 + dec ** 2).sum()
        loss.backward()
        grads[method] = np.concatenate([p0.grad.cpu().numpy(), v0.grad.cpu().numpy(),
                                        a1.grad.cpu().numpy()[None], a2.grad.cpu().numpy()[None]])
    _check_close(grads["adjoint"], grads["stm"], 1e-8)


def test_adjoint_forms_identical(gpu):
    """The up-front parallel replay of every checkpoint block (with its dense block order and
    queue) and the sweep's own per-block replay give the same gradients bit for bit, on a
    population whose objects hold different numbers of checkpoint blocks."""
    from kete_b200.autodiff import (propagate_n_body_adjoint, propagate_n_body_checkpointed,
                                    set_adjoint_form)

    pos, vel, ng = _population(40, 8, seed=131)
    n = pos.shape[1]
    epochs = EPOCH + np.linspace(20.0, 500.0, 7)
    states, st, ck = propagate_n_body_checkpointed(pos, vel, np.full(n, EPOCH), epochs,
                                                   nongrav=ng)
    assert (st == 0).all()
    seed = np.random.default_rng(5).normal(size=(7, 6, n))
    try:
        grads = []
        for form in (0, 1, 0):
            set_adjoint_form(form)
            g, gst = propagate_n_body_adjoint(ck, seed)
            assert (gst == 0).all()
            grads.append(g)
    finally:
        set_adjoint_form(0)
    assert np.isfinite(grads[0]).all()
    assert np.array_equal(grads[0], grads[1])
    assert np.array_equal(grads[0], grads[2])
    from kete_b200._lib import KeteB200Error

    with pytest.raises(KeteB200Error):
        set_adjoint_form(2)
