"""Gradients of N-body predictions behind torch.autograd.

Two GPU routes differentiate kete's N-body propagation (src/kete_core/src/propagation/
mod.rs:70-118) through a sequence of epochs with respect to the initial position, initial
velocity and the JPL comet A1/A2 parameters, both as derivatives of the Radau steps the
GPU executed (step sizes held fixed):

* reverse mode (the default): ``propagate_n_body_checkpointed`` integrates and stores a
  checkpoint every 16 step attempts; ``propagate_n_body_adjoint`` turns dL/d(states) into
  dL/d(pos0, vel0, A1, A2) by re-running each checkpoint block and transposing its steps;
* forward mode: ``propagate_n_body_stm_arrays`` returns the 6 x 8 sensitivity matrix of
  every state (the check of the reverse mode, and the tool when the matrices themselves
  are wanted, e.g. for covariance propagation).

``nbody_states`` / ``nbody_positions`` wrap either as a torch.autograd.Function, so losses
built on predicted positions (RA/Dec residuals) differentiate with torch.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .state import Frames


CHECKPOINT_FULL = 8
SENS_CK_ATTEMPTS = 16


def checkpoint_doubles() -> int:
    """Doubles per checkpoint, as the library lays them out."""
    return int(_lib.lib().kete_b200_checkpoint_doubles())


def _bind():
    L = _lib.lib()
    v = ctypes.c_void_p
    i, i64 = ctypes.c_int, ctypes.c_int64
    L.kete_b200_propagate_n_body_stm.argtypes = [i64, v, v, v, i, v, i, i64, i, v, v, v, v, i, v]
    L.kete_b200_propagate_n_body_checkpointed.argtypes = [i64, v, v, v, i, v, i, i64, i, v, v, v,
                                                          i, v, v, v, i, v]
    L.kete_b200_propagate_n_body_adjoint.argtypes = [i64, i, v, i, i, v, i, v, v, v, v, v, v, v,
                                                     i, v]
    return L


def set_sensitivity_form(form: int = 0):
    """Form of the forward sensitivities (kete_b200_set_sensitivity_form): 0 = eight lanes per
    object with each node's Jacobian taken once per step attempt (default); 1 = one object
    per thread with every corrector iteration's Jacobian at its own points."""
    L = _lib.lib()
    L.kete_b200_set_sensitivity_form.argtypes = [ctypes.c_int]
    _lib.check(L.kete_b200_set_sensitivity_form(int(form)))


def set_adjoint_form(form: int = 0):
    """Form of the adjoint pass's replays (kete_b200_set_adjoint_form): 0 = every checkpoint
    block replayed in one parallel launch before the sweep (default, when the records fit the
    library's bounded scratch); 1 = the sweep re-runs each block just before transposing it.
    The gradients are identical."""
    L = _lib.lib()
    L.kete_b200_set_adjoint_form.argtypes = [ctypes.c_int]
    _lib.check(L.kete_b200_set_adjoint_form(int(form)))


def propagate_n_body_stm_arrays(pos, vel, jd0, epochs, frame=Frames.Ecliptic, center=10,
                                include_asteroids=False, nongrav=None):
    """States at each epoch and their sensitivities.

    pos/vel (3, n), jd0 (n,), epochs (K,) shared; nongrav None or (10, n).  Host numpy
    arrays or torch CUDA tensors (all on the same side).  Returns (states (K, 6, n),
    stm (K, 6, 8, n), status (n,))."""
    _lib.init()
    L = _bind()
    n = int(pos.shape[1])
    if _lib._is_torch_cuda(pos):
        import torch

        if not _lib._is_torch_cuda(epochs):
            epochs = torch.as_tensor(np.asarray(epochs, np.float64), device=pos.device)
        K = int(epochs.shape[0])
        states = torch.empty((K, 6, n), dtype=torch.float64, device=pos.device)
        stm = torch.empty((K, 6, 8, n), dtype=torch.float64, device=pos.device)
        st = torch.empty(n, dtype=torch.int32, device=pos.device)
    else:
        epochs = np.ascontiguousarray(np.atleast_1d(np.asarray(epochs, np.float64)))
        K = int(epochs.size)
        states, stm = np.empty((K, 6, n)), np.empty((K, 6, 8, n))
        st = np.empty(n, dtype=np.int32)
    a = _lib.Args()
    args = [a.ptr(pos), a.ptr(vel), a.ptr(jd0), K, a.ptr(epochs), int(frame), int(center),
            int(bool(include_asteroids)), a.ptr(nongrav), a.ptr(states), a.ptr(stm),
            a.ptr(st, np.int32)]
    _lib.check(L.kete_b200_propagate_n_body_stm(n, *args, a.on_device, a.stream))
    return states, stm, st


class Checkpoints:
    """What the adjoint pass needs from a checkpointed forward pass."""

    def __init__(self, n, epochs, frame, include_asteroids, nongrav, capacity, ckpt, count,
                 segment, status):
        self.n, self.epochs, self.frame = n, epochs, frame
        self.include_asteroids, self.nongrav, self.capacity = include_asteroids, nongrav, capacity
        self.ckpt, self.count, self.segment, self.status = ckpt, count, segment, status


def _default_capacity(jd0, epochs):
    """Checkpoints per object for spans of at least 1 day per attempt on average."""
    e = np.asarray(epochs.detach().cpu() if hasattr(epochs, "detach") else epochs, np.float64)
    j = np.asarray(jd0.detach().cpu() if hasattr(jd0, "detach") else jd0, np.float64)
    span = np.abs(e[0] - j).max() + np.abs(np.diff(e)).sum() if e.size else 0.0
    return int(e.size + np.ceil(span / SENS_CK_ATTEMPTS) + 2)


def propagate_n_body_checkpointed(pos, vel, jd0, epochs, frame=Frames.Ecliptic, center=10,
                                  include_asteroids=False, nongrav=None, capacity=None):
    """Forward pass of the reverse-mode gradient: states (K, 6, n), status (n,) and the
    Checkpoints for ``propagate_n_body_adjoint``.  Objects that need more checkpoints than
    the capacity are re-run once with the capacity they reported."""
    _lib.init()
    L = _bind()
    n = int(pos.shape[1])
    dev = _lib._is_torch_cuda(pos)
    if dev:
        import torch

        if not _lib._is_torch_cuda(epochs):
            epochs = torch.as_tensor(np.asarray(epochs, np.float64), device=pos.device)
        K = int(epochs.shape[0])
    else:
        epochs = np.ascontiguousarray(np.atleast_1d(np.asarray(epochs, np.float64)))
        K = int(epochs.size)
    cap = int(capacity or _default_capacity(jd0, epochs))
    stride = checkpoint_doubles()
    for _ in range(2):
        if dev:
            states = torch.empty((K, 6, n), dtype=torch.float64, device=pos.device)
            st = torch.empty(n, dtype=torch.int32, device=pos.device)
            ck = torch.empty((n, cap, stride), dtype=torch.float64, device=pos.device)
            cnt = torch.empty(n, dtype=torch.int32, device=pos.device)
            seg = torch.empty((K, n), dtype=torch.int32, device=pos.device)
        else:
            states, st = np.empty((K, 6, n)), np.empty(n, dtype=np.int32)
            ck = np.empty((n, cap, stride))
            cnt, seg = np.empty(n, dtype=np.int32), np.empty((K, n), dtype=np.int32)
        a = _lib.Args()
        args = [a.ptr(pos), a.ptr(vel), a.ptr(jd0), K, a.ptr(epochs), int(frame), int(center),
                int(bool(include_asteroids)), a.ptr(nongrav), a.ptr(states), a.ptr(st, np.int32),
                cap, a.ptr(ck), a.ptr(cnt, np.int32), a.ptr(seg, np.int32)]
        _lib.check(L.kete_b200_propagate_n_body_checkpointed(n, *args, a.on_device, a.stream))
        full = (st == CHECKPOINT_FULL)
        if not bool(full.any()):
            break
        cap = int(cnt.max())
    return states, st, Checkpoints(n, epochs, frame, include_asteroids, nongrav, cap, ck, cnt, seg,
                                   st)


def propagate_n_body_adjoint(ck: Checkpoints, seed):
    """dL/d(pos0, vel0, A1, A2) (8, n) from seed = dL/d(states) (K, 6, n); also the
    adjoint pass's own status (n,)."""
    L = _bind()
    n = ck.n
    K = int(ck.epochs.shape[0])
    # the library reads these extents through raw pointers: check them here
    if tuple(ck.ckpt.shape) != (n, ck.capacity, checkpoint_doubles()):
        raise ValueError("checkpoint array does not match its capacity")
    if tuple(seed.shape) != (K, 6, n):
        raise ValueError(f"seed must have shape ({K}, 6, {n})")
    if (tuple(ck.count.shape) != (n,) or tuple(ck.segment.shape) != (K, n)
            or tuple(ck.status.shape) != (n,)):
        raise ValueError("checkpoint bookkeeping arrays do not match")
    if _lib._is_torch_cuda(ck.ckpt):
        import torch

        grad = torch.empty((8, n), dtype=torch.float64, device=ck.ckpt.device)
        gst = torch.empty(n, dtype=torch.int32, device=ck.ckpt.device)
        seed = seed.to(torch.float64).contiguous()
    else:
        grad, gst = np.empty((8, n)), np.empty(n, dtype=np.int32)
        seed = np.ascontiguousarray(seed, dtype=np.float64)
    a = _lib.Args()
    args = [K, a.ptr(ck.epochs), int(ck.frame), int(bool(ck.include_asteroids)),
            a.ptr(ck.nongrav), ck.capacity, a.ptr(ck.ckpt), a.ptr(ck.count, np.int32),
            a.ptr(ck.segment, np.int32), a.ptr(ck.status, np.int32), a.ptr(seed), a.ptr(grad),
            a.ptr(gst, np.int32)]
    _lib.check(L.kete_b200_propagate_n_body_adjoint(n, *args, a.on_device, a.stream))
    return grad, gst


def _torch_function():
    import torch

    class NBodyStates(torch.autograd.Function):
        """States (K, 6, n) at `epochs` as a differentiable function of the initial
        position (3, n), velocity (3, n) and JPL comet A1, A2 (n,) of each object."""

        @staticmethod
        def forward(ctx, pos0, vel0, a1, a2, jd0, epochs, frame, center, nongrav_rest, method):
            ng = nongrav_rest.detach().clone()
            ng[1] = a1.detach()
            ng[2] = a2.detach()
            ng = ng.contiguous()
            p0, v0 = pos0.detach().contiguous(), vel0.detach().contiguous()
            ctx.method = method
            if method == "stm":
                states, stm, st = propagate_n_body_stm_arrays(p0, v0, jd0, epochs, frame, center,
                                                              False, ng)
                ctx.save_for_backward(stm)
            else:
                states, st, ck = propagate_n_body_checkpointed(p0, v0, jd0, epochs, frame, center,
                                                               False, ng)
                ctx.ck = ck
            ctx.status = st
            return states

        @staticmethod
        def backward(ctx, grad_states):
            if ctx.method == "stm":
                (stm,) = ctx.saved_tensors
                # d loss / d p = sum_k sum_c grad[k, c] * d state_c / d p
                g = torch.einsum("kcn,kcpn->pn", grad_states, stm)
            else:
                g, _ = propagate_n_body_adjoint(ctx.ck, grad_states)
            return g[0:3], g[3:6], g[6], g[7], None, None, None, None, None, None

    return NBodyStates


_NBody = None


def nbody_states(pos0, vel0, a1, a2, jd0, epochs, nongrav_rest=None, frame=Frames.Ecliptic,
                 center=10, method="adjoint"):
    """Differentiable predicted states (K, 6, n) (torch CUDA tensors in and out).

    nongrav_rest: (10, n) rows supplying the comet model's other terms (kind, A3, alpha, r0,
    m, n, k, dt = 0); defaults to the JPL comet defaults (nongrav.rs:97-109).  method:
    "adjoint" (reverse mode, checkpointed) or "stm" (forward sensitivities)."""
    global _NBody
    import torch

    if method not in ("adjoint", "stm"):
        raise ValueError("method must be 'adjoint' or 'stm'")
    if _NBody is None:
        _NBody = _torch_function()
    n = pos0.shape[1]
    if nongrav_rest is None:
        base = torch.tensor([1.0, 0.0, 0.0, 0.0, 0.1112620426, 2.808, 2.15, 5.093, 4.6142, 0.0],
                            dtype=torch.float64, device=pos0.device)
        nongrav_rest = base[:, None].expand(10, n).contiguous()
    return _NBody.apply(pos0, vel0, a1, a2, jd0, epochs, int(frame), int(center), nongrav_rest,
                        method)


def nbody_positions(pos0, vel0, a1, a2, jd0, epochs, nongrav_rest=None, frame=Frames.Ecliptic,
                    center=10, method="adjoint"):
    """Differentiable predicted positions (K, 3, n); see ``nbody_states``."""
    return nbody_states(pos0, vel0, a1, a2, jd0, epochs, nongrav_rest, frame, center,
                        method)[:, 0:3, :]


def radec(vec_eq):
    """Right ascension and declination (radians) of equatorial vectors (..., 3, n)."""
    import torch

    x, y, z = vec_eq[..., 0, :], vec_eq[..., 1, :], vec_eq[..., 2, :]
    r = torch.sqrt(x * x + y * y + z * z)
    return torch.atan2(y, x), torch.asin(z / r)


def ecliptic_to_equatorial_torch(v):
    """Rotate (..., 3, n) ecliptic vectors into the J2000 equatorial frame."""
    import torch

    c, s = np.cos(0.40909280422232897), np.sin(0.40909280422232897)
    R = torch.tensor([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]], dtype=v.dtype, device=v.device)
    return torch.einsum("ij,...jn->...in", R, v)
