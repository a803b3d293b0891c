"""Gradients of N-body predictions: forward sensitivities behind torch.autograd.

``propagate_n_body_stm_arrays`` runs kete's N-body propagation (src/kete_core/src/
propagation/mod.rs:70-118) through a sequence of epochs and returns, with each state, its
6 x 8 derivative with respect to the initial position, initial velocity and the JPL comet
A1/A2 parameters -- the exact derivative of the Radau steps the GPU executed (step sizes
held fixed).  ``NBodyPositions`` wraps it as a torch.autograd.Function, so losses built on
the predicted positions (e.g. RA/Dec residuals) differentiate with torch.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .state import Frames


def _bind():
    L = _lib.lib()
    v = ctypes.c_void_p
    L.kete_b200_propagate_n_body_stm.argtypes = [ctypes.c_int64, v, v, v, ctypes.c_int, v,
                                                 ctypes.c_int, ctypes.c_int64, ctypes.c_int, v, v,
                                                 v, v, ctypes.c_int, v]
    return L


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


def _torch_function():
    import torch

    class NBodyPositions(torch.autograd.Function):
        """Positions (K, 3, n) at `epochs` as a differentiable function of the initial
        position (3, n), velocity (3, n) and JPL comet A1, A2 (n,) of each object."""

        @staticmethod
        def forward(ctx, pos0, vel0, a1, a2, jd0, epochs, frame, center, nongrav_rest):
            ng = nongrav_rest.clone()
            ng[1] = a1
            ng[2] = a2
            states, stm, st = propagate_n_body_stm_arrays(pos0.detach().contiguous(),
                                                          vel0.detach().contiguous(), jd0,
                                                          epochs, frame, center, False,
                                                          ng.contiguous())
            ctx.save_for_backward(stm)
            ctx.status = st
            return states[:, 0:3, :].clone()

        @staticmethod
        def backward(ctx, grad_pos):
            (stm,) = ctx.saved_tensors
            # d loss / d p = sum_k sum_c grad_pos[k, c] * dpos_c/dp
            g = torch.einsum("kcn,kcpn->pn", grad_pos, stm[:, 0:3, :, :])
            return g[0:3], g[3:6], g[6], g[7], None, None, None, None, None

    return NBodyPositions


_NBody = None


def nbody_positions(pos0, vel0, a1, a2, jd0, epochs, nongrav_rest=None, frame=Frames.Ecliptic,
                    center=10):
    """Differentiable predicted positions (K, 3, n) (torch CUDA tensors in and out).

    nongrav_rest: (10, n) rows supplying the comet model's other terms (kind, A3, alpha, r0,
    m, n, k, dt); defaults to the JPL comet defaults (nongrav.rs:97-109)."""
    global _NBody
    import torch

    if _NBody is None:
        _NBody = _torch_function()
    n = pos0.shape[1]
    if nongrav_rest is None:
        base = torch.tensor([1.0, 0.0, 0.0, 0.0, 0.1112620426, 2.808, 2.15, 5.093, 4.6142, 0.0],
                            dtype=torch.float64, device=pos0.device)
        nongrav_rest = base[:, None].expand(10, n).contiguous()
    return _NBody.apply(pos0, vel0, a1, a2, jd0, epochs, int(frame), int(center), nongrav_rest)


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
