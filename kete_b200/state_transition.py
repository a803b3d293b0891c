"""kete.state_transition on the GPU: two-body state-transition matrices and covariance
propagation (src/kete/state_transition.py:8-59).

``compute_stm`` returns d(pos1, vel1)/d(pos0, vel0) of kete's closed-form two-body
propagation, computed by the ``two_body_stm_kernel`` of libketeb200.so.  kete's own routine
(kete_core/propagation/state_transition.rs:52-122) integrates the variational equations
with a Jacobian off by a factor -1/2 (acceleration.rs:267-290), uses the unscaled GM in
scaled time, and returns the transpose; its Python wrapper also calls the binding with one
argument too few.  The matrix here is the one the two-body propagation has, and
``propagate_covariance`` returns Phi C Phi^T with it.

``propagate_covariance_n_body`` does the same through the N-body model with the forward
sensitivities of ``autodiff.propagate_n_body_stm_arrays`` (6 x 8: position, velocity and
the JPL comet A1, A2).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .state import Frames, State, pack


def _alloc_like(template, shape):
    if _lib._is_torch_cuda(template):
        import torch

        return torch.empty(shape, dtype=torch.float64, device=template.device)
    return np.empty(shape, dtype=np.float64)


def compute_stm_arrays(pos, vel, jd0, jd1, central_mass=1.0, covariance=None):
    """Batched two-body STMs of n Sun-centred states, object i from jd0[i] to jd1[i].

    pos/vel (3, n); jd0/jd1 (n,); covariance None or (6, 6, n).  Host numpy arrays or torch
    CUDA tensors (all on the same side).  Returns (pos (3, n), vel (3, n), stm (6, 6, n),
    covariance (6, 6, n) or None, status (n,))."""
    n = int(pos.shape[1])
    _lib.init()
    out_p, out_v = _alloc_like(pos, (3, n)), _alloc_like(pos, (3, n))
    out_m = _alloc_like(pos, (6, 6, n))
    out_c = None if covariance is None else _alloc_like(pos, (6, 6, n))
    if _lib._is_torch_cuda(pos):
        import torch

        st = torch.empty(n, dtype=torch.int32, device=pos.device)
    else:
        st = np.empty(n, dtype=np.int32)
        jd0 = np.ascontiguousarray(np.broadcast_to(np.asarray(jd0, np.float64), (n,)))
        jd1 = np.ascontiguousarray(np.broadcast_to(np.asarray(jd1, np.float64), (n,)))
    a = _lib.Args()
    L = _lib.lib()
    v = _lib.C.c_void_p
    L.kete_b200_compute_stm.argtypes = [_lib.C.c_int64, v, v, v, v, _lib.C.c_double] + [v] * 6 + [
        _lib.C.c_int, v]
    rc = L.kete_b200_compute_stm(n, a.ptr(pos), a.ptr(vel), a.ptr(jd0), a.ptr(jd1),
                                 float(central_mass), a.ptr(covariance), a.ptr(out_p),
                                 a.ptr(out_v), a.ptr(out_m), a.ptr(out_c), a.ptr(st, np.int32),
                                 a.on_device, a.stream)
    _lib.check(rc)
    return out_p, out_v, out_m, out_c, st


def covariance_transform_arrays(stm, covariance):
    """Phi C Phi^T per object: stm (rows, cols, n), covariance (cols, cols, n) -> (rows,
    rows, n), on the GPU."""
    rows, cols, n = (int(x) for x in stm.shape)
    _lib.init()
    out = _alloc_like(stm, (rows, rows, n))
    a = _lib.Args()
    L = _lib.lib()
    v = _lib.C.c_void_p
    L.kete_b200_covariance_transform.argtypes = [_lib.C.c_int64, _lib.C.c_int, _lib.C.c_int, v,
                                                 v, v, _lib.C.c_int, v]
    _lib.check(L.kete_b200_covariance_transform(n, rows, cols, a.ptr(stm), a.ptr(covariance),
                                                a.ptr(out), a.on_device, a.stream))
    return out


def _sun_centred(state: State):
    """(pos, vel) of the state about the Sun in its own frame (the STM does not depend on
    the centre's motion, which is added back at fixed epochs)."""
    pos, vel, jd0 = pack([state])
    if int(state.center_id) != 10:
        from . import spice

        shift = spice._center_shift(int(state.center_id), 10, jd0, int(state.frame))
        if not bool(shift["ok"][0]):
            raise ValueError("cannot move the state to the Sun's centre")
        pos, vel = pos - shift["pos"], vel - shift["vel"]
    return pos, vel, jd0


def compute_stm(state: State, jd_end: float, central_mass: float = 1.0) -> np.ndarray:
    """kete.compute_stm: the 6x6 two-body state-transition matrix of ``state`` to
    ``jd_end`` (columns: d/d(x, y, z, vx, vy, vz) at the start, in the state's frame)."""
    pos, vel, jd0 = _sun_centred(state)
    _, _, m, _, st = compute_stm_arrays(pos, vel, jd0, np.array([float(jd_end)]), central_mass)
    if st[0] != 0:
        raise ValueError("two-body propagation failed to converge")
    return np.array(m[:, :, 0])


def propagate_covariance(state: State, covariance, jd_end: float,
                         central_mass: float = 1.0) -> np.ndarray:
    """kete.propagate_covariance: the 6x6 covariance of [X, Y, Z, Vx, Vy, Vz] (AU, AU/day)
    moved to ``jd_end`` with the two-body STM, Phi C Phi^T."""
    cov = np.asarray(covariance, dtype=np.float64)
    if cov.shape != (6, 6):
        raise ValueError("covariance must be 6x6")
    pos, vel, jd0 = _sun_centred(state)
    _, _, _, c, st = compute_stm_arrays(pos, vel, jd0, np.array([float(jd_end)]), central_mass,
                                        np.ascontiguousarray(cov.reshape(6, 6, 1)))
    if st[0] != 0:
        raise ValueError("two-body propagation failed to converge")
    return np.array(c[:, :, 0])


def propagate_covariance_n_body(states, covariances, jd_end, include_asteroids=False,
                                non_gravs=None):
    """Covariances through the N-body model: each state's 6x6 covariance of (pos, vel), or
    8x8 of (pos, vel, A1, A2) with a JPL comet model, moved to ``jd_end`` with the forward
    sensitivities of the Radau propagation.  All states share frame and centre; returns a
    list of 6x6 matrices in that frame."""
    from . import autodiff

    states = list(states)
    n = len(states)
    if n == 0:
        return []
    frame, center = states[0].frame, states[0].center_id
    if any(s.frame != frame or s.center_id != center for s in states):
        raise ValueError("all states must share frame and centre")
    covs = np.asarray(covariances, dtype=np.float64)
    if covs.ndim != 3 or covs.shape[0] != n or covs.shape[1] != covs.shape[2] or \
            covs.shape[1] not in (6, 8):
        raise ValueError("covariances must be (n, 6, 6) or (n, 8, 8)")
    pos, vel, jd0 = pack(states)
    ng = None
    if non_gravs is not None:
        non_gravs = list(non_gravs)
        if len(non_gravs) != n:
            raise ValueError("non_gravs must be the same length as states.")
        if any(m is not None for m in non_gravs):
            ng = np.zeros((10, n))
            for i, m in enumerate(non_gravs):
                if m is not None:
                    ng[:, i] = m.row
    _, stm, st = autodiff.propagate_n_body_stm_arrays(pos, vel, jd0, [float(jd_end)], Frames(frame),
                                                      int(center), include_asteroids, ng)
    dim = covs.shape[1]
    phi = np.ascontiguousarray(stm[0, :, :dim, :])
    c = np.ascontiguousarray(np.transpose(covs, (1, 2, 0)))
    out = covariance_transform_arrays(phi, c)
    res = []
    for i in range(n):
        res.append(np.full((6, 6), np.nan) if st[i] != 0 else np.array(out[:, :, i]))
    return res
