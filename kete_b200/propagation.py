"""kete's propagation entry points on the GPU.

``propagate_two_body`` and ``propagate_n_body`` keep the signatures, argument meaning and
error behaviour of kete's PyO3 functions (src/kete/rust/kepler.rs:68-108 and
src/kete/rust/propagation.rs:70-151); the per-object rayon loop becomes one batched call
into libketeb200.so.  The ``*_arrays`` functions are the batched forms on SoA arrays
(numpy on the host or torch tensors already on the GPU).
"""
from __future__ import annotations

import ctypes as C
import sys
from dataclasses import dataclass

import numpy as np

from . import _lib
from .state import Frames, State, pack

GMS = 0.00029591220828411956


@dataclass(frozen=True)
class NonGravModel:
    """Non-gravitational force model (kete_core/propagation/nongrav.rs:12-61)."""

    row: tuple

    @staticmethod
    def new_comet(a1=0.0, a2=0.0, a3=0.0, alpha=0.1112620426, r_0=2.808, m=2.15, n=5.093,
                  k=4.6142, dt=0.0) -> "NonGravModel":
        """JPL comet model, defaults as src/kete/rust/nongrav.rs:106-130."""
        return NonGravModel((1.0, a1, a2, a3, alpha, r_0, m, n, k, dt))

    @staticmethod
    def new_asteroid(a1, a2, a3, alpha=1.0, r_0=1.0, m=2.0, n=1.0, k=0.0, dt=0.0):
        """JPL model with g(r) = 1/r^2 defaults (src/kete/rust/nongrav.rs:132-157)."""
        return NonGravModel((1.0, a1, a2, a3, alpha, r_0, m, n, k, dt))

    @staticmethod
    def new_dust(beta: float) -> "NonGravModel":
        """Radiation pressure + Poynting-Robertson model (nongrav.rs:91-94)."""
        return NonGravModel((2.0, beta, 0, 0, 0, 0, 0, 0, 0, 0))


def _status_error(code: int, what: str):
    return ValueError(f"{what}: {_lib.STATUS_NAMES.get(int(code), code)}")


# ------------------------------------------------------------------------------------------
# array forms
# ------------------------------------------------------------------------------------------
def _alloc_like(template, shape, dtype):
    if _lib._is_torch_cuda(template):
        import torch

        tdt = {np.float64: torch.float64, np.int32: torch.int32}[dtype]
        return torch.empty(shape, dtype=tdt, device=template.device)
    return np.empty(shape, dtype=dtype)


def _out_array(given, template, shape, dtype, name):
    """A caller's output array (checked: shape, dtype, contiguous, the inputs' side), or a new
    one like ``template``."""
    if given is None:
        return _alloc_like(template, shape, dtype)
    if not (isinstance(given, np.ndarray) or _lib._is_torch_cuda(given)):
        raise ValueError(f"{name}: expected a numpy array or a CUDA tensor")
    if tuple(given.shape) != tuple(shape):
        raise ValueError(f"{name}: expected shape {tuple(shape)}, got {tuple(given.shape)}")
    if _lib._is_torch_cuda(given) != _lib._is_torch_cuda(template):
        raise ValueError(f"{name}: output and inputs must live on the same side")
    if _lib._is_torch_cuda(given):
        import torch

        tdt = {np.float64: torch.float64, np.int32: torch.int32}[dtype]
        if given.dtype != tdt or not given.is_contiguous():
            raise ValueError(f"{name}: expected a contiguous {tdt} tensor")
    elif (not isinstance(given, np.ndarray) or given.dtype != dtype
          or not given.flags.c_contiguous):
        raise ValueError(f"{name}: expected a C-contiguous numpy array of "
                         f"{np.dtype(dtype).name}")
    return given


def propagate_two_body_arrays(pos, vel, jd0, jd1, observer_pos=None):
    """Two-body propagation of n Sun-centred states (SoA (3, n) arrays), object i from
    jd0[i] to jd1[i].  Returns (pos, vel, jd, status)."""
    n = int(pos.shape[1])
    _lib.init()
    out_p = _alloc_like(pos, (3, n), np.float64)
    out_v = _alloc_like(pos, (3, n), np.float64)
    out_j = _alloc_like(pos, (n,), np.float64)
    st = _alloc_like(pos, (n,), np.int32)
    a = _lib.Args()
    args = [a.ptr(pos), a.ptr(vel), a.ptr(jd0), a.ptr(jd1), a.ptr(observer_pos), a.ptr(out_p),
            a.ptr(out_v), a.ptr(out_j), a.ptr(st, np.int32)]
    _lib.check(_lib.lib().kete_b200_propagate_two_body(n, *args, a.on_device, a.stream))
    return out_p, out_v, out_j, st


def propagate_n_body_arrays(pos, vel, jd0, jd1, frame=Frames.Ecliptic, center=10,
                            include_asteroids=False, nongrav=None, mode=_lib.MODE_AUTO,
                            with_details=False, out=None):
    """N-body Radau propagation of n states sharing ``frame`` and ``center``.

    pos/vel: (3, n); jd0/jd1: (n,); nongrav: None or (10, n) rows.  Returns
    (pos, vel, status) and, with ``with_details``, a dict with impact_id, impact_jd,
    min_dist and counters (3, n: accepted steps, corrector iterations, exact evals).
    ``out``: None, or the (pos (3, n) float64, vel (3, n) float64, status (n,) int32) arrays
    to write the results into, on the inputs' side (host arrays in pinned memory that a
    caller reuses across calls are copied back at full bus speed)."""
    n = int(pos.shape[1])
    _lib.init()
    o_p, o_v, o_s = out if out is not None else (None, None, None)
    out_p = _out_array(o_p, pos, (3, n), np.float64, "out[0]")
    out_v = _out_array(o_v, pos, (3, n), np.float64, "out[1]")
    st = _out_array(o_s, pos, (n,), np.int32, "out[2]")
    det = None
    if with_details:
        det = dict(impact_id=_alloc_like(pos, (n,), np.int32),
                   impact_jd=_alloc_like(pos, (n,), np.float64),
                   min_dist=_alloc_like(pos, (n,), np.float64),
                   counters=_alloc_like(pos, (3, n), np.int32))
    a = _lib.Args()
    args = [a.ptr(pos), a.ptr(vel), a.ptr(jd0), a.ptr(jd1)]
    ng = a.ptr(nongrav)
    outs = [a.ptr(out_p), a.ptr(out_v), a.ptr(st, np.int32)]
    if det:
        extra = [a.ptr(det["impact_id"], np.int32), a.ptr(det["impact_jd"]),
                 a.ptr(det["min_dist"]), a.ptr(det["counters"], np.int32)]
    else:
        extra = [None, None, None, None]
    _lib.check(_lib.lib().kete_b200_propagate_n_body(
        n, *args, int(frame), int(center), int(bool(include_asteroids)), ng, *outs, *extra,
        int(mode), a.on_device, a.stream))
    if with_details:
        return out_p, out_v, st, det
    return out_p, out_v, st


# body lists of vec_accel_arrays, with their NAIF ids in order (constants/gravity.rs:43-153)
BODY_LISTS = {
    "planets": (0, (10, 1, 2, 399, 301, 4, 5, 6, 7, 8)),
    "masses": (1, (10, 1, 2, 399, 301, 4, 5, 6, 7, 8, 20000001, 20000002, 20000004, 20000010,
                   20000704)),
    "simple_planets": (2, (10, 1, 2, 3, 4, 5, 6, 7, 8)),
}


def spk_accel_arrays(jd, pos, vel, include_asteroids=False, nongrav=None, exact=False):
    """spk_accel (kete_core/propagation/acceleration.rs:121-168) at n points.

    jd (n,); pos/vel (3, n) relative to the solar-system barycentre, equatorial; nongrav None
    or (10, n).  Returns (acc (3, n), status (n,), impact_id (n,))."""
    n = int(pos.shape[1])
    _lib.init()
    out = _alloc_like(pos, (3, n), np.float64)
    st = _alloc_like(pos, (n,), np.int32)
    iid = _alloc_like(pos, (n,), np.int32)
    a = _lib.Args()
    L = _lib.lib()
    v = C.c_void_p
    L.kete_b200_spk_accel.argtypes = [C.c_int64, v, v, v, C.c_int, v, C.c_int, v, v, v, C.c_int,
                                      v]
    _lib.check(L.kete_b200_spk_accel(n, a.ptr(jd), a.ptr(pos), a.ptr(vel),
                                     int(bool(include_asteroids)), a.ptr(nongrav), int(exact),
                                     a.ptr(out), a.ptr(st, np.int32), a.ptr(iid, np.int32),
                                     a.on_device, a.stream))
    return out, st, iid


def vec_accel_arrays(massive, pos, vel, bodies="planets", nongrav=None, exact=False):
    """vec_accel (acceleration.rs:197-249) on n test particles under massive bodies.

    massive (6, m): barycentric equatorial states of the list ``bodies`` ("planets",
    "masses" or "simple_planets", ids in BODY_LISTS) in its order; pos/vel (3, n).  Returns
    (acc (3, n), status (n,), impact_id (n,))."""
    code, ids = BODY_LISTS[bodies]
    if tuple(massive.shape) != (6, len(ids)):
        raise ValueError(f"massive must be (6, {len(ids)}) for {bodies}")
    n = int(pos.shape[1])
    _lib.init()
    out = _alloc_like(pos, (3, n), np.float64)
    st = _alloc_like(pos, (n,), np.int32)
    iid = _alloc_like(pos, (n,), np.int32)
    a = _lib.Args()
    L = _lib.lib()
    v = C.c_void_p
    L.kete_b200_vec_accel.argtypes = [C.c_int64, C.c_int, v, v, v, v, C.c_int, v, v, v, C.c_int,
                                      v]
    _lib.check(L.kete_b200_vec_accel(n, code, a.ptr(massive), a.ptr(pos), a.ptr(vel),
                                     a.ptr(nongrav), int(exact), a.ptr(out),
                                     a.ptr(st, np.int32), a.ptr(iid, np.int32), a.on_device,
                                     a.stream))
    return out, st, iid


def radau_central_arrays(pos, vel, t0, t1):
    """RadauIntegrator with the Sun-only force (kete_core/propagation/mod.rs:126-138)."""
    n = int(pos.shape[1])
    _lib.init()
    out_p = _alloc_like(pos, (3, n), np.float64)
    out_v = _alloc_like(pos, (3, n), np.float64)
    st = _alloc_like(pos, (n,), np.int32)
    a = _lib.Args()
    args = [a.ptr(pos), a.ptr(vel), a.ptr(t0), a.ptr(t1), a.ptr(out_p), a.ptr(out_v),
            a.ptr(st, np.int32)]
    _lib.check(_lib.lib().kete_b200_radau_central(n, *args, a.on_device, a.stream))
    return out_p, out_v, st


# ------------------------------------------------------------------------------------------
# kete-compatible State API
# ------------------------------------------------------------------------------------------
def _jd(jd) -> float:
    return float(getattr(jd, "jd", jd))


def propagate_two_body(states, jd, observer_pos=None):
    """kete.propagate_two_body (src/kete/rust/kepler.rs:68-108).

    States are moved to the Sun-centred frame they came in, propagated to ``jd`` (with
    the light delay to ``observer_pos`` when given) and returned with their original
    centre.  Failures give NaN states, as in the reference."""
    jd = _jd(jd)
    states = list(states)
    if not states:
        return []
    from . import spice

    out = [None] * len(states)
    groups = {}
    for i, s in enumerate(states):
        groups.setdefault((int(s.frame), int(s.center_id)), []).append(i)
    for (frame, center), idx in groups.items():
        sub = [states[i] for i in idx]
        pos, vel, jd0 = pack(sub)
        ok = np.ones(len(sub), dtype=bool)
        if center != 10:
            shift0 = spice._center_shift(center, 10, jd0, frame)
            ok &= shift0["ok"]
            pos = pos - shift0["pos"]
            vel = vel - shift0["vel"]
        jd1 = np.full(len(sub), jd)
        obs = None if observer_pos is None else np.asarray(observer_pos, dtype=np.float64).reshape(3).copy()
        p, v, ojd, st = propagate_two_body_arrays(pos, vel, jd0, jd1, obs)
        if center != 10:
            shift1 = spice._center_shift(center, 10, ojd, frame)
            ok &= shift1["ok"]
            p = p + shift1["pos"]
            v = v + shift1["vel"]
        for k, i in enumerate(idx):
            s = states[i]
            if st[k] != 0 or not ok[k]:
                out[i] = State.new_nan(s.desig, jd, s.frame, s.center_id)
            else:
                out[i] = State(s.desig, float(ojd[k]), p[:, k], v[:, k], s.frame, s.center_id)
    return out


def propagate_n_body(states, jd, include_asteroids=False, non_gravs=None, suppress_errors=True,
                     suppress_impact_errors=False):
    """kete.propagate_n_body (src/kete/rust/propagation.rs:70-151)."""
    jd = _jd(jd)
    states = list(states)
    if non_gravs is None:
        non_gravs = [None] * len(states)
    non_gravs = list(non_gravs)
    if len(non_gravs) != len(states):
        raise ValueError("non_gravs must be the same length as states.")
    out = [None] * len(states)
    groups = {}
    for i, s in enumerate(states):
        if not s.is_finite:
            if not suppress_errors:
                raise ValueError("Input state contains NaNs.")
            out[i] = State.new_nan(s.desig, jd, s.frame, s.center_id)
            continue
        groups.setdefault((int(s.frame), int(s.center_id)), []).append(i)
    for (frame, center), idx in groups.items():
        sub = [states[i] for i in idx]
        pos, vel, jd0 = pack(sub)
        ng = None
        if any(non_gravs[i] is not None for i in idx):
            ng = np.zeros((10, len(sub)))
            for k, i in enumerate(idx):
                if non_gravs[i] is not None:
                    ng[:, k] = non_gravs[i].row
        jd1 = np.full(len(sub), jd)
        p, v, st, det = propagate_n_body_arrays(pos, vel, jd0, jd1, frame, center,
                                                include_asteroids, ng, with_details=True)
        for k, i in enumerate(idx):
            s = states[i]
            if st[k] == 0:
                out[i] = State(s.desig, jd, p[:, k], v[:, k], s.frame, s.center_id)
                continue
            if not suppress_errors:
                raise _status_error(st[k], f"propagation of {s.desig!r} failed")
            if st[k] == _lib.IMPACT and not suppress_impact_errors:
                print(f"Impact detected between ({s.desig!r}) <-> ({int(det['impact_id'][k])}) "
                      f"at time {float(det['impact_jd'][k])}", file=sys.stderr)
            out[i] = State.new_nan(s.desig, jd, s.frame, s.center_id)
    return out


SIMPLE_PLANET_IDS = (10, 1, 2, 3, 4, 5, 6, 7, 8)


def propagate_n_body_long_arrays(pos, vel, jd0, jd1, planets=None, nongrav=None, batch_size=10):
    """propagate_n_body_vec on arrays: pos/vel (3, n) heliocentric equatorial at jd0;
    planets None (read from the loaded SPK) or (9, 6) heliocentric equatorial states of the
    SIMPLE_PLANETS at jd0.  Returns (pos, vel, planets (9, 6), status), heliocentric
    equatorial at jd1.  Host numpy arrays or torch CUDA tensors."""
    _lib.init()
    n = int(pos.shape[1])
    out_p = _alloc_like(pos, (3, n), np.float64)
    out_v = _alloc_like(pos, (3, n), np.float64)
    out_pl = _alloc_like(pos, (9, 6), np.float64)
    st = _alloc_like(pos, (n,), np.int32)
    a = _lib.Args()
    v = _lib.C.c_void_p
    L = _lib.lib()
    L.kete_b200_propagate_n_body_long.argtypes = [_lib.C.c_int64, v, v, _lib.C.c_double,
                                                  _lib.C.c_double, v, v, _lib.C.c_int, v, v, v,
                                                  v, _lib.C.c_int, v]
    args = [a.ptr(pos), a.ptr(vel), float(jd0), float(jd1), a.ptr(planets), a.ptr(nongrav),
            int(batch_size), a.ptr(out_p), a.ptr(out_v), a.ptr(out_pl), a.ptr(st, np.int32)]
    _lib.check(L.kete_b200_propagate_n_body_long(n, *args, a.on_device, a.stream))
    return out_p, out_v, out_pl, st


def propagate_n_body_long(states, jd_final, planet_states=None, non_gravs=None, batch_size=10):
    """kete.propagate_n_body_long (src/kete/rust/propagation.rs:203-249 over
    propagate_n_body_vec, kete_core/propagation/mod.rs:142-237): the states (one common
    epoch, centred on the Sun) integrated together with the Sun, the planets and the
    Earth-Moon barycentre, batch_size objects per integration.  Returns (states, planets)
    at jd_final, heliocentric J2000 equatorial."""
    from .state import ecliptic_to_equatorial

    jd1 = _jd(jd_final)
    states = list(states)
    if not states:
        return [], []
    if non_gravs is None:
        non_gravs = [None] * len(states)
    non_gravs = list(non_gravs)
    if len(non_gravs) != len(states):
        raise ValueError("Number of non-grav models doesnt match the number of provided objects.")
    jd0 = states[0].jd
    n = len(states)
    pos, vel = np.empty((3, n)), np.empty((3, n))
    for i, s in enumerate(states):
        if s.jd != jd0:
            raise ValueError("All input states must have the same JD")
        if int(s.center_id) != 10:
            raise ValueError("Center of all states must be 10 (the Sun).")
        p, v = np.asarray(s.pos, float), np.asarray(s.vel, float)
        if Frames(s.frame) == Frames.Ecliptic:
            p, v = ecliptic_to_equatorial(p), ecliptic_to_equatorial(v)
        pos[:, i], vel[:, i] = p, v
    planets, names = None, list(SIMPLE_PLANET_IDS)
    if planet_states is not None:
        planet_states = list(planet_states)
        if len(planet_states) != len(SIMPLE_PLANET_IDS):
            raise ValueError("Input planet states must contain the correct number of states.")
        if planet_states[0].jd != jd0:
            raise ValueError("Planet states JD must match JD of input state.")
        planets = np.empty((9, 6))
        for k, ps in enumerate(planet_states):
            p, v = np.asarray(ps.pos, float), np.asarray(ps.vel, float)
            if Frames(ps.frame) == Frames.Ecliptic:
                p, v = ecliptic_to_equatorial(p), ecliptic_to_equatorial(v)
            planets[k, :3], planets[k, 3:] = p, v
        names = [ps.desig for ps in planet_states]
    ng = None
    if any(m is not None for m in non_gravs):
        ng = np.zeros((10, n))
        for i, m in enumerate(non_gravs):
            if m is not None:
                ng[:, i] = m.row
    p, v, pl, st = propagate_n_body_long_arrays(pos, vel, jd0, jd1, planets, ng, batch_size)
    bad = np.nonzero(st != 0)[0]
    if bad.size:
        raise _status_error(st[bad[0]], f"propagation of {states[bad[0]].desig!r} failed")
    out = [State(s.desig, jd1, p[:, i], v[:, i], Frames.Equatorial, 10)
           for i, s in enumerate(states)]
    planets_out = [State(names[k], jd1, pl[k, :3], pl[k, 3:], Frames.Equatorial, 10)
                   for k in range(9)]
    return out, planets_out
