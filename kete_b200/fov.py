"""kete's field-of-view checks on the GPU.

``RectangleFOV`` mirrors kete's RectangleFOV (src/kete/rust/fovs/definitions.rs:400-418 over
GenericRectangle, kete_core/fov/generic.rs:14-62) and ``fov_state_check`` mirrors
src/kete/rust/fovs/checks.rs:24-110: fields are sorted by epoch, grouped into chunks shorter
than 2*dt_limit, the population is re-propagated with the reference's big-step / small-step
schedule (N-body, on the GPU), and each chunk's fields are checked for all objects in one
call of ``kete_b200_fov_check_visible``.  Objects whose propagation fails are dropped from
then on, as the reference's ``filter_map`` drops them.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .propagation import propagate_n_body_arrays
from .state import Frames, SimultaneousStates, State, ecliptic_to_equatorial, equatorial_to_ecliptic

FOV_STRIDE = 19


# ------------------------------------------------------------------------------------------
# OnSkyRectangle::new (kete_core/fov/patches.rs:122-155), evaluated in the same operation
# order as nalgebra (Rotation3::from_axis_angle, frames/definitions.rs:356-363).
# ------------------------------------------------------------------------------------------
def _rotate_around(v, axis, angle):
    if angle == 0.0:  # from_axis_angle gives the identity for a zero angle
        return list(v)
    n = math.sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2])
    ux, uy, uz = axis[0] / n, axis[1] / n, axis[2] / n
    sqx, sqy, sqz = ux * ux, uy * uy, uz * uz
    s, c = math.sin(angle), math.cos(angle)
    omc = 1.0 - c
    m = [[sqx + (1.0 - sqx) * c, ux * uy * omc - uz * s, ux * uz * omc + uy * s],
         [ux * uy * omc + uz * s, sqy + (1.0 - sqy) * c, uy * uz * omc - ux * s],
         [ux * uz * omc - uy * s, uy * uz * omc + ux * s, sqz + (1.0 - sqz) * c]]
    return [(v[0] * m[i][0] + v[1] * m[i][1]) + v[2] * m[i][2] for i in range(3)]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def rect_normals(pointing, rotation, lon_width, lat_width):
    """Edge normals (4 x 3) of OnSkyRectangle::new; angles in radians."""
    p = [float(x) for x in pointing]
    up0 = _rotate_around([0.0, 0.0, 1.0], p, -rotation)
    left = _cross(p, up0)
    up = _cross(p, left)
    n1 = _rotate_around(left, up, -lon_width / 2.0)
    n2 = _rotate_around(up, left, lat_width / 2.0)
    n3 = _rotate_around([-x for x in left], up, lon_width / 2.0)
    n4 = _rotate_around([-x for x in up], left, -lat_width / 2.0)
    return np.array([n1, n2, n3, n4])


class RectangleFOV:
    """Rectangular field: pointing vector, rotation and widths in degrees, observer State
    (src/kete/rust/fovs/definitions.rs:400-418)."""

    def __init__(self, pointing, rotation, observer: State, lon_width, lat_width):
        self.observer = observer
        self.pointing = np.asarray(pointing, dtype=np.float64).reshape(3)
        self.rotation = float(rotation)
        self.lon_width = float(lon_width)
        self.lat_width = float(lat_width)
        d2r = math.pi / 180.0  # f64::to_radians
        self.normals = rect_normals(self.pointing, self.rotation * d2r, self.lon_width * d2r,
                                    self.lat_width * d2r)

    @property
    def jd(self) -> float:
        return self.observer.jd

    def ecliptic_column(self):
        """The field as one column of the device table: observer jd, pos, vel, normals
        (converted to the ecliptic frame as FOVListLike::into_sorted_vec_fov does)."""
        o = self.observer
        pos, vel, nrm = o.pos, o.vel, self.normals
        if Frames(o.frame) == Frames.Equatorial:
            pos, vel = equatorial_to_ecliptic(pos), equatorial_to_ecliptic(vel)
            nrm = np.array([equatorial_to_ecliptic(x) for x in nrm])
        return np.concatenate([[o.jd], pos, vel, np.asarray(nrm).reshape(12)])


def _bind():
    L = _lib.lib()
    v = ctypes.c_void_p
    L.kete_b200_fov_check_visible.argtypes = [ctypes.c_int64, v, v, v, v, ctypes.c_int64, v,
                                              ctypes.c_double, ctypes.c_int, ctypes.c_int64, v, v,
                                              v, v, ctypes.c_int, v]
    return L


def fov_check_visible_arrays(pos, vel, jd, valid, fov_table, dt_limit=3.0,
                             include_asteroids=False, capacity=None):
    """Visibility of n objects (SoA (3, n) at epochs jd (n,), valid (n,) uint8 or None) in
    the fields of fov_table (19, F).  Host numpy arrays or torch CUDA tensors.

    Returns (fov_index, obj_index, state7) as numpy arrays sorted by field, then object."""
    _lib.init()
    L = _bind()
    n = int(pos.shape[1])
    F = int(fov_table.shape[1])
    cap = int(capacity or max(1024, n // 8))
    on_dev = _lib._is_torch_cuda(pos)
    for _ in range(3):
        if on_dev:
            import torch

            out_f = torch.empty(cap, dtype=torch.int32, device=pos.device)
            out_o = torch.empty(cap, dtype=torch.int32, device=pos.device)
            out_s = torch.empty((7, cap), dtype=torch.float64, device=pos.device)
        else:
            out_f, out_o = np.empty(cap, dtype=np.int32), np.empty(cap, dtype=np.int32)
            out_s = np.empty((7, cap))
        nvis = ctypes.c_int64(0)
        a = _lib.Args()
        args = [a.ptr(pos), a.ptr(vel), a.ptr(jd), a.ptr(valid, np.uint8) if valid is not None
                else None, F, a.ptr(fov_table), float(dt_limit), int(bool(include_asteroids)),
                cap, a.ptr(out_f, np.int32), a.ptr(out_o, np.int32), a.ptr(out_s)]
        _lib.check(L.kete_b200_fov_check_visible(n, *args, ctypes.byref(nvis), a.on_device,
                                                 a.stream))
        m = nvis.value
        if m <= cap:
            break
        cap = m + 1024
    if on_dev:
        out_f, out_o, out_s = out_f[:m].cpu().numpy(), out_o[:m].cpu().numpy(), out_s[:, :m].cpu().numpy()
    else:
        out_f, out_o, out_s = out_f[:m], out_o[:m], out_s[:, :m]
    order = np.lexsort((out_o, out_f))
    return out_f[order], out_o[order], out_s[:, order]


def chunk_bounds(jds, dt_limit):
    """Start indices of the chunks of time-sorted field epochs (checks.rs:37-57): a chunk
    closes when the next field is 2*dt_limit or more after the chunk's first field."""
    starts = []
    first = None
    for k, jd in enumerate(jds):
        if first is None or abs(jd - first) >= 2.0 * dt_limit:
            starts.append(k)
            first = jd
    return starts + [len(jds)]


def fov_state_check_arrays(pos, vel, jd, fov_table, dt_limit=3.0, include_asteroids=False,
                           nongrav=None, on_chunk=None):
    """The fov_state_check schedule (src/kete/rust/fovs/checks.rs:24-110) on device arrays.

    pos/vel (3, n) heliocentric ecliptic torch CUDA tensors at the common epoch ``jd``;
    fov_table (19, F) columns sorted by observer epoch (row 0).  Chunks of fields shorter
    than 2*dt_limit are checked against the population re-propagated (N-body) to the
    chunk's mean epoch, re-seeded from a big-step copy every 25-50 dt_limit as the
    reference does; objects whose propagation fails are dropped from then on.  Returns
    (fov_index, obj_index, state7) numpy arrays over all fields, sorted by field then
    object.  ``on_chunk(k0, k1)``, when given, is called after each chunk."""
    import torch

    n = int(pos.shape[1])
    dev = pos.device
    table = fov_table if _lib._is_torch_cuda(fov_table) else torch.as_tensor(
        np.ascontiguousarray(fov_table), device=dev)
    jds = table[0].cpu().numpy()
    if np.any(np.diff(jds) < 0):
        raise ValueError("fields must be sorted by epoch")

    class Pop:
        def __init__(self, P, V, ok, t):
            self.P, self.V, self.ok, self.t = P, V, ok, t

        def copy(self):
            return Pop(self.P.clone(), self.V.clone(), self.ok.clone(), self.t)

        def propagate(self, target):
            jd0 = torch.full((n,), self.t, dtype=torch.float64, device=dev)
            jd1 = torch.full((n,), target, dtype=torch.float64, device=dev)
            P, V, st = propagate_n_body_arrays(self.P, self.V, jd0, jd1, Frames.Ecliptic, 10,
                                               include_asteroids, nongrav)
            self.P, self.V, self.t = P, V, target
            self.ok = self.ok & (st == 0)

    cur_jd = float(jd)
    big_jd = cur_jd
    cur = Pop(pos, vel, torch.ones(n, dtype=torch.bool, device=dev), cur_jd)
    big = cur.copy()
    out_f, out_o, out_s = [], [], []
    bounds = chunk_bounds(jds, dt_limit)
    for k0, k1 in zip(bounds[:-1], bounds[1:]):
        jd_mean = (jds[k1 - 1] + jds[k0]) / 2.0
        if abs(jd_mean - big_jd) >= dt_limit * 50.0:
            big_jd = jd_mean
            big.propagate(cur_jd)  # the reference propagates the big step to the current jd
        if abs(jd_mean - cur_jd) >= dt_limit:
            if abs(cur_jd - big_jd) >= dt_limit * 25.0:
                cur = big.copy()
            cur_jd = jd_mean
            cur.propagate(cur_jd)
        epochs = torch.full((n,), cur.t, dtype=torch.float64, device=dev)
        ff, oo, ss = fov_check_visible_arrays(cur.P, cur.V, epochs, cur.ok.to(torch.uint8),
                                              table[:, k0:k1].contiguous(), dt_limit,
                                              include_asteroids)
        out_f.append(ff + k0)
        out_o.append(oo)
        out_s.append(ss)
        if on_chunk is not None:
            on_chunk(k0, k1)
    if not out_f:
        return np.empty(0, np.int32), np.empty(0, np.int32), np.empty((7, 0))
    return np.concatenate(out_f), np.concatenate(out_o), np.concatenate(out_s, axis=1)


def fov_state_check(obj_state, fovs, dt_limit=3.0, include_asteroids=False):
    """kete.fov_state_check: objects (SimultaneousStates, or a list of States sharing one
    epoch, heliocentric ecliptic) visible in each field; returns a list of
    SimultaneousStates, one per field with at least one visible object."""
    import torch

    states = list(obj_state.states if isinstance(obj_state, SimultaneousStates) else obj_state)
    if not states:
        return []
    fovs = sorted(list(fovs), key=lambda f: f.jd)
    n = len(states)
    pos = np.empty((3, n))
    vel = np.empty((3, n))
    for i, s in enumerate(states):
        p, v = s.pos, s.vel
        if Frames(s.frame) == Frames.Equatorial:
            p, v = equatorial_to_ecliptic(p), equatorial_to_ecliptic(v)
        pos[:, i], vel[:, i] = p, v
    desig = [s.desig for s in states]
    dev = torch.device("cuda", torch.cuda.current_device())
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    table = np.stack([f.ecliptic_column() for f in fovs], axis=1)
    ff, oo, ss = fov_state_check_arrays(T(pos), T(vel), states[0].jd, table, dt_limit,
                                        include_asteroids)
    results = []
    for k, f in enumerate(fovs):
        sel = np.nonzero(ff == k)[0]
        if sel.size == 0:
            continue
        vis = [State(desig[oo[j]], ss[0, j], ss[1:4, j], ss[4:7, j], Frames.Ecliptic, 10)
               for j in sel]
        results.append(SimultaneousStates(vis, f))
    return results
