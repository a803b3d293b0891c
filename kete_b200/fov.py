"""kete's fields of view and visibility checks on the GPU.

Field types mirror kete's (src/kete/rust/fovs/definitions.rs over kete_core/fov):
``RectangleFOV`` (generic.rs:14-62), ``ConeFOV`` (generic.rs:140-190),
``OmniDirectionalFOV`` (generic.rs:97-135), ``WiseCmos`` (wise.rs), ``NeosCmos`` and the
four-chip ``NeosVisit`` (neos.rs), ``ZtfCcdQuad`` and the multi-quad ``ZtfField`` (ztf.rs).
Each is a list of sky patches (rectangles by their 4 edge normals, cones, or everything);
a field with several patches reports an object in its first patch that contains it
(closest_inside, patches.rs:21-35).

``fov_state_check`` mirrors src/kete/rust/fovs/checks.rs:24-110: fields are sorted by epoch,
grouped into chunks shorter than 2*dt_limit, the population is re-propagated with the
reference's big-step / small-step schedule (N-body, on the GPU), and each chunk's patches are
checked for all objects in one call of ``kete_b200_fov_check_visible``.  Objects whose
propagation fails are dropped from then on, as the reference's ``filter_map`` drops them.
``fov_spk_check`` and ``fov_static_check`` mirror checks.rs:111-188.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import _lib
from .propagation import propagate_n_body_arrays
from .state import Frames, SimultaneousStates, State, ecliptic_to_equatorial, equatorial_to_ecliptic

FOV_STRIDE = 20  # rows per patch column of the device table (KETE_B200_FOV_ROWS)
PATCH_RECTANGLE, PATCH_CONE, PATCH_OMNIDIRECTIONAL = 0, 1, 2
NEOS_WIDTH = 0.12391837689159739   # radians (kete_core/constants/neos.rs:8)
NEOS_HEIGHT = 0.029321531433504737  # radians (neos.rs:14)
WISE_WIDTH = 0.01367174580728       # radians (kete_core/constants/wise.rs:22)


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


def _normalize(v):
    n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return [v[0] / n, v[1] / n, v[2] / n]


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _polygon_pointing(normals):
    """SphericalPolygon::pointing (patches.rs:258-283): the normalised sum of the unit
    crossings of consecutive edge normals."""
    x = y = z = 0.0
    d = len(normals)
    for i in range(d):
        v = _normalize(_cross(normals[i], normals[(i + 1) % d]))
        x += v[0]
        y += v[1]
        z += v[2]
    return _normalize([x, y, z])


def rect_normals_from_corners(corners):
    """OnSkyRectangle::from_corners (patches.rs:157-180): edge normals of 4 corners given in
    order, flipped and reversed when they describe the far side of the sphere."""
    c = [[float(x) for x in v] for v in corners]
    n = [_normalize(_cross(c[i], c[(i + 1) % 4])) for i in range(4)]
    if math.copysign(1.0, _dot(c[0], _polygon_pointing(n))) < 0:
        n = [[-x for x in v] for v in n][::-1]
    return np.array(n)


def _to_ecliptic(v, frame):
    return equatorial_to_ecliptic(v) if Frames(frame) == Frames.Equatorial else np.asarray(v, float)


class _Field:
    """A field of view: an observer State and its sky patches, (kind, parameters) pairs in the
    observer's frame."""

    observer: State
    _patches: list

    @property
    def jd(self) -> float:
        return self.observer.jd

    def n_patches(self) -> int:
        return len(self._patches)

    def get_fov(self, idx: int = 0):
        """The single-patch field a detection in patch ``idx`` is reported against."""
        if idx != 0:
            raise IndexError("this field has a single patch")
        return self

    def columns(self):
        """Device-table columns of the patches (FOV_STRIDE values each): observer epoch,
        heliocentric ecliptic position and velocity, parameters, kind (converted to the
        ecliptic frame as FOVListLike::into_sorted_vec_fov does)."""
        o = self.observer
        pos, vel = _to_ecliptic(o.pos, o.frame), _to_ecliptic(o.vel, o.frame)
        cols = []
        for kind, prm in self._patches:
            p = np.zeros(12)
            if kind == PATCH_RECTANGLE:
                p[:] = np.concatenate([_to_ecliptic(v, o.frame) for v in np.asarray(prm).reshape(4, 3)])
            elif kind == PATCH_CONE:
                p[0:3] = _to_ecliptic(prm[0:3], o.frame)
                p[3] = prm[3]
            cols.append(np.concatenate([[o.jd], pos, vel, p, [float(kind)]]))
        return cols

    def ecliptic_column(self):
        """The column of a single-patch field."""
        (col,) = self.columns()
        return col


class _RectangleField(_Field):
    normals: np.ndarray

    def _set_rectangle(self, normals):
        self.normals = np.asarray(normals, dtype=np.float64).reshape(4, 3)
        self._patches = [(PATCH_RECTANGLE, self.normals.ravel())]

    @property
    def pointing(self):
        return np.array(_polygon_pointing([list(v) for v in self.normals]))

    @property
    def corners(self):
        """SphericalPolygon corners (patches.rs:182-194)."""
        return [np.array(_cross(self.normals[i], self.normals[(i + 1) % 4])) for i in range(4)]


class RectangleFOV(_RectangleField):
    """Rectangular field: pointing vector, rotation and widths in degrees, observer State
    (src/kete/rust/fovs/definitions.rs:400-418)."""

    def __init__(self, pointing, rotation, observer: State, lon_width, lat_width):
        self.observer = observer
        self.rotation = float(rotation)
        self.lon_width = float(lon_width)
        self.lat_width = float(lat_width)
        d2r = math.pi / 180.0  # f64::to_radians
        self._set_rectangle(rect_normals(np.asarray(pointing, dtype=np.float64).reshape(3),
                                         self.rotation * d2r, self.lon_width * d2r,
                                         self.lat_width * d2r))

    @staticmethod
    def from_corners(corners, observer: State):
        """RectangleFOV.from_corners (definitions.rs:429-433): 4 corners in order."""
        f = RectangleFOV.__new__(RectangleFOV)
        f.observer = observer
        f.rotation = float("nan")
        f._set_rectangle(rect_normals_from_corners(corners))
        return f


class ConeFOV(_Field):
    """Cone field: pointing vector, half-angle in degrees, observer State
    (definitions.rs:490-505 over GenericCone, generic.rs:140-190)."""

    def __init__(self, pointing, angle, observer: State):
        self.observer = observer
        self.pointing = np.array(_normalize([float(x) for x in pointing]))
        self.angle = float(angle) * math.pi / 180.0
        self._patches = [(PATCH_CONE, np.concatenate([self.pointing, [self.angle]]))]


class OmniDirectionalFOV(_Field):
    """Everything is visible (generic.rs:97-135)."""

    def __init__(self, observer: State):
        self.observer = observer
        self._patches = [(PATCH_OMNIDIRECTIONAL, np.zeros(0))]


class WiseCmos(_RectangleField):
    """A WISE frame from its corners (definitions.rs:325-339, wise.rs); ``from_pointing``
    builds it from a pointing and a rotation in degrees with the WISE field width."""

    def __init__(self, corners, observer: State, frame_num, scan_id):
        self.observer = observer
        self.frame_num = int(frame_num)
        self.scan_id = str(scan_id)
        self.rotation = float("nan")
        self._set_rectangle(rect_normals_from_corners(corners))

    @staticmethod
    def from_pointing(pointing, rotation, observer: State, frame_num, scan_id):
        f = WiseCmos.__new__(WiseCmos)
        f.observer = observer
        f.frame_num = int(frame_num)
        f.scan_id = str(scan_id)
        f.rotation = float(rotation)
        f._set_rectangle(rect_normals(np.asarray(pointing, float).reshape(3),
                                      math.radians(f.rotation), WISE_WIDTH, WISE_WIDTH))
        return f


class NeosCmos(_RectangleField):
    """One NEOS detector (definitions.rs:569-601, neos.rs:46-80): pointing, rotation in
    degrees, observer and the exposure's identifiers; NEOS_WIDTH x NEOS_HEIGHT."""

    def __init__(self, pointing, rotation, observer: State, side_id, stack_id, quad_id,
                 loop_id, subloop_id, exposure_id, cmos_id, band, _normals=None):
        self.observer = observer
        self.rotation = float(rotation)
        self.side_id, self.stack_id, self.quad_id = int(side_id), int(stack_id), int(quad_id)
        self.loop_id, self.subloop_id = int(loop_id), int(subloop_id)
        self.exposure_id, self.cmos_id, self.band = int(exposure_id), int(cmos_id), int(band)
        if _normals is None:
            _normals = rect_normals(np.asarray(pointing, float).reshape(3),
                                    math.radians(self.rotation), NEOS_WIDTH, NEOS_HEIGHT)
        self._set_rectangle(_normals)


class NeosVisit(_Field):
    """Four NEOS chips side by side with gaps (definitions.rs:708-744,
    NeosVisit::from_pointing neos.rs:215-340): widths and gap in degrees; the pointing sits
    in the middle of the central gap.  Pointing and observer are taken in the equatorial
    frame, as the reference does."""

    def __init__(self, x_width, y_width, gap_angle, pointing, rotation, observer: State,
                 side_id, stack_id, quad_id, loop_id, subloop_id, exposure_id, band):
        if Frames(observer.frame) != Frames.Equatorial:
            observer = State(observer.desig, observer.jd, ecliptic_to_equatorial(observer.pos),
                             ecliptic_to_equatorial(observer.vel), Frames.Equatorial,
                             observer.center_id)
        self.observer = observer
        self.rotation = float(rotation)
        xw, yw, gap = math.radians(x_width), math.radians(y_width), math.radians(gap_angle)
        p = [float(x) for x in np.asarray(pointing, float).reshape(3)]
        up0 = _rotate_around([0.0, 0.0, 1.0], p, -math.radians(self.rotation))
        left = _cross(p, up0)
        up = _cross(p, left)
        neg = lambda v: [-x for x in v]
        y_top = _rotate_around(up, left, yw / 2.0)
        y_bottom = _rotate_around(neg(up), left, -yw / 2.0)
        half_gap = gap / 2.0
        chip = (xw - 3.0 * gap) / 4.0
        bounds = [(-xw / 2.0, -xw / 2.0 + chip), (-chip - half_gap, -half_gap),
                  (half_gap, chip + half_gap), (xw / 2.0 - chip, xw / 2.0)]
        ids = (side_id, stack_id, quad_id, loop_id, subloop_id, exposure_id)
        self.chips = []
        for k, (a, b) in enumerate(bounds):
            na = _rotate_around(left, up, a)
            nb = neg(_rotate_around(left, up, b))
            self.chips.append(NeosCmos(p, rotation, observer, *ids, k, band,
                                       _normals=np.array([na, y_top, nb, y_bottom])))
        self.side_id, self.stack_id, self.quad_id = int(side_id), int(stack_id), int(quad_id)
        self.loop_id, self.subloop_id = int(loop_id), int(subloop_id)
        self.exposure_id, self.band = int(exposure_id), int(band)
        self._patches = [c._patches[0] for c in self.chips]

    def __len__(self):
        return 4

    def __getitem__(self, idx):
        return self.chips[idx]

    def get_fov(self, idx: int = 0):
        return self.chips[idx]


class ZtfCcdQuad(_RectangleField):
    """One ZTF CCD quadrant from its corners (definitions.rs:865-897, ztf.rs:36-61)."""

    def __init__(self, corners, observer: State, field, filefracday, ccdid, filtercode,
                 imgtypecode, qid, maglimit, fid):
        self.observer = observer
        self.field, self.filefracday, self.ccdid = int(field), int(filefracday), int(ccdid)
        self.filtercode, self.imgtypecode = str(filtercode), str(imgtypecode)
        self.qid, self.maglimit, self.fid = int(qid), float(maglimit), int(fid)
        self._set_rectangle(rect_normals_from_corners(corners))


class ZtfField(_Field):
    """A ZTF exposure: quadrants sharing field, filter, image type and epoch
    (ztf.rs:107-145)."""

    def __init__(self, ccd_quads):
        quads = list(ccd_quads)
        if not quads:
            raise ValueError("Ztf Field must contains ZtfCcdQuads")
        q0 = quads[0]
        for q in quads:
            if (q.field != q0.field or q.fid != q0.fid or q.filtercode != q0.filtercode
                    or q.imgtypecode != q0.imgtypecode or q.observer.jd != q0.observer.jd):
                raise ValueError("All ZtfCcdQuads must have matching values except CCD ID etc.")
        self.ccd_quads = quads
        self.observer = q0.observer
        self.field, self.fid = q0.field, q0.fid
        self.filtercode, self.imgtypecode = q0.filtercode, q0.imgtypecode
        self._patches = [q._patches[0] for q in quads]

    def __len__(self):
        return len(self.ccd_quads)

    def __getitem__(self, idx):
        return self.ccd_quads[idx]

    def get_fov(self, idx: int = 0):
        return self.ccd_quads[idx]


def _bind():
    L = _lib.lib()
    v = ctypes.c_void_p
    L.kete_b200_fov_check_visible.argtypes = [ctypes.c_int64, v, v, v, v, ctypes.c_int64, v,
                                              ctypes.c_double, ctypes.c_int, ctypes.c_int64, v, v,
                                              v, v, ctypes.c_int, v]
    return L


def set_fov_form(form: int = 0):
    """Form of the field checks (kete_b200_set_fov_form): 0 = linear screen of every (object,
    field) pair, then the two-body solve on the pairs that pass (default); 1 = one fused
    pass.  Same results."""
    L = _lib.lib()
    L.kete_b200_set_fov_form.argtypes = [ctypes.c_int]
    _lib.check(L.kete_b200_set_fov_form(int(form)))


def fov_check_visible_arrays(pos, vel, jd, valid, fov_table, dt_limit=3.0,
                             include_asteroids=False, capacity=None):
    """Visibility of n objects (SoA (3, n) at epochs jd (n,), valid (n,) uint8 or None) in
    the field patches of fov_table (FOV_STRIDE, F).  Host numpy arrays or torch CUDA tensors.

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
                           nongrav=None, on_chunk=None, stage_times=None):
    """The fov_state_check schedule (src/kete/rust/fovs/checks.rs:24-110) on device arrays.

    pos/vel (3, n) heliocentric ecliptic torch CUDA tensors at the common epoch ``jd``;
    fov_table (FOV_STRIDE, F) patch columns sorted by observer epoch (row 0).  Chunks of fields shorter
    than 2*dt_limit are checked against the population re-propagated (N-body) to the
    chunk's mean epoch, re-seeded from a big-step copy every 25-50 dt_limit as the
    reference does; objects whose propagation fails are dropped from then on.  Returns
    (fov_index, obj_index, state7) numpy arrays over all fields, sorted by field then
    object.  ``on_chunk(k0, k1)``, when given, is called after each chunk.  ``stage_times``,
    when given (a dict), accumulates the seconds spent in the N-body re-propagations
    ("propagate") and in the field checks ("check"), each measured with the device
    synchronized on both sides."""
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
            t_start = _stage_start()
            jd0 = torch.full((n,), self.t, dtype=torch.float64, device=dev)
            jd1 = torch.full((n,), target, dtype=torch.float64, device=dev)
            P, V, st = propagate_n_body_arrays(self.P, self.V, jd0, jd1, Frames.Ecliptic, 10,
                                               include_asteroids, nongrav)
            self.P, self.V, self.t = P, V, target
            self.ok = self.ok & (st == 0)
            _stage_end("propagate", t_start)

    def _stage_start():
        if stage_times is None:
            return 0.0
        torch.cuda.synchronize(dev)
        return time.perf_counter()

    def _stage_end(name, t_start):
        if stage_times is not None:
            torch.cuda.synchronize(dev)
            stage_times[name] = stage_times.get(name, 0.0) + time.perf_counter() - t_start

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
        t_start = _stage_start()
        epochs = torch.full((n,), cur.t, dtype=torch.float64, device=dev)
        ff, oo, ss = fov_check_visible_arrays(cur.P, cur.V, epochs, cur.ok.to(torch.uint8),
                                              table[:, k0:k1].contiguous(), dt_limit,
                                              include_asteroids)
        _stage_end("check", t_start)
        out_f.append(ff + k0)
        out_o.append(oo)
        out_s.append(ss)
        if on_chunk is not None:
            on_chunk(k0, k1)
    if not out_f:
        return np.empty(0, np.int32), np.empty(0, np.int32), np.empty((7, 0))
    return np.concatenate(out_f), np.concatenate(out_o), np.concatenate(out_s, axis=1)


def _flatten(fovs):
    """Time-sorted fields, their patch columns as one table, and each column's (field,
    patch) owner."""
    fovs = sorted(list(fovs), key=lambda f: f.jd)
    cols, owner = [], []
    for fi, f in enumerate(fovs):
        for pi, col in enumerate(f.columns()):
            cols.append(col)
            owner.append((fi, pi))
    table = np.stack(cols, axis=1) if cols else np.zeros((FOV_STRIDE, 0))
    return fovs, np.ascontiguousarray(table), owner


def _first_patch(keys, owner):
    """closest_inside (patches.rs:21-35): of the columns a target is inside, its field keeps
    the first patch.  keys: (column, target index, row) triples; returns
    {(field, target): (patch, row)}."""
    best = {}
    for col, tgt, row in keys:
        fi, pi = owner[col]
        k = (fi, tgt)
        if k not in best or pi < best[k][0]:
            best[k] = (pi, row)
    return best


def fov_state_check(obj_state, fovs, dt_limit=3.0, include_asteroids=False):
    """kete.fov_state_check: objects (SimultaneousStates, or a list of States sharing one
    epoch, heliocentric ecliptic) visible in each field; returns a list of
    SimultaneousStates, one per field patch with at least one visible object, fields in
    time order."""
    import torch

    states = list(obj_state.states if isinstance(obj_state, SimultaneousStates) else obj_state)
    if not states:
        return []
    fovs, table, owner = _flatten(fovs)
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
    ff, oo, ss = fov_state_check_arrays(T(pos), T(vel), states[0].jd, table, dt_limit,
                                        include_asteroids)
    best = _first_patch(((int(ff[j]), int(oo[j]), j) for j in range(len(ff))), owner)
    return _group_states(fovs, best, lambda i: desig[i], ss)


def _group_states(fovs, best, name_of, ss):
    per = {}
    for (fi, tgt), (pi, row) in best.items():
        per.setdefault((fi, pi), []).append((tgt, row))
    results = []
    for fi, f in enumerate(fovs):
        for pi in range(f.n_patches()):
            hits = sorted(per.get((fi, pi), []))
            if not hits:
                continue
            vis = [State(name_of(t), ss[0, r], ss[1:4, r], ss[4:7, r], Frames.Ecliptic, 10)
                   for t, r in hits]
            results.append(SimultaneousStates(vis, f.get_fov(pi)))
    return results


def fov_spk_check(obj_ids, fovs):
    """kete.fov_spk_check (src/kete/rust/fovs/checks.rs:111-135, FovLike::check_spks
    fov_like.rs:196-226): objects loaded from SPK files (NAIF ids) visible in each field,
    with the light delay applied (two-body back-propagation); states heliocentric
    ecliptic.  The SPK states are read on the GPU at every field epoch."""
    from . import spice

    fovs, table, owner = _flatten(fovs)
    ids = [int(i) for i in obj_ids]
    if not ids or not fovs:
        return []
    field_cols = {}
    for col, (fi, _) in enumerate(owner):
        field_cols.setdefault(fi, []).append(col)
    jds = np.array([f.jd for f in fovs])
    st6 = np.empty((len(ids), 6, len(fovs)))
    ok = np.empty((len(ids), len(fovs)), dtype=bool)
    for k, oid in enumerate(ids):
        out6, st = spice.get_states_arrays(oid, jds, 10, Frames.Ecliptic)
        st6[k], ok[k] = out6, st == 0
    rows, keys = [], []
    for fi in range(len(fovs)):
        sel = np.nonzero(ok[:, fi])[0]
        if sel.size == 0:
            continue
        cols = field_cols[fi]
        pos = np.ascontiguousarray(st6[sel, 0:3, fi].T)
        vel = np.ascontiguousarray(st6[sel, 3:6, fi].T)
        # the states are at the field's epoch: the reference goes straight to the two-body
        # light-time check, which an unbounded dt_limit reproduces (no linear pre-filter)
        ff, oo, ss = fov_check_visible_arrays(pos, vel, np.full(sel.size, jds[fi]), None,
                                              np.ascontiguousarray(table[:, cols]), 1e300)
        for j in range(len(ff)):
            keys.append((cols[int(ff[j])], int(sel[oo[j]]), len(rows)))
            rows.append(ss[:, j])
    if not rows:
        return []
    ss = np.stack(rows, axis=1)
    best = _first_patch(keys, owner)
    return _group_states(fovs, best, lambda i: ids[i], ss)


def fov_static_check(pos, fovs):
    """kete.fov_static_check (src/kete/rust/fovs/checks.rs:137-188): fixed sky directions
    (observer to target, ecliptic; each a 3-vector) contained in each field.  Returns a list
    of (indices of the contained directions, field patch), fields in time order."""
    vec = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).reshape(-1, 3).T)
    fovs, table, owner = _flatten(fovs)
    n_vec = vec.shape[1]
    if n_vec == 0 or not fovs:
        return []
    _lib.init()
    L = _lib.lib()
    v = ctypes.c_void_p
    L.kete_b200_fov_contains.argtypes = [ctypes.c_int64, v, ctypes.c_int64, v, ctypes.c_int64,
                                         v, v, v, ctypes.c_int, v]
    cap = max(1024, n_vec)
    for _ in range(3):
        out_f = np.empty(cap, dtype=np.int32)
        out_i = np.empty(cap, dtype=np.int32)
        found = ctypes.c_int64(0)
        a = _lib.Args()
        _lib.check(L.kete_b200_fov_contains(n_vec, a.ptr(vec), table.shape[1], a.ptr(table), cap,
                                            a.ptr(out_f, np.int32), a.ptr(out_i, np.int32),
                                            ctypes.byref(found), a.on_device, a.stream))
        m = found.value
        if m <= cap:
            break
        cap = m + 1024
    best = _first_patch(((int(out_f[j]), int(out_i[j]), j) for j in range(m)), owner)
    per = {}
    for (fi, idx), (pi, _) in best.items():
        per.setdefault((fi, pi), []).append(idx)
    out = []
    for fi, f in enumerate(fovs):
        for pi in range(f.n_patches()):
            if (fi, pi) in per:
                out.append((sorted(per[(fi, pi)]), f.get_fov(pi)))
    return out
