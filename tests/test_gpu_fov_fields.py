"""GPU visibility for every field type against the oracle.

Cones, omnidirectional fields, NEOS visits (4 chips) and ZTF fields (several quadrants) are
checked through kete_b200_fov_check_visible / _fov_contains, and through
fov_state_check / fov_spk_check / fov_static_check, against the oracle's patch containment
(ko_patch_contains) and check_visible.  Membership must be identical except for targets
within 1e-10 rad of a patch edge; a target in several patches of one field counts in the
first (closest_inside, patches.rs:21-35).
"""
import math

import numpy as np
import pytest

from kete_b200 import fov as F
from kete_b200 import synthetic
from kete_b200.state import Frames, State

pytestmark = pytest.mark.gpu
EPOCH = synthetic.EPOCH
EDGE_RAD = 1e-10


def _observer(oracle_spk, jd, frame=Frames.Ecliptic):
    rc, s = oracle_spk.spk_get_state(399, jd, 10, int(frame))
    assert rc == 0
    return State("observer", jd, s[:3], s[3:], frame, 10)


def _population(n, seed):
    pm, vm = synthetic.main_belt(n - n // 5, seed=seed)
    pn, vn = synthetic.neo(n // 5, seed=seed + 1)
    return np.concatenate([pm, pn], axis=1), np.concatenate([vm, vn], axis=1)


def _edge_distance(col, v):
    """Angular distance of direction v from the nearest edge of a patch column."""
    v = np.asarray(v) / np.linalg.norm(v)
    kind = int(col[19])
    if kind == F.PATCH_CONE:
        return abs(math.acos(min(1.0, max(-1.0, float(np.dot(col[7:10], v))))) - col[10])
    if kind == F.PATCH_OMNIDIRECTIONAL:
        return np.inf
    n = col[7:19].reshape(4, 3)
    return float(np.min(np.abs(n @ v) / np.linalg.norm(n, axis=1)))


def _fields(oracle_spk, pos, seed):
    """One field of each type, aimed at objects so that every type sees some."""
    rng = np.random.default_rng(seed)
    out = []
    jds = EPOCH + np.sort(rng.uniform(0.0, 2.0, 6))
    for k, jd in enumerate(jds):
        obs = _observer(oracle_spk, jd)
        tgt = pos[:, rng.integers(pos.shape[1])] - obs.pos
        tgt = tgt / np.linalg.norm(tgt)
        if k == 0:
            out.append(F.ConeFOV(tgt, 6.0, obs))
        elif k == 1:
            out.append(F.OmniDirectionalFOV(obs))
        elif k == 2:
            eq = _observer(oracle_spk, jd, Frames.Equatorial)
            out.append(F.NeosVisit(12.0, 4.0, 0.6, F.ecliptic_to_equatorial(tgt), 10.0, eq,
                                   1, 2, 3, 4, 5, 6, 1))
        elif k == 3:
            quads = []
            for dx in (-1, 1):
                for dy in (-1, 1):
                    c = F.RectangleFOV(tgt, 0.0, obs, 3.0, 3.0)
                    # quadrant corners: shift the pointing by +-1.5 deg in two directions
                    ax1 = np.array(F._cross(list(tgt), [0.0, 0.0, 1.0]))
                    ax1 /= np.linalg.norm(ax1)
                    ax2 = np.cross(tgt, ax1)
                    centre = tgt + math.radians(1.5) * (dx * ax1 + dy * ax2)
                    q = F.RectangleFOV(centre, 0.0, obs, 3.2, 3.2)  # overlapping quadrants
                    quads.append(F.ZtfCcdQuad(q.corners, obs, 700, 1, len(quads) + 1, "zg",
                                              "sci", 1, 20.0, 1))
            out.append(F.ZtfField(quads))
        elif k == 4:
            out.append(F.WiseCmos.from_pointing(tgt, 30.0, obs, 17, "01234a"))
        else:
            out.append(F.NeosCmos(tgt, 5.0, obs, 1, 1, 1, 1, 1, 1, 0, 1))
    return out


def _oracle_field(oracle_spk, f, pos, vel, jd, dt_limit):
    """{object: (patch, state7)} of one field by the oracle (first containing patch)."""
    found = {}
    for pi, col in enumerate(f.columns()):
        flags, out7 = oracle_spk.fov_check_visible(col[:7], col[7:19], pos, vel, jd, dt_limit,
                                                   kind=int(col[19]))
        for i in np.nonzero(flags)[0]:
            if int(i) not in found:
                found[int(i)] = (pi, out7[:, i], col)
    return found


def test_field_types_in_fov_state_check(gpu, oracle_spk):
    n = 3000
    pos, vel = _population(n, 41)
    fovs = _fields(oracle_spk, pos, 42)
    states = [gpu.State(f"o{i}", EPOCH, pos[:, i], vel[:, i]) for i in range(n)]
    res = gpu.fov_state_check(states, fovs, dt_limit=3.0)
    got = {}
    for sim in res:
        for s in sim.states:
            got[(id(sim.fov), int(s.desig[1:]))] = s
    # all fields lie within 2 days of the epoch: one chunk, no re-propagation
    n_types = set()
    for f in sorted(fovs, key=lambda f: f.jd):
        ref = _oracle_field(oracle_spk, f, pos, vel, np.full(n, EPOCH), 3.0)
        for i, (pi, st, col) in ref.items():
            key = (id(f.get_fov(pi)), i)
            if key not in got:
                assert _edge_distance(col, st[1:4] - col[1:4]) < EDGE_RAD, (type(f), i)
                continue
            assert np.abs(got[key].pos - st[1:4]).max() < 1e-12
            n_types.add(type(f).__name__)
        for (fid, i), s in got.items():
            if any(fid == id(f.get_fov(pi)) for pi in range(f.n_patches())):
                assert i in ref or min(_edge_distance(c, s.pos - c[1:4]) for c in f.columns()) < EDGE_RAD
    assert len(n_types) >= 5, n_types  # the aimed fields see objects


def test_fov_static_check(gpu, oracle_spk):
    pos, _ = _population(200, 51)
    fovs = _fields(oracle_spk, pos, 52)
    rng = np.random.default_rng(53)
    vecs = rng.normal(size=(20000, 3))
    for f in fovs[:3]:  # plenty of directions near the aimed patches
        col = f.columns()[0]
        centre = col[7:10] if int(col[19]) == F.PATCH_CONE else np.zeros(3)
        if np.any(centre):
            vecs[:2000] = centre + rng.normal(scale=0.05, size=(2000, 3))
    res = gpu.fov_static_check(vecs, fovs)
    got = {(id(f), i) for idx, f in res for i in idx}
    total = 0
    for f in sorted(fovs, key=lambda f: f.jd):
        for i, v in enumerate(vecs):
            for pi, col in enumerate(f.columns()):
                inside, _ = oracle_spk.patch_contains(col[7:19], int(col[19]), v)
                if inside:
                    key = (id(f.get_fov(pi)), i)
                    assert key in got or _edge_distance(col, v) < EDGE_RAD
                    total += 1
                    break
    assert total > 100
    assert len(got) <= total


def test_fov_spk_check(gpu, oracle_spk):
    """The planets seen from the Earth's position: SPK states at each field epoch, light
    delay by two-body back-propagation (fov_like.rs:196-226)."""
    ids = [1, 2, 4, 5, 6, 7, 8, 301]
    fovs = []
    for k, jd in enumerate(EPOCH + np.array([0.3, 10.0, 40.5])):
        obs = _observer(oracle_spk, jd)
        for body in ids[k::3]:
            rc, s = oracle_spk.spk_get_state(body, jd, 10, 2)
            fovs.append(F.ConeFOV(s[:3] - obs.pos, 1.0, obs))
        fovs.append(F.OmniDirectionalFOV(obs))
    res = gpu.fov_spk_check(ids, fovs)
    got = {(id(sim.fov), s.desig): s for sim in res for s in sim.states}
    for f in sorted(fovs, key=lambda f: f.jd):
        col = f.columns()[0]
        for body in ids:
            rc, s = oracle_spk.spk_get_state(body, f.jd, 10, 2)
            flags, out7 = oracle_spk.fov_check_visible(col[:7], col[7:19], s[:3, None],
                                                       s[3:, None], f.jd, 1e300,
                                                       kind=int(col[19]))
            if flags[0]:
                assert (id(f), body) in got
                assert np.abs(got[(id(f), body)].pos - out7[1:4, 0]).max() < 1e-12
            else:
                assert (id(f), body) not in got or _edge_distance(col, out7[1:4, 0] - col[1:4]) < EDGE_RAD
    assert sum(1 for k in got if k[1] in ids) >= 3 + 3 * len(ids)
