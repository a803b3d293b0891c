"""Field-of-view constructors (host logic) and the oracle's patch containment.

Rectangles from corners must contain exactly what the pointing form contains, whichever way
round the corners are listed (OnSkyRectangle::from_corners flips a far-side ordering);
NeosVisit's four chips tile the visit with three gaps, the pointing in the central gap
(neos.rs:215-340); cones follow SphericalCone::contains (patches.rs:300-337), including the
outside distance; multi-patch fields report their first containing patch.
"""
import math

import numpy as np
import pytest

from kete_b200 import fov as F
from kete_b200.state import Frames, State


def _obs(jd=2460000.5, frame=Frames.Ecliptic):
    return State("observer", jd, [0.9, -0.4, 0.0], [0.005, 0.015, 0.0], frame, 10)


def _inside(normals, v):
    return all(math.copysign(1.0, float(np.dot(v, n))) > 0 for n in np.asarray(normals).reshape(4, 3))


def test_rectangle_from_corners_matches_pointing_form(oracle):
    rng = np.random.default_rng(3)
    for _ in range(20):
        p = rng.normal(size=3)
        r = F.RectangleFOV(p, rng.uniform(0, 180), _obs(), rng.uniform(0.5, 5), rng.uniform(0.5, 5))
        for corners in (r.corners, r.corners[::-1]):
            c = F.RectangleFOV.from_corners(corners, _obs())
            for _ in range(200):
                v = p / np.linalg.norm(p) + rng.normal(scale=0.05, size=3)
                assert _inside(r.normals, v) == _inside(c.normals, v)
                assert oracle.patch_contains(c.normals, 0, v)[0] == _inside(c.normals, v)
        assert np.allclose(c.pointing, p / np.linalg.norm(p), atol=1e-9)


def test_reference_rectangle_patch_cases(oracle):
    """patches.rs:366-384 through the oracle's containment."""
    fov = F.rect_normals([1.0, 0.0, 0.0], 0.0, 0.1, 0.1)
    rot = F.rect_normals([1.0, 0.0, 0.0], math.radians(45.0), 0.1, 0.1)
    s = math.sin(0.05)
    assert oracle.patch_contains(fov, 0, [1.0, 0.01, 0.01])[0]
    assert oracle.patch_contains(fov, 0, [1.0, s * 0.99, s * 0.99])[0]
    assert not oracle.patch_contains(fov, 0, [1.0, 0.1, 0.0])[0]
    assert not oracle.patch_contains(fov, 0, [1.0, s * 1.01, s * 1.01])[0]
    assert oracle.patch_contains(rot, 0, [1.0, 0.01, 0.01])[0]
    assert not oracle.patch_contains(rot, 0, [1.0, s * 0.99, s * 0.99])[0]


def test_neos_visit_chips_and_gaps():
    x_w, y_w, gap = 7.1, 1.68, 0.3
    p = np.array([0.2, 0.9, 0.3])
    p /= np.linalg.norm(p)
    v = F.NeosVisit(x_w, y_w, gap, p, 20.0, _obs(frame=Frames.Equatorial), 1, 2, 3, 4, 5, 6, 1)
    assert len(v) == 4 and [c.cmos_id for c in v.chips] == [0, 1, 2, 3]
    chip = math.radians((x_w - 3 * gap) / 4)
    # walk along the visit's long axis through the pointing
    up0 = F._rotate_around([0.0, 0.0, 1.0], list(p), -math.radians(20.0))
    left = np.array(F._cross(list(p), up0))
    left /= np.linalg.norm(left)
    centres = [-1.5 * chip - math.radians(gap), -0.5 * chip - math.radians(gap) / 2,
               0.5 * chip + math.radians(gap) / 2, 1.5 * chip + math.radians(gap)]
    for k, a in enumerate(centres):
        d = math.cos(a) * p + math.sin(a) * left
        hits = [j for j, c in enumerate(v.chips) if _inside(c.normals, d)]
        assert hits == [k], (k, hits)
    for g in (0.0, chip + math.radians(gap) / 2):  # centres of the gaps
        for sgn in (1, -1):
            d = math.cos(sgn * g) * p + math.sin(sgn * g) * left
            assert not any(_inside(c.normals, d) for c in v.chips)
    assert Frames(v.observer.frame) == Frames.Equatorial


def test_cone_contains(oracle):
    prm = [1.0, 0.0, 0.0, math.radians(5.0)]
    assert oracle.patch_contains(prm, 1, [1.0, math.tan(math.radians(4.9)), 0.0])[0]
    inside, d = oracle.patch_contains(prm, 1, [2.0, 2.0 * math.tan(math.radians(6.0)), 0.0])
    r = 2.0 / math.cos(math.radians(6.0))
    assert not inside and abs(d - math.sin(math.radians(1.0)) * r) < 1e-12
    inside, d = oracle.patch_contains(prm, 1, [-1.0, 0.0, 0.0])  # behind: move the full distance
    assert not inside and abs(d - 1.0) < 1e-15
    assert oracle.patch_contains([], 2, [0.3, -2.0, 1.0]) == (True, 0.0)


def test_field_columns_and_validation():
    c = F.ConeFOV([0, 3, 4], 2.0, _obs())
    col = c.ecliptic_column()
    assert col.size == F.FOV_STRIDE and col[-1] == F.PATCH_CONE
    assert np.allclose(col[7:10], [0, 0.6, 0.8]) and abs(col[10] - math.radians(2.0)) < 1e-15
    o = F.OmniDirectionalFOV(_obs())
    assert o.ecliptic_column()[-1] == F.PATCH_OMNIDIRECTIONAL
    eq = F.RectangleFOV([1, 0, 0], 0.0, _obs(frame=Frames.Equatorial), 1.0, 1.0)
    col = eq.ecliptic_column()  # patch normals follow the observer into the ecliptic frame
    assert np.allclose(col[7:10], F.equatorial_to_ecliptic(eq.normals[0]))
    corners = [[1, -0.01, -0.01], [1, 0.01, -0.01], [1, 0.01, 0.01], [1, -0.01, 0.01]]
    q1 = F.ZtfCcdQuad(corners, _obs(), 500, 20230101, 1, "zr", "sci", 1, 20.5, 2)
    q2 = F.ZtfCcdQuad(corners, _obs(2460001.5), 500, 20230101, 2, "zr", "sci", 1, 20.5, 2)
    with pytest.raises(ValueError):
        F.ZtfField([q1, q2])
    z = F.ZtfField([q1, q1])
    assert z.n_patches() == 2 and z.get_fov(1) is q1
