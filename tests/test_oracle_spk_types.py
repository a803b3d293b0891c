"""The oracle's SPK types 3 (Chebyshev position and velocity) and 1/21 (modified difference
arrays), pinned to the data themselves.

Type 21 (tests/golden/spk_type21_subset.bsp, a slice of the JPL type-21 asteroid file in the
reference's documentation): every record's reference epoch is its final epoch, where the
interpolation returns the record's stored reference state; just after a final epoch the next
record takes over and must continue the previous record's state.  Both agree to 1e-11 AU,
the rounding of the epoch through Julian days (4e-5 s at 20 km/s).  Type 3: a synthetic file
fitted to known orbits reproduces them to the fit's accuracy (1e-11 AU, 1e-13 AU/day).
"""
import os

import numpy as np
import pytest

from kete_b200 import synthetic

AU_KM = 149597870.7
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SUBSET = os.path.join(GOLDEN, "spk_type21_subset.bsp")
# the full JPL file the fixture was cut from, when a reference checkout is named
FULL = os.environ.get("KETE_REFERENCE_BSP", "")


def _load(oracle, *paths):
    oracle.spk_reset()
    for p in paths:
        with open(p, "rb") as f:
            oracle.spk_load_bytes(f.read())


def _records(path):
    (_, _, _, _, s0, s1, data), = synthetic.read_daf_segments(path)
    n, md = int(data[-1]), int(data[-2])
    rl = 4 * md + 11
    return data, n, md, rl, data[n * rl:n * rl + n], s0, s1


def test_type21_reference_epochs_and_continuity(oracle):
    _load(oracle, SUBSET)
    data, n, md, rl, ep, s0, s1 = _records(SUBSET)
    for r in range(n):
        ref = data[r * rl + 1 + md:r * rl + 7 + md]
        rc, s = oracle.spk_get_state(20000042, ep[r] / 86400.0 + 2451545.0, 10, 1)
        assert rc == 0
        assert np.abs(s[:3] - ref[0::2] / AU_KM).max() < 1e-11
        assert np.abs(s[3:] - ref[1::2] / AU_KM * 86400.0).max() < 1e-12
        if r + 1 < n:  # one second later the next record continues the state
            rc, s2 = oracle.spk_get_state(20000042, (ep[r] + 1.0) / 86400.0 + 2451545.0, 10, 1)
            assert rc == 0
            assert np.abs(s2[:3] - (ref[0::2] + ref[1::2]) / AU_KM).max() < 1e-11


def test_type21_outside_coverage(oracle):
    _load(oracle, SUBSET)
    _, _, _, _, _, s0, s1 = _records(SUBSET)
    rc, _ = oracle.spk_get_state(20000042, s1 / 86400.0 + 2451545.0 + 1.0, 10, 1)
    assert rc == 3  # DAFLimits


@pytest.mark.skipif(not FULL or not os.path.exists(FULL),
                    reason="KETE_REFERENCE_BSP does not name the reference's type-21 file")
def test_type21_subset_matches_full_file(oracle):
    _, _, _, _, _, s0, s1 = _records(SUBSET)
    jds = np.linspace(s0 + 10.0, s1 - 10.0, 97) / 86400.0 + 2451545.0
    _load(oracle, SUBSET)
    a = [oracle.spk_get_state(20000042, jd, 10, 1)[1] for jd in jds]
    _load(oracle, FULL)
    b = [oracle.spk_get_state(20000042, jd, 10, 1)[1] for jd in jds]
    assert np.array_equal(np.array(a), np.array(b))


def test_type3_reproduces_fitted_orbits(oracle, tmp_path):
    path = synthetic.write_type3_spk(str(tmp_path / "t3.bsp"))
    _load(oracle, path)
    jds = np.linspace(2459010.3, 2460990.7, 211)
    truth = synthetic.synthetic_bodies(jds)
    for body in synthetic.ASTEROIDS[:2]:
        p, v, c = truth[body]
        for k, jd in enumerate(jds):
            rc, s = oracle.spk_get_state(body, jd, 10, 1)
            assert rc == 0
            assert np.abs(s[:3] - p[:, k] / AU_KM).max() < 1e-11
            assert np.abs(s[3:] - v[:, k] / AU_KM * 86400.0).max() < 1e-13
