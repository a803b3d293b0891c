"""GPU SPK types 3 and 21 against the oracle (kete_b200_spk_get_states).

The type-21 slice of a JPL asteroid file (tests/golden/spk_type21_subset.bsp) and a synthetic
type-3 file are loaded beside the synthetic planetary ephemeris on the GPU and in the
oracle; states agree to 5e-14 of their magnitude (the modified difference arrays and the
Chebyshev sums run the same operations; fused multiply-adds move the last bits), relative
to the Sun and to the solar-system barycentre (chained through the Sun's type-2 segment).
"""
import os

import numpy as np
import pytest

from kete_b200 import synthetic

pytestmark = pytest.mark.gpu
SUBSET = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "spk_type21_subset.bsp")


@pytest.fixture()
def mixed_kernels(gpu, oracle, spk_path, tmp_path):
    t3 = synthetic.write_type3_spk(str(tmp_path / "t3.bsp"))
    files = [spk_path, SUBSET, t3]
    gpu.spice.kernel_reload(files)
    oracle.spk_reset()
    for p in files:
        with open(p, "rb") as f:
            oracle.spk_load_bytes(f.read())
    yield gpu, oracle
    gpu.spice.kernel_reload([spk_path])  # the other tests' ephemeris
    oracle.spk_reset()
    with open(spk_path, "rb") as f:
        oracle.spk_load_bytes(f.read())


def _compare(gpu, oracle, body, jds, center, frame):
    out, st = gpu.spice.get_states_arrays(body, jds, center, frame)
    assert (st == 0).all()
    for k, jd in enumerate(jds):
        rc, ref = oracle.spk_get_state(body, jd, center, frame)
        assert rc == 0
        scale_p = np.abs(ref[:3]).max()
        scale_v = np.abs(ref[3:]).max()
        assert np.abs(out[:3, k] - ref[:3]).max() <= 5e-14 * scale_p, (body, jd)
        assert np.abs(out[3:, k] - ref[3:]).max() <= 5e-14 * scale_v, (body, jd)


@pytest.mark.parametrize("center,frame", [(10, 1), (0, 1), (10, 2)])
def test_type21_states(mixed_kernels, center, frame):
    gpu, oracle = mixed_kernels
    (_, _, _, _, s0, s1, _), = synthetic.read_daf_segments(SUBSET)
    jds = np.linspace(s0 + 1.0, s1 - 1.0, 301) / 86400.0 + 2451545.0
    _compare(gpu, oracle, 20000042, jds, center, frame)


@pytest.mark.parametrize("center,frame", [(10, 1), (0, 2)])
def test_type3_states(mixed_kernels, center, frame):
    gpu, oracle = mixed_kernels
    jds = np.linspace(2459001.0, 2460999.0, 257)
    for body in synthetic.ASTEROIDS[:2]:
        _compare(gpu, oracle, body, jds, center, frame)


def test_type21_outside_coverage_is_daf_limits(mixed_kernels):
    gpu, _ = mixed_kernels
    (_, _, _, _, s0, s1, _), = synthetic.read_daf_segments(SUBSET)
    _, st = gpu.spice.get_states_arrays(20000042, [s1 / 86400.0 + 2451545.0 + 2.0], 10, 1)
    assert st.tolist() == [3]


def test_invalid_mda_record_is_rejected(gpu, tmp_path):
    """A type-21 record whose interpolation order exceeds its arrays is refused at load."""
    (tgt, ctr, frm, typ, s0, s1, data), = synthetic.read_daf_segments(SUBSET)
    bad = data.copy()
    md = int(data[-2])
    bad[4 * md + 7] = md + 5.0  # KQMAX1 beyond MAXDIM + 1 in record 0
    path = str(tmp_path / "bad21.bsp")
    synthetic.write_daf_spk(path, [(tgt, ctr, frm, typ, s0, s1, bad)])
    with pytest.raises(gpu.KeteB200Error, match="invalid contents"):
        gpu.spice.load_spk(path)
