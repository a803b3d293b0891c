"""Write tests/golden/spk_type21_subset.bsp: a slice of a real type-21 (extended modified
difference array) SPK segment, for the tests of SPK types 1/21.

The source is the asteroid ephemeris that ships with the reference's documentation
(docs/data/20000042.bsp: JPL Horizons output for (42) Isis, centre the Sun, J2000
equatorial, MAXDIM 20).  The slice keeps RECORDS consecutive records of the segment that
covers JD 2460000.5 and their final epochs, and writes them as one type-21 segment (no
epoch directory: fewer than 100 records) whose coverage starts at the first kept record's
start (the previous record's final epoch) and ends at the last kept record's final epoch.

Run from the repository root:  python tests/golden/make_spk_fixtures.py [path-to-20000042.bsp]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from kete_b200 import synthetic  # noqa: E402

RECORDS = 48
TARGET_JD = 2460000.5


def main(src):
    segs = [s for s in synthetic.read_daf_segments(src) if s[3] == 21]
    target_s = (TARGET_JD - 2451545.0) * 86400.0
    tgt, ctr, frm, typ, s0, s1, data = next(s for s in segs if s[4] <= target_s <= s[5])
    n_rec = int(data[-1])
    md = int(data[-2])
    rl = 4 * md + 11
    epochs = data[n_rec * rl:n_rec * rl + n_rec]
    first = max(1, int(np.searchsorted(epochs, target_s)) - RECORDS // 2)
    last = first + RECORDS
    recs = data[first * rl:last * rl]
    ep = epochs[first:last]
    start_s = epochs[first - 1]
    out = np.concatenate([recs, ep, [float(md), float(RECORDS)]])
    path = os.path.join(HERE, "spk_type21_subset.bsp")
    synthetic.write_daf_spk(path, [(tgt, ctr, frm, 21, start_s, ep[-1], out)],
                            internal_name="slice of a JPL type-21 asteroid SPK")
    print(path, "records", RECORDS, "MAXDIM", md, "JD", start_s / 86400 + 2451545.0,
          ep[-1] / 86400 + 2451545.0)


if __name__ == "__main__":
    path = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KETE_REFERENCE_BSP")
    if not path:
        sys.exit("usage: make_spk_fixtures.py <path to the reference's docs/data/20000042.bsp> "
                 "(or set KETE_REFERENCE_BSP)")
    main(path)
