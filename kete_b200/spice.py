"""SPK loading and state queries, mirroring kete.spice (src/kete/spice.py) for the parts the
propagation path needs: ``kernel_reload``, ``get_state`` and ``loaded_objects``.

The ephemeris is parsed by libketeb200.so and kept resident on the GPU; states are
evaluated there (batched SpkCollection::try_get_state, src/kete_core/src/spice/spk.rs:87-96).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from .state import Frames, State

NAMES = {"sun": 10, "mercury": 1, "venus": 2, "earth": 399, "moon": 301, "mars": 4,
         "jupiter": 5, "saturn": 6, "uranus": 7, "neptune": 8, "ssb": 0,
         "solar system barycenter": 0, "earth-moon barycenter": 3, "emb": 3}


def _naif(x) -> int:
    if isinstance(x, (int, np.integer)):
        return int(x)
    key = str(x).strip().lower()
    if key in NAMES:
        return NAMES[key]
    return int(key)


def kernel_reload(filenames=None, include_cache=False):
    """Reset the loaded kernels and load the given SPK files (kete.spice.kernel_reload).
    There is no network or kernel cache here: files must be given explicitly."""
    _lib.init()
    _lib.check(_lib.lib().kete_b200_spk_reset())
    for fn in filenames or []:
        load_spk(fn)


def load_spk(filename):
    """Add one SPK file to the loaded ephemeris."""
    _lib.init()
    _lib.check(_lib.lib().kete_b200_spk_load_file(os.fsencode(filename)))


def loaded_ids():
    n = _lib.lib().kete_b200_spk_loaded_ids(None, 0)
    buf = (C.c_int64 * max(n, 1))()
    _lib.lib().kete_b200_spk_loaded_ids(C.cast(buf, C.c_void_p), n)
    return [int(buf[i]) for i in range(n)]


def loaded_objects():
    inv = {v: k for k, v in NAMES.items() if k not in ("ssb", "emb")}
    return [(inv.get(i, str(i)), i) for i in loaded_ids()]


def get_states_arrays(target, jd, center=10, frame=Frames.Ecliptic):
    """State of ``target`` at each epoch of ``jd`` (array) relative to ``center``.
    Returns (out6 (6, n), status (n,))."""
    _lib.init()
    jd = np.ascontiguousarray(np.atleast_1d(np.asarray(jd, dtype=np.float64)))
    n = jd.size
    out6 = np.empty((6, n))
    st = np.empty(n, dtype=np.int32)
    a = _lib.Args()
    args = [a.ptr(jd), int(center), int(frame), a.ptr(out6), a.ptr(st, np.int32)]
    _lib.check(_lib.lib().kete_b200_spk_get_states(n, _naif(target), args[0], args[1], args[2],
                                                   args[3], args[4], a.on_device, a.stream))
    return out6, st


def get_state(target, jd, center="Sun", frame=Frames.Ecliptic) -> State:
    """kete.spice.get_state: state of ``target`` at ``jd`` relative to ``center``."""
    jd = float(getattr(jd, "jd", jd))
    out6, st = get_states_arrays(target, [jd], _naif(center), frame)
    if st[0] != 0:
        raise ValueError(f"SPK query for {target!r} at {jd} failed: "
                         f"{_lib.STATUS_NAMES.get(int(st[0]), st[0])}")
    return State(target if isinstance(target, str) else int(target), jd, out6[:3, 0],
                 out6[3:, 0], frame, _naif(center))


def _center_shift(from_center, to_center, jd, frame):
    """Offset (pos, vel) to add to a state relative to ``to_center`` to express it relative
    to ``from_center`` -- i.e. the state of ``to_center`` relative to ``from_center``."""
    out6, st = get_states_arrays(to_center, jd, from_center, frame)
    return dict(pos=out6[:3], vel=out6[3:], ok=(st == 0))
