"""ctypes binding of libketeb200.so -- the only compute path of this package.

There is no CPU fallback: if the CUDA library is missing or no GPU is visible, calls
raise.  Array arguments are numpy arrays (host) or torch CUDA tensors (device); the
helpers below turn them into pointers and pick the host/device mode of the C ABI.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libketeb200.so")

OK, CONVERGENCE, VALUE_ERROR, DAF_LIMITS, UNKNOWN_FRAME, IO_ERROR, IMPACT, TIMEOUT = range(8)
STATUS_NAMES = {0: "Ok", 1: "Convergence", 2: "ValueError", 3: "DAFLimits", 4: "UnknownFrame",
                5: "IOError", 6: "Impact", 7: "Timeout"}
FRAME_EQUATORIAL, FRAME_ECLIPTIC = 1, 2
MODE_AUTO, MODE_THREAD, MODE_NODES = 0, 1, 2

_lib = None
_initialised = set()

_dp = C.c_void_p


class KeteB200Error(RuntimeError):
    """A call into the CUDA library failed."""


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m kete_b200.build` "
                "(kete_b200 has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        v = C.c_void_p
        L.kete_b200_version.restype = C.c_int
        L.kete_b200_init.argtypes = [C.c_int]
        L.kete_b200_last_error.restype = C.c_char_p
        L.kete_b200_spk_load_file.argtypes = [C.c_char_p]
        L.kete_b200_spk_load_buffer.argtypes = [C.c_char_p, C.c_int64]
        L.kete_b200_spk_loaded_ids.argtypes = [v, C.c_int]
        L.kete_b200_spk_get_states.argtypes = [C.c_int64, C.c_int64, v, C.c_int64, C.c_int, v, v,
                                               C.c_int, v]
        L.kete_b200_propagate_two_body.argtypes = [C.c_int64, v, v, v, v, v, v, v, v, v, C.c_int,
                                                   v]
        L.kete_b200_propagate_n_body.argtypes = [C.c_int64, v, v, v, v, C.c_int, C.c_int64,
                                                 C.c_int, v, v, v, v, v, v, v, v, C.c_int,
                                                 C.c_int, v]
        L.kete_b200_radau_central.argtypes = [C.c_int64, v, v, v, v, v, v, v, C.c_int, v]
        _lib = L
    return _lib


def check(rc: int):
    if rc != 0:
        msg = lib().kete_b200_last_error().decode(errors="replace")
        if rc == -3:
            raise ValueError(msg)
        raise KeteB200Error(f"kete_b200 error {rc}: {msg}")


def init(device: int | None = None):
    """Select and prepare the CUDA device (once per device)."""
    if device is None:
        try:
            import torch

            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        except Exception:  # torch absent or no GPU: let the library report it
            device = 0
    if device not in _initialised:
        check(lib().kete_b200_init(int(device)))
        _initialised.add(device)


def _is_torch_cuda(a) -> bool:
    return type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False)


class Args:
    """Collects array pointers for one call; all arrays must live on the same side."""

    def __init__(self):
        self.keep = []
        self.device = None
        self.stream = None

    def ptr(self, a, dtype=np.float64):
        if a is None:
            return None
        if _is_torch_cuda(a):
            if self.device is False:
                raise ValueError("mixing host and device arrays in one call")
            self.device = True
            if not a.is_contiguous():
                raise ValueError("device arrays must be contiguous")
            if self.stream is None:
                import torch

                self.stream = torch.cuda.current_stream(a.device).cuda_stream
            self.keep.append(a)
            return a.data_ptr()
        if self.device is True:
            raise ValueError("mixing host and device arrays in one call")
        self.device = False
        if not isinstance(a, np.ndarray) or a.dtype != dtype:
            raise TypeError("host arrays must be numpy arrays of " + np.dtype(dtype).name)
        if not a.flags.c_contiguous:
            a = np.ascontiguousarray(a)  # inputs only: outputs are allocated contiguous
        self.keep.append(a)
        return a.ctypes.data

    @property
    def on_device(self) -> int:
        return 1 if self.device else 0
