"""The allocation-free N-body entry point against the regular one.

kete_b200_propagate_n_body_noalloc exists for callers that cannot have device memory
allocated or freed while they run -- cudaMalloc/cudaFree stall the whole device, which a
steady-state propagation loop or a service with a fixed memory budget cannot accept.  It
keeps its per-call scratch in a fixed array inside the library instead.  This file runs
last (pytest collects it after the others) and also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from kete_b200 import synthetic

pytestmark = pytest.mark.gpu

EPOCH = synthetic.EPOCH
TOL_AU = 1e-9  # the N-body position tolerance used throughout the GPU tests


def _bind(lib):
    v = ctypes.c_void_p
    lib.kete_b200_propagate_n_body_noalloc.argtypes = [
        ctypes.c_int64, v, v, v, v, ctypes.c_int, ctypes.c_int64, ctypes.c_int, v, v, v, v, v, v,
        v, v, v]
    lib.kete_b200_propagate_n_body.argtypes = [
        ctypes.c_int64, v, v, v, v, ctypes.c_int, ctypes.c_int64, ctypes.c_int, v, v, v, v, v, v,
        v, v, ctypes.c_int, ctypes.c_int, v]
    lib.kete_b200_last_error.restype = ctypes.c_char_p
    lib.kete_b200_device_allocations.restype = ctypes.c_int64
    return lib


def test_noalloc_matches_regular_entry_point(gpu):
    torch = pytest.importorskip("torch")
    from kete_b200 import _lib

    lib = _bind(_lib.lib())
    n = 3000
    pos, vel, ng = synthetic.mixed(n, seed=91, nongrav_frac=0.2)
    rng = np.random.default_rng(92)
    jd0 = np.full(n, EPOCH)
    jd1 = EPOCH + rng.uniform(-400.0, 400.0, n)  # uneven spans exercise the span ordering
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    P, V, J0, J1, NG = dev(pos), dev(vel), dev(jd0), dev(jd1), dev(ng)
    stream = torch.cuda.current_stream().cuda_stream

    def outputs():
        return (torch.empty((3, n), dtype=torch.float64, device="cuda"),
                torch.empty((3, n), dtype=torch.float64, device="cuda"),
                torch.empty(n, dtype=torch.int32, device="cuda"))

    rp, rv, rs = outputs()
    rc = lib.kete_b200_propagate_n_body(n, P.data_ptr(), V.data_ptr(), J0.data_ptr(),
                                        J1.data_ptr(), 2, 10, 0, NG.data_ptr(), rp.data_ptr(),
                                        rv.data_ptr(), rs.data_ptr(), None, None, None, None,
                                        2, 1, stream)
    assert rc == 0, lib.kete_b200_last_error()
    torch.cuda.synchronize()
    allocations = lib.kete_b200_device_allocations()
    for call in range(2):  # the shared scratch must be reset correctly on every call
        op, ov, os_ = outputs()
        rc = lib.kete_b200_propagate_n_body_noalloc(
            n, P.data_ptr(), V.data_ptr(), J0.data_ptr(), J1.data_ptr(), 2, 10, 0,
            NG.data_ptr(), op.data_ptr(), ov.data_ptr(), os_.data_ptr(), None, None, None, None,
            stream)
        assert rc == 0, lib.kete_b200_last_error()
        torch.cuda.synchronize()
        assert torch.equal(os_, rs), call
        ok = (rs == 0).cpu().numpy()
        assert ok.mean() > 0.99
        err = (op - rp).abs().max(dim=0).values.cpu().numpy()
        assert err[ok].max() < TOL_AU, (call, err[ok].max())
        verr = (ov - rv).abs().max(dim=0).values.cpu().numpy()
        assert verr[ok].max() < TOL_AU, (call, verr[ok].max())
        # the library allocated no device memory for either call
        assert lib.kete_b200_device_allocations() == allocations, call


def test_noalloc_rejects_more_objects_than_its_scratch(gpu):
    torch = pytest.importorskip("torch")
    from kete_b200 import _lib

    lib = _bind(_lib.lib())
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    too_many = 1048576 + 1  # KETE_B200_NOALLOC_MAX_OBJECTS + 1; rejected before any launch
    rc = lib.kete_b200_propagate_n_body_noalloc(too_many, p, p, p, p, 2, 10, 0, None, p, p, p,
                                                None, None, None, None, None)
    assert rc == -1
    assert b"exceed" in lib.kete_b200_last_error()
