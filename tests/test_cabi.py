"""The C-ABI library builds, loads and exports every entry point include/*.h declares.
No compute call is made here (no GPU needed)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        syms.update(re.findall(r"\b(kete_b200_\w+)\s*\(", text))
    return sorted(syms)


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("kete_b200_propagate_two_body", "kete_b200_propagate_n_body",
              "kete_b200_spk_load_file", "kete_b200_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from kete_b200 import build

    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_call_needs_no_gpu():
    from kete_b200 import build

    lib = ctypes.CDLL(build.build())
    assert lib.kete_b200_version() >= 100
