"""Build recipe for libketeb200.so (sm_100a only).

Run ``python -m kete_b200.build`` (or ``__graft_entry__.build()``).  The shared library is
written next to this file so it travels with the source tree; nothing is installed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libketeb200.so")
OBJ_DIR = os.path.join(HERE, "_build")  # object files of the incremental build (not shipped)
SOURCES = ["sens.cu", "adjoint.cu", "nodes.cu", "kernels.cu", "long.cu", "capi.cu",
           "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the kete_b200 CUDA library cannot be built")


def host_compiler() -> list[str]:
    # /usr/bin/g++ is the image's full toolchain; another g++ early on PATH may lack parts
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def sources() -> list[str]:
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "kete_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, obj: str, ptxas_info: bool) -> subprocess.CompletedProcess:
    cmd = [nvcc(), *host_compiler(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-c",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-I", os.path.join(HERE, "..", "include"),
           "-o", obj, src]
    if ptxas_info:
        cmd.insert(1, "-Xptxas=-v")
    return subprocess.run(cmd, capture_output=True, text=True)


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    """Compile the translation units whose sources or headers changed to object files under
    kete_b200/_build (in parallel), then link the shared library next to this file."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(OBJ_DIR, os.path.basename(s) + ".o") for s in srcs]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if not f.endswith(".cu")]
    headers.append(os.path.join(HERE, "..", "include", "kete_b200.h"))
    newest_header = max(os.path.getmtime(h) for h in headers if os.path.exists(h))
    todo = [(s, o) for s, o in zip(srcs, objs)
            if force or ptxas_info or not os.path.exists(o)
            or os.path.getmtime(o) < max(newest_header, os.path.getmtime(s))]
    if todo:
        with ThreadPoolExecutor(max_workers=len(todo)) as ex:
            results = list(ex.map(lambda so: _compile(so[0], so[1] + ".tmp", ptxas_info), todo))
        for (s, o), res in zip(todo, results):
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed on {os.path.basename(s)}:\n" + res.stdout + res.stderr)
            if verbose or ptxas_info:
                print(res.stdout + res.stderr, file=sys.stderr)
            os.replace(o + ".tmp", o)
    link = [nvcc(), *host_compiler(), *ARCH, "--shared", "-o", LIB + ".tmp", *objs,
            "-lcudart_static", "-ldl", "-lpthread", "-lrt"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv, force=True)
    print(LIB)
