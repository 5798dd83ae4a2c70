"""Build libwql3d.so in-tree for sm_100a with nvcc (no JIT cache, no Python extension).

Each translation unit of csrc/ compiles to its own object in parallel; the
stage-launcher families (stage_*.cu) compile twice, once per precision
(WQL3D_REAL = double / float), and nvcc links the objects into the shared
library.  An object is rebuilt when its source, any header of csrc/ or
include/wql3d.h is newer than it.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

_HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(_HERE)
CSRC = os.path.join(_HERE, "csrc")
OUT = os.path.join(_HERE, "libwql3d.so")
OBJ = os.path.join(_HERE, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-diag-suppress", "177",
]

PRECISIONS = (("f64", "double"), ("f32", "float"))


def units():
    """(object path, source path, extra defines) for every translation unit."""
    out = []
    for f in sorted(os.listdir(CSRC)):
        if not f.endswith(".cu"):
            continue
        src = os.path.join(CSRC, f)
        stem = f[:-3]
        if f.startswith("stage_"):
            for tag, real in PRECISIONS:
                out.append((os.path.join(OBJ, f"{stem}_{tag}.o"), src, [f"-DWQL3D_REAL={real}", f"-DWQL3D_TAG={tag}"]))
        else:
            out.append((os.path.join(OBJ, stem + ".o"), src, []))
    return out


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if not f.endswith(".cu")]
    return hs + [os.path.join(ROOT, "include", "wql3d.h")]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in deps)


def needs_build() -> bool:
    """The library is older than a source or header (objects are only a cache)."""
    return _stale(OUT, [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + _headers())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    heads = _headers()
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    jobs = []
    for obj, src, defs in units():
        if force or _stale(obj, [src] + heads):
            jobs.append([nvcc] + NVCC_FLAGS + inc + defs + ["-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        return subprocess.run(cmd, capture_output=True, text=True)

    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        results = list(ex.map(run, jobs))
    for cmd, r in zip(jobs, results):
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise subprocess.CalledProcessError(r.returncode, cmd)
    link = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT] + [u[0] for u in units()]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.check_call(link)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
