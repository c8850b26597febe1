"""Build the sm_100a shared library ``chromatix_b200/_lib/libcx_b200.so``.

nvcc compiles every ``csrc/*.cu`` for ``sm_100a`` (cross-compiles without a
GPU) in parallel and links them with the static CUDA runtime, so the library
exports only the C ABI of ``include/cx_b200.h`` and carries no torch types.

    python -m chromatix_b200.build [--force] [-j N]
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libcx_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-v", "-I", INCLUDE]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return sorted(hs)


def _digest(path: str, headers) -> str:
    h = hashlib.sha256()
    for p in [path] + list(headers):
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()[:16]


def _compile(src: str, headers, force: bool):
    base = os.path.splitext(os.path.basename(src))[0]
    obj = os.path.join(OBJ_DIR, base + ".o")
    stamp = obj + ".sha"
    dg = _digest(src, headers)
    if not force and os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == dg:
        return obj, None
    cmd = [_nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr[-6000:]}")
    with open(stamp, "w") as f:
        f.write(dg)
    with open(os.path.join(OBJ_DIR, base + ".ptxas.txt"), "w") as f:
        f.write(r.stderr)
    return obj, r.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    """Compile all kernels and link the shared library; returns its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    headers = _headers()
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, headers, force), srcs))
    objs = [o for o, _ in results]
    relink = force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)
    if relink:
        tmp = LIB + ".tmp"
        cmd = [_nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
        os.replace(tmp, LIB)
    if verbose:
        for o, log in results:
            if log:
                print(log[-3000:])
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.j, a.v))


if __name__ == "__main__":
    sys.exit(main())
