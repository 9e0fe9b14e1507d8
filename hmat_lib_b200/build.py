"""Builds libhodlr_b200.so in-tree with nvcc for sm_100a.

    python -m hmat_lib_b200.build [--force]

Objects go to hmat_lib_b200/_build/ (compiled in parallel, rebuilt when a
source or header is newer); the shared library lands next to this file so it
travels with the source tree.
"""
from __future__ import annotations

import glob
import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libhodlr_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE,
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def source_hash() -> str:
    """SHA-256 (first 16 hex digits) of every source and header the library
    is built from (csrc/ and include/hmat_lib/, paths and contents, sorted).
    Compiled into the library and returned by hodlr_b200_version(), so a
    caller can tell whether a binary was built from the sources beside it."""
    files = sorted(_sources() + glob.glob(os.path.join(CSRC, "*.h")) +
                   glob.glob(os.path.join(CSRC, "*.cuh")) +
                   glob.glob(os.path.join(INCLUDE, "hmat_lib", "*.h")))
    h = hashlib.sha256()
    for f in files:
        h.update(os.path.relpath(f, os.path.dirname(HERE)).encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def _hash_object(force: bool):
    """Object file defining hb_source_hash() for the current sources."""
    digest = source_hash()
    src = os.path.join(BUILD, "source_hash.cpp")
    text = ('// generated by hmat_lib_b200/build.py\n'
            f'extern "C" const char *hb_source_hash(void) {{ return "{digest}"; }}\n')
    old = open(src).read() if os.path.exists(src) else None
    if old != text:
        with open(src, "w") as f:
            f.write(text)
    return _compile(src, force, 0.0)


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "hmat_lib", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, force, hdr_time):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj):
        t = os.path.getmtime(obj)
        if t >= os.path.getmtime(src) and t >= hdr_time:
            return obj, None
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj, None


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr = _newest_header()
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force, hdr), srcs))
    results.append(_hash_object(force))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT)
                                                for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-Xlinker", "-Bsymbolic",
               "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("built", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
