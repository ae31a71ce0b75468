"""Builds the sm_100a shared library ``lib/libleco_b200.so`` with nvcc.

The library is compiled in-tree (no JIT cache) so the built file travels with
the repository snapshot.  Host code is compiled with -ffp-contract=off and
device code with --fmad=false: the codec's FP64 model arithmetic must round
every multiply and add separately, exactly as the reference's
-ffp-contract=off build does.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libleco_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    inc = os.path.join(os.path.dirname(HERE), "include")
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [__file__])


FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off"]


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object file in parallel (one nvcc per file),
    then links the shared library."""
    if not force and up_to_date():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    obj_dir = os.path.join(LIB_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    extra = ["-Xptxas=-v"] if verbose else []
    jobs = []
    newest_header = max(os.path.getmtime(f) for f in headers() + [__file__])
    for src in sources():
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        # an object is reused only when it is newer than its source, every header and this script
        fresh = (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                 and os.path.getmtime(obj) >= newest_header)
        jobs.append((obj, None if fresh else [nvcc, *ARCH, *FLAGS, *extra, "-c", "-o", obj, src]))
    if verbose:
        for _, cmd in jobs:
            if cmd:
                print(" ".join(cmd), file=sys.stderr)
    procs = [(subprocess.Popen(cmd), cmd) for _, cmd in jobs if cmd]
    failed = [" ".join(cmd) for p, cmd in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    subprocess.check_call([nvcc, *ARCH, "-shared", "-o", LIB + ".tmp", *[o for o, _ in jobs], "-lpthread"])
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
