"""Build the engine library crpropa3_b200/lib/libcrp_b200.so for sm_100a.

nvcc cross-compiles without a GPU.  The FP64 stepping translation unit is
compiled with -fmad=false so that no multiply-add is contracted (bit parity
with the reference built without FMA); the other units use the default
contraction.  Objects go to _build/ at the repository root.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "lib", "libcrp_b200.so")
# microbenchmarks of the roofline denominators (benchmark only)
PEAKS_LIB = os.path.join(PKG, "lib", "libcrp_peaks.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]

# source -> extra flags
SOURCES = {
    "step_fp64.cu": ["-fmad=false"],
    "step_mixed.cu": [],
    "step_mixed_bp.cu": [],
    "adjoint.cu": [],
    "turbulence.cu": [],
    "crp_engine.cu": [],
    "source.cu": [],
    "noalloc.cu": [],
    "host_tools.cpp": ["-Xcompiler", "-ffp-contract=off"],
}
PEAKS_SOURCES = {"peaks.cu": []}
LINK_LIBS = ["-lcufft", "-lz"]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


_INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(path, seen=None):
    """The source and every header it includes with #include "..." (found
    next to the including file, in csrc/ or in include/), recursively."""
    seen = set() if seen is None else seen
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path, encoding="utf-8", errors="replace") as f:
        text = f.read()
    for name in _INCLUDE_RE.findall(text):
        for d in (os.path.dirname(path), CSRC, INCLUDE):
            cand = os.path.join(d, name)
            if os.path.exists(cand):
                _deps(cand, seen)
                break
    return seen


def _compile(nvcc, src, flags, verbose):
    out = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = sorted(_deps(path)) + [os.path.abspath(__file__)]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    cmd = [nvcc] + ARCH + COMMON + flags
    if src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    cmd += ["-c", path, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr[-6000:]}")
    with open(out + ".log", "w") as f:
        f.write(r.stderr)
    if verbose:
        print(f"[build] {src}", file=sys.stderr)
    return out


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    nvcc = _nvcc()
    missing = [s for s in SOURCES if not os.path.exists(os.path.join(CSRC, s))]
    if missing:
        raise RuntimeError(f"engine sources missing: {missing}")
    present = SOURCES
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda kv: _compile(nvcc, kv[0], kv[1], verbose), present.items()))
        pobjs = list(ex.map(lambda kv: _compile(nvcc, kv[0], kv[1], verbose), PEAKS_SOURCES.items()))
    _link(nvcc, LIB, objs, LINK_LIBS)
    _link(nvcc, PEAKS_LIB, pobjs, [])
    return LIB


def _link(nvcc, lib, objs, libs):
    if os.path.exists(lib) and all(os.path.getmtime(lib) >= os.path.getmtime(o) for o in objs):
        return
    cmd = [nvcc] + ARCH + ["-shared", "-o", lib] + objs + ["-L/usr/local/cuda/lib64"] + libs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link of {os.path.basename(lib)} failed:\n{r.stderr[-6000:]}")


if __name__ == "__main__":
    print(build(verbose=True))
