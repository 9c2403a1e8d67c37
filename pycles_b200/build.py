"""Build ``pycles_b200/lib/libpycles_b200.so`` for sm_100a (in-tree).

    python -m pycles_b200.build [--force]

The library is one nvcc translation unit (csrc/pb_all.cu) exporting the
C ABI declared in include/pycles_b200.h.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpycles_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "-diag-suppress", "177",
]


def _sources():
    out = [os.path.join(ROOT, "include", "pycles_b200.h")]
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cuh")):
            out.append(os.path.join(CSRC, f))
    return out


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in _sources())


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


# Translation units and their extra flags.  The thermodynamics, the FP64
# plain-form advection, the surface fluxes, the subgrid scale, the
# statistics and the forcing are compiled without FMA contraction so that they
# follow the reference's separately rounded arithmetic (see csrc/crmath.cuh
# and csrc/advection_f64.cu).
UNITS = [("pb_all.cu", []), ("thermo.cu", ["-fmad=false"]), ("advection_f64.cu", ["-fmad=false"]),
         ("thermo_fast.cu", []), ("surface.cu", ["-fmad=false"]), ("sgs.cu", ["-fmad=false"]),
         ("stats.cu", ["-fmad=false"]), ("forcing.cu", ["-fmad=false"]),
         ("radiation.cu", ["-fmad=false"])]


def _run(cmd):
    r = subprocess.run(cmd, cwd=CSRC, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout.decode()[-4000:])
    return r.stdout.decode()


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    from concurrent.futures import ThreadPoolExecutor
    objs, cmds = [], []
    for src, extra in UNITS:
        obj = os.path.join(LIBDIR, src.replace(".cu", ".o"))
        cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
        cmd.remove("-shared")
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(obj)
    with ThreadPoolExecutor(len(cmds)) as ex:
        log = list(ex.map(_run, cmds))
    tmp = LIB + ".tmp"
    _run([nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC"] + objs
         + ["-o", tmp])
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
