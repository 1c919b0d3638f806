"""Build ``libqedf.so`` in-tree for sm_100a with nvcc (no torch involved)."""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libqedf.so")
SOURCES = ["qedf_ops.cu", "qedf_pcg.cu", "qedf_capi.cu", "qedf_static.cu", "qedf_bond.cu", "qedf_fmass.cu"]
HEADERS = ["qedf_common.cuh", "qedf_slice.cuh", "qedf_internal.h", "qedf_precon_table.h"]
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-diag-suppress", "20013,20015"]


def _newest_input():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(HERE, "..", "include", "qedf.h"))
    return max(os.path.getmtime(f) for f in files)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library unless it is newer than every source; returns its path."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input():
        return LIB
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    # one nvcc per translation unit, in parallel, then one link
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        procs.append((src, subprocess.Popen([nvcc] + FLAGS + ["-c", "-o", obj, src], cwd=CSRC,
                                            stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    for src, pr in procs:
        out, err = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src} ({pr.returncode}):\n{err[-4000:]}")
        if verbose:
            print(err[-2000:])
    tmp = LIB + ".tmp"
    objs = [os.path.join(objdir, s.replace(".cu", ".o")) for s in SOURCES]
    res = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp] + objs,
                         capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed ({res.returncode}):\n{res.stderr[-4000:]}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
