"""Build libtce.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python -m william_ci_b200.build          # or: from william_ci_b200.build import build; build()
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtce.so")
SOURCES = ["tce_api.cu", "tce_kernels.cu", "tce_kernels_s.cu", "tce_kernels_slg.cu", "tce_kernels_tc.cu", "tce_kernels_sp2.cu", "tce_quartets.cu", "tce_lg.cu", "tce_mp2.cu", "tce_onee.cu", "tce_dfjk.cu", "tce_kmo.cu", "tce_df.cu", "tce_lgsetup.cu"]
OBJDIR = os.path.join(HERE, "_build")
HEADERS = ["tce_device.cuh", "tce_kernels.h", "tce_handle.h", "tce_kernels_s.cuh", "tce_kernels_tc.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _mtime(path):
    return os.path.getmtime(path) if os.path.exists(path) else -1.0


def _headers():
    return [os.path.join(CSRC, f) for f in HEADERS] + [os.path.join(ROOT, "include", "tce.h")]


def _compile(src: str, obj: str, verbose: bool, ptxas_info: bool) -> None:
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c",
           "-I", os.path.join(ROOT, "include"), "-o", obj + ".tmp", src]
    if ptxas_info:
        cmd[1:1] = ["-Xptxas", "-v"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s%s" % (src, r.stdout, r.stderr))
    if ptxas_info:
        sys.stdout.write(r.stdout + r.stderr)
    os.replace(obj + ".tmp", obj)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile each source to an object (only when it or a header changed, in
    parallel), then link."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJDIR, exist_ok=True)
    hdr_t = max(_mtime(h) for h in _headers())
    objs, relink, todo = [], force or not os.path.exists(LIB), []
    for f in SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJDIR, f.replace(".cu", ".o"))
        objs.append(obj)
        if force or _mtime(obj) < max(_mtime(src), hdr_t):
            todo.append((src, obj))
            relink = True
        elif _mtime(obj) > _mtime(LIB):
            relink = True
    if todo:
        with ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 1)) as ex:
            for fut in [ex.submit(_compile, s, o, verbose, ptxas_info) for s, o in todo]:
                fut.result()
    if relink:
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
