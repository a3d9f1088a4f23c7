"""Build librbx.so (sm_100a) in-tree with nvcc.

The CUDA sources under csrc/ and the C++ host shim under csrc/host/ compile
into rbmd_b200/librbx.so, the C-ABI library declared in include/rbx.h.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librbx.so")

CU_SOURCES = ["rbx_capi.cu", "rbx_capi_f32.cu", "rbx_rbe.cu", "rbx_pair.cu", "rbx_cells.cu", "rbx_engine.cu",
              "rbx_batch.cu", "rbx_adjoint.cu", "rbx_thermo.cu", "rbx_shake.cu",
              "rbx_special.cu", "rbx_rbsog.cu"]
CXX_SOURCES = ["host/config_data.cpp", "host/lj_cut_coul_kspace.cpp", "host/lammps_data.cpp",
               "host/md_files.cpp", "host/special_bonds.cpp",
               "host/rbsog.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _common_flags():
    return ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", "g++",
            "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _compile(src, obj, extra):
    cmd = [nvcc()] + _common_flags() + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(CSRC, "host", f) for f in os.listdir(os.path.join(CSRC, "host"))
                if f.endswith(".h")]
    headers.append(os.path.join(ROOT, "include", "rbx.h"))
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace("/", "_") + ".o")
        objs.append(obj)
        extra = ARCH + (["-Xptxas", "-v"] if ptxas_info else [])
        if ptxas_info or _stale(obj, [src] + headers):
            jobs.append((src, obj, extra))
    for s in CXX_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace("/", "_") + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            jobs.append((src, obj, ["-x", "cu"] + ARCH))
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        futs = {ex.submit(_compile, *j): j for j in jobs}
        for f in cf.as_completed(futs):
            logs.append((futs[f][0], f.result()))
    if jobs or not os.path.exists(LIB):
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs + [
            "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose or ptxas_info:
        for src, log in logs:
            if log.strip():
                print(f"== {os.path.basename(src)}\n{log}", file=sys.stderr)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
