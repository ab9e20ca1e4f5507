"""Build libqnd_b200.so in-tree for sm_100a.

    python -m tdse_nd_mpi_b200.build        (or tdse_nd_mpi_b200.build.build())

Compiles csrc/qnd_pass_inst.cu once per supported line length (-DQND_L=...), the
auxiliary kernels and the host engine, in parallel, then links a shared library
with a plain C ABI (include/qnd.h). Objects go to tdse_nd_mpi_b200/_build/.
Rebuilds only what is older than its sources.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libqnd_b200.so")
LENGTHS = (2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")] + ARCH


def _nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _deps():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdrs.append(os.path.join(ROOT, "include", "qnd.h"))
    return max(os.path.getmtime(h) for h in hdrs)


def _jobs():
    jobs = []
    for L in LENGTHS:
        jobs.append((os.path.join(CSRC, "qnd_pass_inst.cu"), os.path.join(BUILD, f"qnd_pass_L{L}.o"), [f"-DQND_L={L}"]))
    for name in ("qnd_aux", "qnd_engine"):
        jobs.append((os.path.join(CSRC, name + ".cu"), os.path.join(BUILD, name + ".o"), []))
    # the persistent sweep kernel, one precision per object (the longest compilations: start them first)
    for fp64 in (1, 0):
        jobs.insert(0, (os.path.join(CSRC, "qnd_sweep.cu"), os.path.join(BUILD, f"qnd_sweep_fp{64 if fp64 else 32}.o"),
                        [f"-DQND_SWEEP_FP64={fp64}"]))
    return jobs


def _compile(job, nvcc, verbose):
    src, obj, extra = job
    cmd = [nvcc] + NVFLAGS + extra + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(obj)}:\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    dep_time = _deps()
    todo = []
    for job in _jobs():
        src, obj, _ = job
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(dep_time, os.path.getmtime(src)):
            todo.append(job)
    if todo:
        workers = jobs or max(1, min(len(todo), os.cpu_count() or 4))
        with cf.ThreadPoolExecutor(workers) as ex:
            for obj, log in ex.map(lambda j: _compile(j, nvcc, verbose), todo):
                if verbose and log:
                    print(log, file=sys.stderr)
    objs = [obj for _, obj, _ in _jobs()]
    if force or todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc, "-shared"] + ARCH + ["-o", tmp] + objs + ["-lcudart", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(tmp, LIB)
    build_drivers(force)
    return LIB


DRIVERS = {"QuantumND_imag": ["quantumnd_imag.c", "params.c"], "QuantumND_real": ["quantumnd_real.c", "params.c"]}


def build_drivers(force: bool = False) -> list[str]:
    """The drop-in C drivers (drivers/*.c), linked against libqnd_b200.so next to them."""
    cc = shutil.which("gcc") or "cc"
    src_dir = os.path.join(PKG, "drivers")
    out = []
    for exe, srcs in DRIVERS.items():
        target = os.path.join(PKG, exe)
        paths = [os.path.join(src_dir, f) for f in srcs]
        deps = paths + [os.path.join(src_dir, "params.h"), os.path.join(ROOT, "include", "qnd.h"), LIB]
        if force or not os.path.exists(target) or os.path.getmtime(target) < max(os.path.getmtime(d) for d in deps):
            cmd = [cc, "-O2", "-std=gnu11", "-I", os.path.join(ROOT, "include"), "-o", target] + paths + \
                  ["-L", PKG, "-lqnd_b200", "-Wl,-rpath,$ORIGIN", "-lm"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"driver build failed ({exe}):\n{r.stderr}")
        out.append(target)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
