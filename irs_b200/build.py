"""Build the irs_b200 shared libraries for sm_100a with nvcc.

Produces, under irs_b200/lib/:
  lib_ipm.so, lib_ipm_double.so   IPM, float / double (reference lib_ipm.so ABI)
  lib_irs.so, lib_irs_double.so   IRS, float / double (same conventions)
  lib_ccf.so                      critical curves, double (reference lib_ccf.so ABI)
  lib_ncc.so                      caustic-crossing maps, double (reference lib_ncc.so ABI)
and under irs_b200/bin/ the command-line tools of the reference
(src/main_ipm_irs.cu, src/main_ccf.cu, src/main_ncc.cu): ipm_gpu,
ipm_gpu_double, irs_gpu, irs_gpu_double, ccf_gpu, ncc_gpu.

Usage: python -m irs_b200.build [--jobs N] [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BINDIR = os.path.join(HERE, "bin")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-std=c++17",
    "-O3",
    "-lineinfo",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fopenmp",  # host-side copies of the maps
    "-shared",
    "--expt-relaxed-constexpr",
]

EXECUTABLES = {
    "ipm_gpu": ["-DIRSB_DOUBLE=0", "-DIRSB_IRS=0"],
    "ipm_gpu_double": ["-DIRSB_DOUBLE=1", "-DIRSB_IRS=0"],
    "irs_gpu": ["-DIRSB_DOUBLE=0", "-DIRSB_IRS=1"],
    "irs_gpu_double": ["-DIRSB_DOUBLE=1", "-DIRSB_IRS=1"],
}

VARIANTS = {
    "lib_ipm.so": ["-DIRSB_DOUBLE=0", "-DIRSB_IRS=0"],
    "lib_ipm_double.so": ["-DIRSB_DOUBLE=1", "-DIRSB_IRS=0"],
    "lib_irs.so": ["-DIRSB_DOUBLE=0", "-DIRSB_IRS=1"],
    "lib_irs_double.so": ["-DIRSB_DOUBLE=1", "-DIRSB_IRS=1"],
}


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh", ".hpp", ".h"))]


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in _sources())


def build_one(name: str, defs, force: bool = False, extra=None, source: str = "capi.cu") -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, name)
    if not force and not _stale(out):
        return out
    cmd = [nvcc()] + NVCC_FLAGS + list(defs) + list(extra or []) + [
        "-I", CSRC, os.path.join(CSRC, source), "-o", out + ".tmp", "-lcurand", "-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed for {name}")
    os.replace(out + ".tmp", out)
    return out


def build_exe(name: str, defs, force: bool = False, source: str = "cli.cu") -> str:
    os.makedirs(BINDIR, exist_ok=True)
    out = os.path.join(BINDIR, name)
    if not force and not _stale(out):
        return out
    flags = [f for f in NVCC_FLAGS if f not in ("-shared",)]
    cmd = [nvcc()] + flags + list(defs) + ["-I", CSRC, os.path.join(CSRC, source), "-o", out + ".tmp",
                                            "-lcurand", "-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed for {name}")
    os.replace(out + ".tmp", out)
    return out


def build(force: bool = False, jobs: int = 4, extra=None, executables: bool = True) -> list[str]:
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(build_one, n, d, force, extra) for n, d in VARIANTS.items()]
        futs.append(ex.submit(build_one, "lib_ccf.so", [], force, extra, "ccf_capi.cu"))
        futs.append(ex.submit(build_one, "lib_ncc.so", [], force, extra, "ncc_capi.cu"))
        if executables:
            futs += [ex.submit(build_exe, n, d, force) for n, d in EXECUTABLES.items()]
            futs.append(ex.submit(build_exe, "ccf_gpu", [], force, "cli_ccf.cu"))
            futs.append(ex.submit(build_exe, "ncc_gpu", [], force, "cli_ncc.cu"))
        return [f.result() for f in cf.as_completed(futs)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=4)
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_verbose else None
    for p in build(a.force, a.jobs, extra):
        print(p)


if __name__ == "__main__":
    main()
