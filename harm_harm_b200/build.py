"""Build the native libraries of harm_harm_b200 in-tree.

  lib/libharm_host.so   host-side input producers (C, OpenMP)         csrc/host_setup.c
  lib/libharm_b200.so   sm_100a kernels and the C ABI (CUDA C++)      csrc/*.cu

The device library is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``)
with the CUDA runtime linked statically, so the built file is self-contained and travels with
the repository tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
INCLUDE = os.path.join(ROOT, "include")

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def host_cc() -> str:
    """A gcc that supports OpenMP (the image's default CC wrapper lacks libgomp)."""
    for cand in ("/usr/bin/gcc", shutil.which("gcc") or ""):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("no gcc found")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC", ""), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc") or ""):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")


def _newer(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_host(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libharm_host.so")
    src = os.path.join(CSRC, "host_setup.c")
    deps = [src, os.path.join(INCLUDE, "harm_b200.h")]
    if force or not _newer(out, deps):
        _run([host_cc(), "-O2", "-fPIC", "-fopenmp", "-shared", "-std=gnu11", "-I" + INCLUDE, "-o", out, src, "-lm"])
    return out


def device_sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def device_flags(src: str) -> list[str]:
    """Per-file flags: the FP64 path is compiled without FMA contraction so that its FP64
    operations are the IEEE operations of the C restatement, in the same order; the mixed
    path uses the fast FP32 division and square root."""
    if src.endswith("_fp64.cu"):
        return ["-fmad=false"]
    if src.endswith("_mixed.cu"):
        # FP32 flux path: fast single-precision division and square root (a few ulp); the
        # FP64 update and inversion in the same file are not affected
        return ["-prec-div=false", "-prec-sqrt=false"]
    return []


def build_device(force: bool = False, extra: list[str] | None = None, out_dir: str | None = None) -> str:
    out_dir = out_dir or LIB
    os.makedirs(out_dir, exist_ok=True)
    objdir = os.path.join(out_dir, "obj")
    os.makedirs(objdir, exist_ok=True)
    out = os.path.join(out_dir, "libharm_b200.so")
    srcs = device_sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(INCLUDE, "harm_b200.h")]
    if force or not _newer(out, srcs + headers):
        objs = []
        for src in srcs:
            obj = os.path.join(objdir, os.path.basename(src) + ".o")
            cmd = [nvcc(), *NVCC_ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE,
                   "-I" + CSRC, *device_flags(src), *(extra or []), "-c", "-o", obj, src]
            _run(cmd)
            objs.append(obj)
        _run([nvcc(), *NVCC_ARCH, "-shared", "--cudart", "static", "-o", out, *objs])
    return out


def build_oracle(force: bool = False) -> str:
    """Build the CPU oracle (test infrastructure) through its Makefile."""
    cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle")]
    if force:
        cmd.insert(1, "-B")
    _run(cmd)
    return os.path.join(ROOT, "oracle", "build", "liborc.so")


def build_all(force: bool = False) -> None:
    build_host(force)
    build_device(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    if "--oracle" in sys.argv:
        build_oracle(force="--force" in sys.argv)
    print("built:", os.listdir(LIB))
