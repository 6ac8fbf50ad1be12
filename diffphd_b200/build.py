"""Builds libdiffphd_b200.so in-tree for sm_100a with nvcc (no JIT, no torch extension cache).

    python -m diffphd_b200.build [--verbose-ptxas]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libdiffphd_b200.so"
SOURCES = ["kernels.cu", "engine.cu", "setup.cpp", "capi.cpp", "noalloc.cu", "contact.cu", "mlp.cu", "mlp_tc.cu",
           "sfactor_plan.cpp", "sfactor_gpu.cu", "contact_precond.cu",
           "ncp_cached.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx():
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")


def build(verbose_ptxas: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    deps = list(CSRC.glob("*")) + [PKG.parent / "include" / "diffphd_b200.h"]
    newest = max(p.stat().st_mtime for p in deps)
    if LIB.exists() and LIB.stat().st_mtime >= newest and not force:
        return LIB
    common = ["-O3", "-std=c++17", "-lineinfo", "-ccbin", _host_cxx(), "-Xcompiler", "-fPIC,-fopenmp,-O3",
              "-I", str(PKG.parent / "include")] + ARCH
    def compile_one(src):
        obj = BUILD / (src + ".o")
        cmd = [nvcc, "-c", str(CSRC / src), "-o", str(obj)] + common
        if verbose_ptxas and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        return src, obj, subprocess.run(cmd, capture_output=True, text=True)

    objs = []
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        for src, obj, res in ex.map(compile_one, SOURCES):
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
            if verbose_ptxas and res.stderr:
                sys.stderr.write(f"--- {src}\n" + res.stderr)
            objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, "-shared", "-o", str(tmp)] + objs + ARCH + ["-ccbin", _host_cxx(), "-Xcompiler", "-fopenmp",
                                                             "-lgomp", "-cudart", "static"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv))
