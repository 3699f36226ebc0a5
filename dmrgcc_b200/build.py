"""Builds libdmrg_b200.so (CUDA kernels + C ABI + C++ host engine) for sm_100a.

    python -m dmrgcc_b200.build [--force] [--jobs N]

Every translation unit under csrc/ is compiled in-tree into dmrgcc_b200/lib/
(object files in dmrgcc_b200/lib/obj/), then linked into one shared library;
the reference's model executables (csrc/apps/) are linked against it beside it.
A unit is recompiled when it, or any header under csrc/ or include/, is newer
than its object file.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libdmrg_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cxx() -> str:
    # The system compiler; an inherited CXX may point at a toolchain without libgomp.
    return shutil.which("g++", path="/usr/bin") or "g++"


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "host", "*.cc")))


def headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(CSRC, "host", "*.h")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def obj_of(src: str) -> str:
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(OBJDIR, rel + ".o")


def compile_one(src: str) -> tuple[str, str]:
    obj = obj_of(src)
    common = ["-I", INCLUDE, "-I", CSRC, "-O3"]
    if src.endswith(".cu"):
        cmd = [nvcc(), *ARCH, "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
               "-Xptxas", "-warn-spills", *common, "-c", src, "-o", obj]
    else:
        cmd = [cxx(), "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function", *common,
               "-I", "/usr/local/cuda/include", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return src, (r.stdout + r.stderr).strip()


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    hdr_time = max((os.path.getmtime(h) for h in headers()), default=0.0)
    todo = []
    for s in sources():
        o = obj_of(s)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time):
            todo.append(s)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            for src, msg in ex.map(compile_one, todo):
                if verbose or ("warning" in msg.lower() and "spill" in msg.lower()):
                    print(f"[build] {os.path.relpath(src, ROOT)}: {msg}", file=sys.stderr)
    objs = [obj_of(s) for s in sources()]
    if todo or force or not os.path.exists(LIB):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-Xlinker", "--no-undefined"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    build_apps(force)
    return LIB


# The reference's model executables (csrc/apps/model_main.cc), one per model,
# linked against the library next to them.
APPS = {"real_spinless_bose_square_model": "real_spinless_bose_square",
        "complex_spinless_bose_square_model": "complex_spinless_bose_square",
        "complex_spinful_bose_square_model": "complex_spinful_bose_square",
        "real_spinful_bose_square_model": "real_spinful_bose_square"}


def build_apps(force: bool = False) -> list[str]:
    src = os.path.join(CSRC, "apps", "model_main.cc")
    deps = [src, LIB, os.path.join(INCLUDE, "dmrg_b200.h"), os.path.join(INCLUDE, "dmrg_b200.hpp")]
    newest = max(os.path.getmtime(d) for d in deps)
    out = []
    for exe, model in APPS.items():
        path = os.path.join(LIBDIR, exe)
        if force or not os.path.exists(path) or os.path.getmtime(path) < newest:
            cmd = [cxx(), "-std=c++17", "-O2", "-Wall", "-Wextra", f'-DDMRG_MODEL="{model}"', "-I", INCLUDE, src,
                   "-L", LIBDIR, "-ldmrg_b200", "-Wl,-rpath,$ORIGIN", "-o", path]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"build of {exe} failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        out.append(path)
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.jobs, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
