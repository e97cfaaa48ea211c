"""In-tree build of the native core for sm_100a.

Produces
  libdescriptor_b200/_lib/libldb200.so      C ABI (include/libdescriptor_b200.h):
                                             CUDA kernels + host core
  libdescriptor_b200/_lib/libldb200_cxx.so  the reference's C++ driver API
                                             (include/cxx/Descriptors.hpp) over it
  libdescriptor_b200/_libdescriptor*.so      pybind11 module over that ABI

Run ``python libdescriptor_b200/build.py`` (or ``__graft_entry__.build()``); the
file is loaded by path because importing the package needs the built extension.
nvcc cross-compiles without a GPU.  Objects are cached under
``libdescriptor_b200/_build/`` and rebuilt when a source or header changes.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libldb200.so")
EXT = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
MOD = os.path.join(HERE, "_libdescriptor" + EXT)
CXX_LIB = os.path.join(LIBDIR, "libldb200_cxx.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-I" + INCLUDE, "-I" + CSRC] + os.environ.get("LDB_NVCC_DEFINES", "").split()
CORE_SOURCES = ["ld_sf.cu", "ld_bs.cu", "ld_util.cu", "ld_core.cpp", "ld_neighbor.cpp", "ld_noalloc.cu",
                "ld_bs2_j0_1_2_3_4.cu", "ld_bs2_j5_6.cu", "ld_bs2_j7.cu", "ld_bs2_j8.cu", "ld_bs2_j9.cu",
                "ld_bs2_j10.cu", "ld_serve.cpp", "ld_sfg.cu", "ld_neighbor_dev.cu", "ld_sfp.cu"]
# host threads for the serving runtime's request staging
EXTRA_FLAGS = {"ld_serve.cpp": ["-Xcompiler", "-fopenmp"]}
HEADERS = [os.path.join(CSRC, "ld_internal.h"), os.path.join(CSRC, "ld_neighbor_math.h"), os.path.join(CSRC, "ld_sf_common.cuh"), os.path.join(CSRC, "ld_csr.cuh"), os.path.join(CSRC, "ld_bulk.cuh"), os.path.join(CSRC, "ld_bs2.cuh"),
           os.path.join(CSRC, "ld_bs2_impl.cuh"), os.path.join(INCLUDE, "libdescriptor_b200.h")]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")


def build(verbose: bool = False, jobs: int | None = None) -> None:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    objs, todo = [], []
    for src in CORE_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _stale(o, [s] + HEADERS):
            todo.append([nvcc] + NVCC_FLAGS + EXTRA_FLAGS.get(src, []) + ["-c", s, "-o", o])
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for f in [ex.submit(_run, c, verbose) for c in todo]:
                f.result()
    if _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread", "-lgomp"], verbose)
    # the C++ driver API (include/cxx/Descriptors.hpp) over the C ABI
    cxx = shutil.which("g++") or "g++"
    shim = os.path.join(CSRC, "ld_cxx.cpp")
    shim_deps = [shim, LIB, os.path.join(INCLUDE, "cxx", "Descriptors.hpp"), os.path.join(CSRC, "ld_fd.h")] + HEADERS
    if _stale(CXX_LIB, shim_deps):
        _run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I" + INCLUDE, shim, "-L" + LIBDIR, "-lldb200",
              "-Wl,-rpath,$ORIGIN", "-o", CXX_LIB], verbose)
    pyb = os.path.join(CSRC, "ld_pybind.cpp")
    if _stale(MOD, [pyb, LIB, os.path.join(CSRC, "ld_fd.h")] + HEADERS):
        import pybind11

        py_inc = sysconfig.get_paths()["include"]
        _run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
              "-I" + INCLUDE, "-I" + pybind11.get_include(), "-I" + py_inc, pyb,
              "-L" + LIBDIR, "-lldb200", "-Wl,-rpath,$ORIGIN/_lib", "-o", MOD], verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
    print(MOD)
