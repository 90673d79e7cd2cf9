"""Build the native libraries in-tree (mdelast_b200/lib/):

* ``libmdelast_cuda.so``: the CUDA kernels and the C-ABI of ``include/mdelast.h``,
  compiled for sm_100a only;
* ``md_driver_module<ext>.so``: the pybind11 module that mirrors the reference's
  ``md_driver_module`` on top of that C-ABI;
* ``data/potentials/``: the potential files of an mdelast checkout, when one is found
  (``$MDELAST_REFERENCE``, else a checkout called ``reference`` beside this repository).
  Their licences keep them out of this repository's history; the directory is ignored by
  git and read by ``mdelast_b200.potentials.find_potential``.

Run ``python -m mdelast_b200.build``. Nothing here needs a GPU.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["atom_kernels.cu", "mixed_kernels.cu", "scalar_kernels.cu", "gr_kernels.cu", "gr_static.cu", "mlp.cu", "driver.cu"]
HOST_SOURCES = ["host_tables.cpp", "host_fluct.cpp"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda_library(verbose_ptxas=False):
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libmdelast_cuda.so")
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "mdelast.h"))
    srcs = [os.path.join(CSRC, f) for f in CUDA_SOURCES + HOST_SOURCES]
    if not _stale(out, srcs + headers) and not verbose_ptxas:
        return out
    objs, cmds = [], []
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    for f in CUDA_SOURCES:
        o = os.path.join(obj_dir, f + ".o")
        cmd = [NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
               "-I" + INCLUDE, "-I" + CSRC, "-c", os.path.join(CSRC, f), "-o", o]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(o)
    for f in HOST_SOURCES:
        o = os.path.join(obj_dir, f + ".o")
        cmds.append(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-Wextra", "-I" + INCLUDE,
                     "-I" + CSRC, "-c", os.path.join(CSRC, f), "-o", o])
        objs.append(o)
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for f in [pool.submit(_run, c) for c in cmds]:
            f.result()
    _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-lcudart"])
    return out


def build_python_module():
    import pybind11

    ext = sysconfig.get_config_var("EXT_SUFFIX")
    out = os.path.join(LIB, "md_driver_module" + ext)
    src = os.path.join(CSRC, "md_driver_module.cpp")
    deps = [src, os.path.join(INCLUDE, "mdelast.h"), os.path.join(LIB, "libmdelast_cuda.so")]
    if not _stale(out, deps):
        return out
    _run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-Wall", "-Wextra",
          "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
          "-I" + INCLUDE, src, "-o", out, "-L" + LIB, "-lmdelast_cuda",
          "-Wl,-rpath,$ORIGIN"])
    return out


def reference_checkout():
    """The mdelast checkout next to this repository, or None."""
    for c in (os.environ.get("MDELAST_REFERENCE"), os.path.join(os.path.dirname(ROOT), "reference")):
        if c and os.path.isdir(os.path.join(c, "potentials")):
            return os.path.abspath(c)
    return None


def stage_potentials():
    """Copy the checkout's potential files into ``data/potentials`` (unchanged files are
    left alone). Returns the number of files staged."""
    ref = reference_checkout()
    if ref is None:
        return 0
    src_dir = os.path.join(ref, "potentials")
    dst_dir = os.path.join(HERE, "data", "potentials")
    os.makedirs(dst_dir, exist_ok=True)
    n = 0
    for name in sorted(os.listdir(src_dir)):
        if not name.endswith((".eam.alloy", ".eam.alloy.txt", ".eam.fs.txt")):
            continue
        src, dst = os.path.join(src_dir, name), os.path.join(dst_dir, name)
        if _stale(dst, [src]) or os.path.getsize(dst) != os.path.getsize(src):
            shutil.copyfile(src, dst)
        n += 1
    return n


def build_all(verbose_ptxas=False):
    lib = build_cuda_library(verbose_ptxas=verbose_ptxas)
    mod = build_python_module() if os.path.exists(os.path.join(CSRC, "md_driver_module.cpp")) else None
    stage_potentials()
    return lib, mod


if __name__ == "__main__":
    build_all(verbose_ptxas="--ptxas" in sys.argv)
