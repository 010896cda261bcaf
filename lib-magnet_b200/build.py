"""Build recipe of the B200 layout pass: compiles the CUDA sources for sm_100a into the C-ABI library
``libmagnet_b200.so`` and the pybind11 module ``magnet_b200/_native`` (the reference-compatible Python
surface) linked against it. Both are written in-tree so that they travel with the repository.

    python lib-magnet_b200/build.py [--force]
"""
import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmagnet_b200.so")
NATIVE_SRC = os.path.join(HERE, "pybind", "native.cpp")
NATIVE = os.path.join(HERE, "magnet_b200", "_native" + sysconfig.get_config_var("EXT_SUFFIX"))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(NVCC))

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "--expt-relaxed-constexpr", "-Xptxas", "-v"]


# per-file flags: owner mode and the graph passes round every product and sum on their own, as the reference's
# plain x86-64 build and numpy do
FILE_FLAGS = {"owner.cu": ["-fmad=false"], "graph.cu": ["-fmad=false"], "spectral.cu": ["-fmad=false"]}


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, log=None):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        with open(log, "w") as f:
            f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r


def build_library(force=False):
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = sources + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    if not force and not _newer(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [NVCC] + NVCC_FLAGS + FILE_FLAGS.get(os.path.basename(src), []) + \
            ["-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    with open(os.path.join(objdir, "ptxas.log"), "w") as logf:
        for cmd, p in procs:
            out, _ = p.communicate()
            logf.write(" ".join(cmd) + "\n" + out + "\n")
            if p.returncode != 0:
                sys.stderr.write(out)
                failed = True
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = LIB + ".tmp"
    _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-lcudart"])
    os.replace(tmp, LIB)
    return LIB


def build_native(force=False):
    deps = [NATIVE_SRC, LIB, os.path.join(ROOT, "include", "magnet_b200.h")]
    if not force and not _newer(NATIVE, deps):
        return NATIVE
    import pybind11
    inc = [sysconfig.get_paths()["include"], pybind11.get_include()]
    tmp = NATIVE + ".tmp"
    cmd = ["g++", "-O2", "-DNDEBUG", "-shared", "-fPIC", "-std=c++17", NATIVE_SRC, "-o", tmp,
           "-I", os.path.join(ROOT, "include")] + [a for i in inc for a in ("-I", i)] + \
          ["-L", HERE, "-lmagnet_b200", "-Wl,-rpath,$ORIGIN/.."]
    _run(cmd)
    os.replace(tmp, NATIVE)
    return NATIVE


def build(force=False):
    build_library(force)
    build_native(force)
    return LIB, NATIVE


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
