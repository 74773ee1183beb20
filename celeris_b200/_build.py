"""Build recipe for the in-tree native artefacts.

  libceleris_b200.so   CUDA kernels + C ABI (nvcc, sm_100a only)
  _celeris*.so         C++ host mirror of the reference's celeris:: API with its
                       pybind11 bindings (links libceleris_b200.so, rpath $ORIGIN)
  oracle/              the checker libraries (make -C oracle)

Artefacts are written next to their sources so they travel with a snapshot of
the repository; object files go to celeris_b200/_build/ (git-ignored).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libceleris_b200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                     "-I" + os.path.join(ROOT, "include")]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(verbose=False, ptxas_verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) + [
        os.path.join(ROOT, "include", "celeris_b200.h")]
    objs = []
    for cu in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        o = os.path.join(OBJ, os.path.basename(cu)[:-3] + ".o")
        objs.append(o)
        if _stale(o, [cu] + headers):
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            r = _run([NVCC] + NVCC_FLAGS + extra + ["-c", cu, "-o", o], verbose)
            if ptxas_verbose:
                sys.stdout.write(r.stderr)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs, verbose)
    return LIB


def ext_name():
    return "_celeris" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so")


def build_host(verbose=False):
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    if not srcs:
        return None
    import pybind11

    out = os.path.join(PKG, ext_name())
    hdrs = glob.glob(os.path.join(HOST, "*.hpp")) + [os.path.join(ROOT, "include", "celeris_b200.h")]
    if _stale(out, srcs + hdrs + [LIB]):
        inc = sysconfig.get_paths()["include"]
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden",
               "-I" + inc, "-I" + pybind11.get_include(), "-I" + os.path.join(ROOT, "include"), "-I" + HOST]
        cmd += srcs + ["-L" + PKG, "-lceleris_b200", "-Wl,-rpath,$ORIGIN", "-o", out, "-lpthread"]
        _run(cmd, verbose)
    return out


# The reference checkout the oracle recipe compiles its checker libraries from
# (CELERIS_REFERENCE overrides; the GPU hosts have none and use the prebuilt files).
REFERENCE = os.environ.get("CELERIS_REFERENCE", "/root/reference")


def build_oracle(verbose=False):
    cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle")]
    if os.path.isdir(os.path.join(REFERENCE, "src", "celeris")):
        cmd.append("REF=" + REFERENCE)
    _run(cmd, verbose)


def build_all(verbose=False):
    build_cuda(verbose)
    build_host(verbose)
    build_oracle(verbose)


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv)
    if "--ptxas" in sys.argv:
        for o in glob.glob(os.path.join(OBJ, "*.o")):
            os.remove(o)
        build_cuda(True, ptxas_verbose=True)
