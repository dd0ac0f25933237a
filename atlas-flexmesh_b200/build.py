"""Build libflexmesh_b200.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed).

    python atlas-flexmesh_b200/build.py

The library lands next to the Python package (flexmesh_b200/) so that it
travels with the source tree and is the one the package loads.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "flexmesh_b200", "libflexmesh_b200.so")
SOURCES = ["fm_api.cu", "fm_kernels.cu", "fm_nodes.cu", "fm_trsv.cu", "fm_trsv_push.cu", "fm_adjoint.cu", "fm_states.cu", "fm_meshsetup.cu",
           "fm_setup.cpp", "fm_checkpoint.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    # the system g++ (the environment's CXX may point at a wrapper without libgomp)
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(ROOT, "include", "fm_api.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "-ccbin", host_cxx(),
           "-Xcompiler", "-fPIC,-O3", "-shared", "-I", os.path.join(ROOT, "include"),
           "-I", CSRC, "-o", OUT + ".tmp"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
