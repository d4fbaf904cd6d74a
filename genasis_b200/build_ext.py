"""Builds the sm_100a shared library libgfx_fluid.so in-tree with nvcc.

--fmad=false keeps every multiply and add separately rounded, as the
reference's Fortran arithmetic is written (the parity contract is per-step
agreement with the reference step to round-off)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgfx_fluid.so")
SOURCES = ["gfx_fluid.cu"]
HEADERS = ["fluid_physics.cuh", "stage_kernel.cuh", "aux_kernels.cuh", "adjoint_physics.cuh",
           "adjoint_kernels.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--shared", "-Xptxas", "-v",
]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "gfx_fluid.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile the library if a source is newer than it; returns the path."""
    if not force and not _stale():
        return LIB
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           "-o", LIB + ".tmp"] + [os.path.join(CSRC, f) for f in SOURCES]
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    log = os.path.join(HERE, "build.log")
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stderr[-8000:])
        raise RuntimeError("nvcc failed; see %s" % log)
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        sys.stdout.write(r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
