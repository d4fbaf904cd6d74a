"""Builds the sm_100a shared libraries in-tree with nvcc.

Two variants of the same sources:

- libgfx_fluid.so (exact): --fmad=false keeps every multiply and add
  separately rounded, as the reference's Fortran arithmetic is written, and
  every division is correctly rounded, so that the step reproduces the
  reference's rounding wherever its arithmetic allows.
- libgfx_fluid_fast.so (fast): --fmad=true and GFX_FAST_MATH=1 (products
  with rounded reciprocals for the divisions by known values, fused
  multiply-adds, the entropy per baryon from two logarithms).  Its results
  stay within the 1e-12 per-step bar of the reference's step, not bit for bit.

Both are compiled at once when either is stale, beside libgfx_probe.so
(csrc/fp64_probe.cu), the FP64 rate probe of the bench's FP64 roofline."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
SOURCES = ["gfx_fluid.cu"]
HEADERS = ["fluid_physics.cuh", "stage_kernel.cuh", "aux_kernels.cuh", "adjoint_physics.cuh",
           "adjoint_kernels.cuh"]

VARIANTS = {
    "exact": ("libgfx_fluid.so", ["--fmad=false"], "build.log"),
    "fast": ("libgfx_fluid_fast.so", ["--fmad=true", "-DGFX_FAST_MATH=1"], "build_fast.log"),
}
LIB = os.path.join(HERE, VARIANTS["exact"][0])

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--shared", "-Xptxas", "-v",
]


def lib_path(variant="exact"):
    return os.path.join(HERE, VARIANTS[variant][0])


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(path):
    if not os.path.exists(path):
        return True
    t = os.path.getmtime(path)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "gfx_fluid.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


PROBE = ("libgfx_probe.so", "fp64_probe.cu", "build_probe.log")


def build(force=False, verbose=False, variants=("exact", "fast")):
    """Compiles the variants whose library is older than a source, and the
    FP64 probe; returns the path of the exact library."""
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    jobs = []
    probe_out = os.path.join(HERE, PROBE[0])
    probe_src = os.path.join(CSRC, PROBE[1])
    if force or not os.path.exists(probe_out) or \
            os.path.getmtime(probe_src) > os.path.getmtime(probe_out):
        cmd = [_nvcc(), *NVCC_FLAGS, "-o", probe_out + ".tmp", probe_src]
        p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                             env=env)
        jobs.append(("probe", probe_out, os.path.join(HERE, PROBE[2]), cmd, p))
    for v in variants:
        name, flags, log = VARIANTS[v]
        out = os.path.join(HERE, name)
        if not force and not _stale(out):
            continue
        cmd = [_nvcc(), *NVCC_FLAGS, *flags, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
               "-o", out + ".tmp"] + [os.path.join(CSRC, f) for f in SOURCES]
        p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                             env=env)
        jobs.append((v, out, os.path.join(HERE, log), cmd, p))
    failed = []
    for v, out, log, cmd, p in jobs:
        so, se = p.communicate()
        with open(log, "w") as f:
            f.write(" ".join(cmd) + "\n" + so + se)
        if p.returncode != 0:
            sys.stderr.write(se[-8000:])
            failed.append(log)
            continue
        os.replace(out + ".tmp", out)
        if verbose:
            sys.stdout.write("[%s]\n%s" % (v, se))
    if failed:
        raise RuntimeError("nvcc failed; see %s" % ", ".join(failed))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
