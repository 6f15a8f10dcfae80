"""Build the in-tree shared libraries of gcdt_b200.

  libgcdt_b200.so  CUDA kernels + C ABI (nvcc, sm_100a only)
  libgcdt_gen.so   seeded workload generators (host C++)

The libraries are written next to this file so that they travel with the
source tree; nothing is installed into site-packages.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
    "-I" + os.path.join(ROOT, "include"),
]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build gcdt_b200")
    return cand


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]))
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(*names):
    files = [os.path.join(CSRC, n) for n in os.listdir(CSRC)
             if n.endswith((".cuh", ".h", ".hpp"))]
    files += [os.path.join(CSRC, n) for n in names]
    files += [os.path.join(ROOT, "include", n) for n in os.listdir(os.path.join(ROOT, "include"))]
    return files


# Compile-time variants of the solver bodies, built next to the default
# library for measurement (GCDT_B200_LIB selects one at import):
#   name -> extra nvcc flags.  None at present.
VARIANTS = {}


def build(force=False, verbose=False, ptxas_verbose=False, variant=None):
    out = os.path.join(HERE, "libgcdt_b200.so" if not variant else "libgcdt_b200_%s.so" % variant)
    srcs = ["gcdt.cu", "batch.cu", "server.cu", "surface.cu", "reorder.cu", "regions.cu", "io.cpp"]
    if force or _stale(out, _deps(*srcs)):
        flags = list(NVCC_FLAGS) + (VARIANTS[variant] if variant else [])
        if ptxas_verbose:
            flags += ["-Xptxas", "-v"]
        r = _run([_nvcc()] + flags + ["-o", out] + [os.path.join(CSRC, s) for s in srcs], verbose)
        if ptxas_verbose:
            sys.stdout.write(r.stderr)
    gen = os.path.join(HERE, "libgcdt_gen.so")
    if force or _stale(gen, [os.path.join(CSRC, "gen.cpp")]):
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", gen,
              os.path.join(CSRC, "gen.cpp")], verbose)
    return out


if __name__ == "__main__":
    var = sys.argv[sys.argv.index("--variant") + 1] if "--variant" in sys.argv else None
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv, variant=var)
