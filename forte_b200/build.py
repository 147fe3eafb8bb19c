"""Builds the engine's shared library (libfcib200.so) in-tree for sm_100a with nvcc."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfcib200.so")
# profiling build: the same sources with the batched solver's phase clocks (-DFCIB_BATCH_PHASES)
LIB_PHASES = os.path.join(HERE, "libfcib200_phases.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cpp", ".h", ".cuh"))] + [os.path.join(HERE, "..", "include", "fcib.h")]


def needs_build(lib=LIB):
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force=False, verbose=False, phases=False):
    """Builds libfcib200.so, or with phases=True the profiling build libfcib200_phases.so."""
    lib = LIB_PHASES if phases else LIB
    if not force and not needs_build(lib):
        return lib
    objdir = os.path.join(HERE, "_build_phases" if phases else "_build")
    os.makedirs(objdir, exist_ok=True)
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo"] + (["-DFCIB_BATCH_PHASES"] if phases else [])
    obj_cu = os.path.join(objdir, "fcib_all.o")
    obj_cpp = os.path.join(objdir, "guess.o")
    cmds = [
        [NVCC, *ARCH, *common, "-c", os.path.join(CSRC, "fcib_all.cu"), "-o", obj_cu],
        [NVCC, *common, "-x", "cu", "-c", os.path.join(CSRC, "guess.cpp"), "-o", obj_cpp] + ARCH,
        [NVCC, *ARCH, "-shared", "-cudart", "static", obj_cu, obj_cpp, "-o", lib + ".tmp"],
    ]
    for c in cmds:
        if verbose:
            print(" ".join(c))
        r = subprocess.run(c, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed: " + " ".join(c))
        elif verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr)
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
