"""Build lib/libdiva_b200.so from csrc/*.cu with nvcc for sm_100a.

Run ``python imau-ice_b200/build.py`` (or call ``build()``).  The library is
built in-tree so it travels with the repository; it is rebuilt only when a
source or header is newer than it.  geometry.cu is compiled with
``--fmad=false`` so the masks and staggered geometry round exactly like the
reference; the rest keeps fused multiply-adds.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(OUT_DIR, "libdiva_b200.so")
OBJ_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
          "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]
SOURCES = {"api.cu": [], "geometry.cu": ["--fmad=false"], "picard.cu": [], "solver.cu": [], "noalloc.cu": [],
           "thickness.cu": ["--fmad=false"], "thermo.cu": ["--fmad=false"], "cnn.cu": []}


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return files


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _deps())


def build(force=False, verbose=False, extra_flags=()):
    if not force and not needs_build():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src, flags in SOURCES.items():
        obj = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        cmd = [nvcc, "-c", os.path.join(CSRC, src), "-o", obj] + ARCH + COMMON + flags + list(extra_flags)
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    # export only the C ABI (diva_*); everything else is local to the library
    vs = os.path.join(OBJ_DIR, "exports.map")
    with open(vs, "w") as f:
        f.write("{ global: diva_*; local: *; };\n")
    cmd = [nvcc, "-shared", "-o", LIB] + objs + ARCH + ["-Xlinker", f"--version-script={vs}"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
