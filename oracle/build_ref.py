"""Build recipe of oracle/_ref: the reference's own tricubic kernels (TEST
INFRASTRUCTURE; only tests/ load what it builds).

The reference as a whole needs MPI, PETSc 3.9.1, AccFFT and FFTW and is not
buildable here.  Its interpolation source, src/interp3.cpp, needs none of
them at run time: it includes mpi.h, petsc.h and accfft.h for type names of
its distributed drivers.  With the declaration-only headers of
oracle/ref_stubs/ and the single-process shim oracle/ref_shim.cpp it compiles
as it lies in the reference tree (nothing is copied) into

* oracle/_ref/libinterp3_ref_f64.so -- double build (the reference's default,
  USESINGLE=no): optimized_interp3_ghost_xyz_p;
* oracle/_ref/libinterp3_ref_f32.so -- single build (PETSC_USE_REAL_SINGLE):
  the same kernel in float (with GCC the header undefines FAST_INTERPV, the
  switch to the Intel-compiler AVX kernels, include/interp3.hpp:37-39).

The reference builds with -O3 -fopenmp -march=native (config/setup.mk:12-22);
here -O3 -fopenmp -mavx2 -mfma (a portable x86-64 instruction set).  The
built libraries travel with the repository's other built files; the
reference tree itself is read only where it is present (the host that builds
the libraries).

  python oracle/build_ref.py
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("CLAIRE_REFERENCE_TREE", "/root/reference")
OUT = os.path.join(HERE, "_ref")
FLAGS = ["-std=c++11", "-O3", "-fopenmp", "-mavx2", "-mfma", "-fPIC", "-w",
         # src/interp3.cpp defines _mm256_set_m128 as a macro before it includes
         # immintrin.h; GCC's header declares a function of that name
         "-include", "immintrin.h"]
VARIANTS = {"f64": [], "f32": ["-DPETSC_USE_REAL_SINGLE"]}


def available() -> bool:
    return os.path.isfile(os.path.join(REFERENCE, "src", "interp3.cpp"))


def lib_path(variant: str) -> str:
    return os.path.join(OUT, f"libinterp3_ref_{variant}.so")


def build(force: bool = False) -> list:
    """Compile both variants; returns the built paths ([] without the reference tree)."""
    if not available():
        return []
    os.makedirs(OUT, exist_ok=True)
    inc = ["-I", os.path.join(HERE, "ref_stubs"), "-I", os.path.join(REFERENCE, "include"),
           "-I", os.path.join(REFERENCE, "deps", "3rdparty")]
    src = os.path.join(REFERENCE, "src", "interp3.cpp")
    shim = os.path.join(HERE, "ref_shim.cpp")
    built = []
    for variant, defs in VARIANTS.items():
        lib = lib_path(variant)
        inputs = [src, shim] + [os.path.join(HERE, "ref_stubs", h) for h in os.listdir(os.path.join(HERE, "ref_stubs"))]
        if not force and os.path.exists(lib) and all(os.path.getmtime(p) <= os.path.getmtime(lib) for p in inputs):
            built.append(lib)
            continue
        objs = []
        for name, path in (("interp3", src), ("shim", shim)):
            obj = os.path.join(OUT, f"{name}_{variant}.o")
            cmd = ["g++", *FLAGS, *defs, *inc, "-c", path, "-o", obj]
            r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
            if r.returncode != 0:
                raise RuntimeError(f"{' '.join(cmd)}\n{r.stdout.decode()}")
            objs.append(obj)
        tmp = lib + ".tmp"
        r = subprocess.run(["g++", "-shared", "-fopenmp", *objs, "-o", tmp], stdout=subprocess.PIPE,
                           stderr=subprocess.STDOUT)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout.decode())
        os.replace(tmp, lib)
        for o in objs:
            os.remove(o)
        built.append(lib)
    return built


if __name__ == "__main__":
    paths = build(force="--force" in sys.argv)
    print("\n".join(paths) if paths else f"reference tree not found at {REFERENCE}: nothing built")
