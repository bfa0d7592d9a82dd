"""ctypes binding and build recipe of the C++/OpenMP restatement (cpu_ref.cpp).

THIS IS TEST INFRASTRUCTURE AND THE TIMED CPU BASELINE.  Only ``tests/``,
``__graft_entry__`` and ``bench.py``'s CPU legs use it; the product library
never does.

``build()`` compiles ``oracle/cpu_ref.cpp`` with g++ (C++17, OpenMP, AVX2/FMA
code generation) into ``oracle/libcpuref.so``.  ``CpuRef`` wraps one problem:
FP64 (the reference's default build: the full-size parity oracle) or FP32
(its single-precision build: the timed CPU baseline).  Arrays cross the ABI as
float64 NumPy arrays in the layouts of oracle/claire_ref.py (scalar fields
(N1, N2, N3), vector fields (3, N1, N2, N3), x3 fastest).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_ref.cpp")
LIB = os.path.join(HERE, "libcpuref.so")
CXXFLAGS = ["-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared"]

NORMS = {"l2": 0, "h1": 1, "h1s": 2, "h2": 3, "h2s": 4, "h3": 5, "h3s": 6}
FSEQ = {"slfs": 0, "qdfs": 1, "none": 2}
STATS = ("J", "D", "R", "J0", "D0", "gnorm", "g0", "iters", "pcg_iters", "reason", "rel_mismatch", "seconds",
         "obj_evals", "grad_evals", "hess_matvecs", "pc_matvecs", "pde_solves", "gathers", "ffts", "krylov_g0")
REASONS = {0: "running", 1: "gttol", 2: "gatol", 3: "maxit", 4: "steptol", 5: "lsfail", -1: "nan"}


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    tmp = LIB + ".tmp"
    r = subprocess.run(["g++", *CXXFLAGS, SRC, "-o", tmp], stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("g++ failed on cpu_ref.cpp:\n" + r.stdout.decode())
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        DP = ctypes.POINTER(ctypes.c_double)
        sig = {
            "cref_create": (P, [I, I, I, I, I, D, D, I, I]),
            "cref_destroy": (None, [P]),
            "cref_max_threads": (I, []),
            "cref_set_threads": (I, [I]),
            "cref_set_gn": (I, [P, I, D, D, I, I, D]),
            "cref_set_images": (I, [P, DP, DP]),
            "cref_objective": (I, [P, DP, DP]),
            "cref_gradient": (I, [P, DP, DP]),
            "cref_hessian_matvec": (I, [P, DP, DP, DP]),
            "cref_hessian_matvec_current": (I, [P, DP, DP]),
            "cref_precond": (I, [P, DP, DP]),
            "cref_reg_apply": (I, [P, I, DP, DP]),
            "cref_reg_functional": (I, [P, DP, DP]),
            "cref_grad": (I, [P, DP, DP]),
            "cref_div": (I, [P, DP, DP]),
            "cref_trajectory": (I, [P, DP, I, DP]),
            "cref_interp": (I, [P, DP, DP, DP]),
            "cref_forward": (I, [P, DP, DP, DP]),
            "cref_begin": (I, [P]),
            "cref_step": (I, [P]),
            "cref_finish": (I, [P]),
            "cref_run": (I, [P]),
            "cref_get_velocity": (I, [P, DP]),
            "cref_get_final_state": (I, [P, DP]),
            "cref_stats": (I, [P, DP]),
            "cref_reset_counters": (I, [P]),
            "cref_last_adjoint": (I, [P, DP, DP]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _in(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class CpuRef:
    """One registration problem of the C++ restatement."""

    def __init__(self, shape, nt: int, norm: str = "h1s", beta0: float = 1e-2, beta1: float = 1e-4,
                 fp64: bool = True, threads: int = 0):
        self.shape = tuple(int(s) for s in shape)
        self.n = int(np.prod(self.shape))
        self.L = lib()
        self.h = self.L.cref_create(*self.shape, int(nt), NORMS[norm], float(beta0), float(beta1),
                                    1 if fp64 else 0, int(threads))
        if not self.h:
            raise ValueError(f"cpu_ref: unsupported grid {self.shape}")

    def close(self):
        if getattr(self, "h", None):
            self.L.cref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _chk(self, rc, what):
        if rc < 0:
            raise RuntimeError(f"cpu_ref {what}: {rc}")
        return rc

    def set_gn(self, maxit=50, gttol=5e-2, gatol=1e-6, krylov_maxit=50, fseq="slfs", krylov_rtol=1e-2):
        self._chk(self.L.cref_set_gn(self.h, int(maxit), float(gttol), float(gatol), int(krylov_maxit),
                                     FSEQ[fseq], float(krylov_rtol)), "set_gn")

    def set_images(self, mR, mT):
        self._mR, self._mT = _in(mR), _in(mT)
        self._chk(self.L.cref_set_images(self.h, _ptr(self._mR), _ptr(self._mT)), "set_images")

    def objective(self, v):
        out = np.zeros(3)
        self._chk(self.L.cref_objective(self.h, _ptr(_in(v)), _ptr(out)), "objective")
        return float(out[0]), float(out[1]), float(out[2])

    def _vec_op(self, fn, args, out_shape):
        out = np.zeros(out_shape)
        self._chk(fn(self.h, *args, _ptr(out)), fn.__name__)
        return out

    def gradient(self, v):
        return self._vec_op(self.L.cref_gradient, [_ptr(_in(v))], (3,) + self.shape)

    def hessian_matvec(self, v, vt):
        return self._vec_op(self.L.cref_hessian_matvec, [_ptr(_in(v)), _ptr(_in(vt))], (3,) + self.shape)

    def hessian_matvec_current(self, vt):
        """Hessian matvec at the velocity of the last gradient() call (its
        state and adjoint reused)."""
        return self._vec_op(self.L.cref_hessian_matvec_current, [_ptr(_in(vt))], (3,) + self.shape)

    def precond(self, x):
        return self._vec_op(self.L.cref_precond, [_ptr(_in(x))], (3,) + self.shape)

    def reg_apply(self, x, kind=0):
        return self._vec_op(self.L.cref_reg_apply, [int(kind), _ptr(_in(x))], (3,) + self.shape)

    def reg_functional(self, v):
        out = np.zeros(1)
        self._chk(self.L.cref_reg_functional(self.h, _ptr(_in(v)), _ptr(out)), "reg_functional")
        return float(out[0])

    def grad(self, f):
        return self._vec_op(self.L.cref_grad, [_ptr(_in(f))], (3,) + self.shape)

    def div(self, v):
        return self._vec_op(self.L.cref_div, [_ptr(_in(v))], self.shape)

    def trajectory(self, v, flag="state"):
        return self._vec_op(self.L.cref_trajectory, [_ptr(_in(v)), 1 if flag == "state" else -1],
                            (3,) + self.shape)

    def interp(self, f, disp):
        return self._vec_op(self.L.cref_interp, [_ptr(_in(f)), _ptr(_in(disp))], self.shape)

    def forward(self, v, m0):
        return self._vec_op(self.L.cref_forward, [_ptr(_in(v)), _ptr(_in(m0))], self.shape)

    def begin(self):
        self._chk(self.L.cref_begin(self.h), "begin")

    def step(self) -> bool:
        return bool(self._chk(self.L.cref_step(self.h), "step"))

    def finish(self):
        self._chk(self.L.cref_finish(self.h), "finish")

    def run(self):
        self._chk(self.L.cref_run(self.h), "run")
        return self.stats()

    def velocity(self):
        out = np.zeros((3,) + self.shape)
        self._chk(self.L.cref_get_velocity(self.h, _ptr(out)), "get_velocity")
        return out

    def final_state(self):
        out = np.zeros(self.shape)
        self._chk(self.L.cref_get_final_state(self.h, _ptr(out)), "get_final_state")
        return out

    def stats(self) -> dict:
        out = np.zeros(len(STATS))
        self._chk(self.L.cref_stats(self.h, _ptr(out)), "stats")
        d = {k: float(x) for k, x in zip(STATS, out)}
        for k in ("iters", "pcg_iters", "reason", "obj_evals", "grad_evals", "hess_matvecs", "pc_matvecs",
                  "pde_solves", "gathers", "ffts"):
            d[k] = int(d[k])
        d["reason_name"] = REASONS.get(d["reason"], "?")
        return d

    def last_adjoint(self):
        """(lambda at t = 0, body force hd b) of the last gradient or Hessian matvec."""
        lam = np.zeros(self.shape)
        bf = np.zeros((3,) + self.shape)
        self._chk(self.L.cref_last_adjoint(self.h, _ptr(lam), _ptr(bf)), "last_adjoint")
        return lam, bf

    def reset_counters(self):
        self._chk(self.L.cref_reset_counters(self.h), "reset_counters")


if __name__ == "__main__":
    print(build(force=True))
