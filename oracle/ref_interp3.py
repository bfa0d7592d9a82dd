"""ctypes binding of the reference's own tricubic kernels built by
oracle/build_ref.py (TEST INFRASTRUCTURE: only tests/ use it).

``interp3(f, disp, precision)`` evaluates the periodic field f at x + disp
(disp in grid units, shape (3, N1, N2, N3)) with the reference's
optimized_interp3_ghost_xyz_p (src/interp3.cpp:2492-2719) in the reference's
double or single build: the points are handed over as the reference's
trajectory leaves them, coordinates normalised by the grid length and
wrapped into (-h, 1) (src/Interp3_Plan.cpp:344-361).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from oracle import build_ref


def available(precision: str = "f64") -> bool:
    return os.path.exists(build_ref.lib_path(precision))


_libs = {}


def _lib(precision):
    if precision not in _libs:
        L = ctypes.CDLL(build_ref.lib_path(precision))
        L.ref_interp3.restype = ctypes.c_int
        L.ref_real_bytes.restype = ctypes.c_int
        _libs[precision] = L
    return _libs[precision]


def normalised_points(disp: np.ndarray, dtype) -> np.ndarray:
    """Query points of x + disp as (npts, 3) normalised coordinates in (-h, 1)."""
    shape = disp.shape[1:]
    idx = np.stack(np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij"))
    q = idx + np.asarray(disp, np.float64)
    Q = np.stack([q[d] / shape[d] for d in range(3)])
    for d in range(3):
        # src/Interp3_Plan.cpp:344-361: add 1 while Q <= -h, subtract 1 while Q >= 1
        h = 1.0 / shape[d]
        keep = (Q[d] > -h) & (Q[d] < 1.0)
        w = Q[d] - np.floor(Q[d])
        w = np.where(w >= 1.0, w - 1.0, w)
        Q[d] = np.where(keep, Q[d], w)
    return np.ascontiguousarray(np.moveaxis(Q, 0, -1).reshape(-1, 3).astype(dtype))


def interp3(f: np.ndarray, disp: np.ndarray, precision: str = "f64") -> np.ndarray:
    dtype = np.float64 if precision == "f64" else np.float32
    L = _lib(precision)
    assert L.ref_real_bytes() == np.dtype(dtype).itemsize
    shape = f.shape
    npts = int(np.prod(shape))
    ff = np.ascontiguousarray(f, dtype=dtype)
    Q = normalised_points(disp, dtype)
    out = np.zeros(npts, dtype=dtype)
    P = ctypes.POINTER(ctypes.c_double if dtype == np.float64 else ctypes.c_float)
    rc = L.ref_interp3(ff.ctypes.data_as(P), (ctypes.c_int * 3)(*shape), npts, Q.ctypes.data_as(P),
                       out.ctypes.data_as(P))
    if rc != 0:
        raise ValueError(f"ref_interp3: {rc} (point count must be a multiple of 16)")
    return out.reshape(shape)
