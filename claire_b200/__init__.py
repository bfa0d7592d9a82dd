"""claire_b200: B200-native CLAIRE Gauss-Newton-Krylov registration path.

The compute path is ``libclaire_b200.so`` (CUDA for sm_100a plus the C++ GN
driver); this module is a thin ctypes mirror of its C ABI
(``include/claire_b200.h``) that keeps the reference's names:

* ``RegOpt``            -- reg::RegOpt (include/RegOpt.hpp:475-635)
* ``CLAIREInterface``   -- reg::CLAIREInterface (include/CLAIREInterface.hpp:42-90)
* ``SemiLagrangian``    -- ComputeTrajectory / Interpolate (include/SemiLagrangian.hpp:43-58)
* ``Regularization``    -- EvaluateFunctional / EvaluateGradient / HessianMatVec /
                           ApplyInverse (include/Regularization.hpp:46-50)
* ``DistanceMeasureSL2``-- EvaluateFunctional (include/DistanceMeasure.hpp:44-50)
* spectral helpers standing in for AccFFT's accfft_grad_t / accfft_divergence_t.

Operator functions take torch CUDA tensors (float32, contiguous) and run on
the current torch stream.  There is no CPU fallback: importing without the
built library raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

__all__ = [
    "lib", "RegOpt", "CLAIREInterface", "SemiLagrangian", "Regularization", "DistanceMeasureSL2",
    "Preconditioner", "fft_grad", "fft_div", "leray", "smooth", "kernel_launches", "ClaireError",
    "NORMS", "MODELS", "Server",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
# CLAIRE_B200_LIB selects another build of the library (A/B comparisons).
LIB_PATH = os.environ.get("CLAIRE_B200_LIB") or os.path.join(_HERE, "libclaire_b200.so")

NORMS = {"l2": 0, "h1": 1, "h1s": 2, "h2": 3, "h2s": 4, "h3": 5, "h3s": 6}
MODELS = {"compressible": 0, "stokes": 1, "relaxedstokes": 2}
REG_KIND = {"gradient": 0, "inverse": 1, "sqrtinverse": 2}
ERRORS = {-1: "invalid argument", -2: "allocation failed", -3: "CUDA error", -4: "numerical error (NaN)",
          -5: "call out of order", -6: "unsupported grid size",
          -7: "too large (fixed workspace, free device memory or HBM budget)", -8: "request cancelled"}
ERR_TOO_LARGE, ERR_CANCELLED = -7, -8


class ClaireError(RuntimeError):
    """Raised for a negative status code from the C ABI."""

    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        msg = f"{where}: {ERRORS.get(code, 'error')} ({code})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


class Opts(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int * 3), ("nt", ctypes.c_int), ("regnorm", ctypes.c_int), ("model", ctypes.c_int),
        ("beta", ctypes.c_double * 3), ("maxit", ctypes.c_int), ("opttol", ctypes.c_double),
        ("gatol", ctypes.c_double), ("krylovmaxit", ctypes.c_int), ("krylovtol", ctypes.c_double * 3),
        ("krylovfseq", ctypes.c_int), ("precond", ctypes.c_int), ("iporder", ctypes.c_int),
        ("verbosity", ctypes.c_int), ("bf16_images", ctypes.c_int), ("betacont", ctypes.c_double),
        ("presolvetol", ctypes.c_double), ("autotune", ctypes.c_int), ("distance", ctypes.c_int),
        ("scalecont", ctypes.c_int), ("gridcont", ctypes.c_int), ("train", ctypes.c_int),
        ("jbound", ctypes.c_double), ("betainit", ctypes.c_double), ("monitordefgrad", ctypes.c_int),
        ("pcgridscale", ctypes.c_double), ("pctolscale", ctypes.c_double), ("pcsolvermaxit", ctypes.c_int),
    ]


class ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_longlong), ("slots_per_pool", ctypes.c_int),
                ("idle_ms", ctypes.c_int), ("device", ctypes.c_int), ("batch_window_us", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [
        ("gn_iterations", ctypes.c_int), ("pcg_iterations", ctypes.c_int), ("obj_evals", ctypes.c_int),
        ("grad_evals", ctypes.c_int), ("hess_matvecs", ctypes.c_int), ("pc_matvecs", ctypes.c_int),
        ("pde_solves", ctypes.c_int), ("converged_reason", ctypes.c_int), ("J", ctypes.c_double),
        ("J0", ctypes.c_double), ("D", ctypes.c_double), ("D0", ctypes.c_double), ("R", ctypes.c_double),
        ("gnorm", ctypes.c_double), ("gnorm0", ctypes.c_double), ("rel_mismatch", ctypes.c_double),
        ("seconds", ctypes.c_double), ("beta", ctypes.c_double), ("solution_status", ctypes.c_int),
        ("det_min", ctypes.c_double), ("det_mean", ctypes.c_double), ("det_max", ctypes.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"claire_b200: {LIB_PATH} is not built; run `python -m claire_b200.build` "
            "(there is no CPU fallback)")
    return ctypes.CDLL(LIB_PATH)


lib = _load()

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_IA = ctypes.POINTER(ctypes.c_int)
_DA = ctypes.POINTER(ctypes.c_double)
_signatures = {
    "claire_b200_default_opts": (_I, [ctypes.POINTER(Opts)]),
    "claire_b200_parse_args": (_I, [ctypes.POINTER(Opts), _I, ctypes.POINTER(ctypes.c_char_p)]),
    "claire_b200_create": (_I, [ctypes.POINTER(Opts), _I, ctypes.POINTER(_P)]),
    "claire_b200_destroy": (_I, [_P]),
    "claire_b200_last_error": (ctypes.c_char_p, [_P]),
    "claire_b200_footprint_bytes": (ctypes.c_longlong, [_P]),
    "claire_b200_estimate_bytes": (ctypes.c_longlong, [ctypes.POINTER(Opts), _I]),
    "claire_b200_set_problem_opts": (_I, [_P, _I, ctypes.POINTER(Opts)]),
    "claire_b200_set_images": (_I, [_P, _I, _P, _P, _I]),
    "claire_b200_set_velocity": (_I, [_P, _I, _P, _I]),
    "claire_b200_set_mask": (_I, [_P, _I, _P, _I]),
    "claire_b200_get_velocity": (_I, [_P, _I, _P, _I]),
    "claire_b200_run": (_I, [_P]),
    "claire_b200_run_masked": (_I, [_P, _IA]),
    "claire_b200_get_final_state": (_I, [_P, _I, _P, _I]),
    "claire_b200_forward": (_I, [_P, _I, _P, _P, _I]),
    "claire_b200_get_stats": (_I, [_P, _I, ctypes.POINTER(Stats)]),
    "claire_b200_objective": (_I, [_P, _I, _P, _DA, _DA, _DA]),
    "claire_b200_gradient": (_I, [_P, _I, _P, _P]),
    "claire_b200_hessian_matvec": (_I, [_P, _I, _P, _P, _P]),
    "claire_b200_precond": (_I, [_P, _I, _P, _P]),
    "claire_b200_get_adjoint": (_I, [_P, _I, _P, _P]),
    "claire_b200_synchronize": (_I, [_P]),
    "claire_b200_set_stream": (_I, [_P, _P]),
    "claire_b200_trajectory": (_I, [_P, _P, _IA, _I, _I, _P]),
    "claire_b200_interp3": (_I, [_P, _P, _P, _IA, _I, _P]),
    "claire_b200_interp3_bf16": (_I, [_P, _P, _P, _IA, _P]),
    "claire_b200_fft_grad": (_I, [_P, _P, _IA, _P]),
    "claire_b200_autotune": (_I, [_I, _I, _P, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_float)]),
    "claire_b200_fft_variant": (_I, [_I]),
    "claire_b200_grid_change": (_I, [_P, _I, _P, _I, _I, _P]),
    "claire_b200_read_nifti": (_I, [ctypes.c_char_p, _IA, _P, ctypes.c_longlong]),
    "claire_b200_write_nifti": (_I, [ctypes.c_char_p, _IA, _P]),
    "claire_b200_read_bin": (_I, [ctypes.c_char_p, _IA, _P]),
    "claire_b200_deformation_map": (_I, [_P, _I, _I, _P]),
    "claire_b200_displacement_field": (_I, [_P, _I, _P]),
    "claire_b200_def_grad": (_I, [_P, _I, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "claire_b200_det_def_grad_disp": (_I, [_P, _I, _P, ctypes.POINTER(ctypes.c_double)]),
    "claire_b200_write_bin": (_I, [ctypes.c_char_p, _IA, _P]),
    "claire_b200_preprocess": (_I, [_P, _IA, _I, _DA, _P]),
    "claire_b200_set_fft_variant": (_I, [_I, _I]),
    "claire_b200_fft_div": (_I, [_P, _P, _IA, _P]),
    "claire_b200_reg_apply": (_I, [_P, _P, _IA, _I, _DA, _I, _P]),
    "claire_b200_reg_functional": (_I, [_P, _DA, _IA, _I, _DA, _P]),
    "claire_b200_reg_apply_noalloc": (_I, [_P, _P, _IA, _I, _DA, _I, _P]),
    "claire_b200_leray": (_I, [_P, _IA, _I, _DA, _P]),
    "claire_b200_smooth": (_I, [_P, _P, _IA, _DA, _P]),
    "claire_b200_distance": (_I, [_P, _P, _IA, _DA, _P]),
    "claire_b200_kernel_launches": (ctypes.c_longlong, []),
    "claire_b200_stage_timeouts": (_I, [ctypes.POINTER(ctypes.c_longlong)]),
    "claire_b200_stage_wait_selftest": (_I, [ctypes.c_longlong, _P]),
    "claire_b200_profile": (_I, [_P, _I]),
    "claire_b200_det_def_grad": (_I, [_P, _I, _I, _P, ctypes.POINTER(ctypes.c_double)]),
    "claire_b200_server_default_opts": (None, [_P]),
    "claire_b200_server_create": (_I, [_P, ctypes.POINTER(_P)]),
    "claire_b200_server_submit": (_I, [_P, _P, _P, _P, ctypes.POINTER(ctypes.c_longlong)]),
    "claire_b200_server_poll": (_I, [_P, ctypes.c_longlong, ctypes.POINTER(_I)]),
    "claire_b200_server_wait": (_I, [_P, ctypes.c_longlong, _I, ctypes.POINTER(_I)]),
    "claire_b200_server_result": (_I, [_P, ctypes.c_longlong, _P, _P, ctypes.POINTER(ctypes.c_double)]),
    "claire_b200_server_info": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(_I)]),
    "claire_b200_server_cancel": (_I, [_P, ctypes.c_longlong]),
    "claire_b200_server_destroy": (_I, [_P]),
    "claire_b200_profile_read": (_I, [_P, _I, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]),
}

# device timer categories (claire_b200_profile_read)
PROF_ADJOINT_STEP, PROF_INCSTATE_STEP, PROF_STATE_STEP, PROF_PRECOND = 0, 1, 2, 3
PROF_OBJECTIVE, PROF_GRADIENT, PROF_HESSIAN = 4, 5, 6
for _name, (_res, _args) in _signatures.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def _check(code: int, where: str, ctx=None):
    if code != 0:
        detail = ""
        if ctx is not None:
            raw = lib.claire_b200_last_error(ctx)
            detail = raw.decode() if raw else ""
        raise ClaireError(code, where, detail)


def autotune(n: int, nbatch: int = 1):
    """Measure the FFT variants of n-point grids (claire_b200_autotune) and keep
    the fastest for this process; returns (variant, {variant: ms})."""
    v = ctypes.c_int()
    ms = (ctypes.c_float * 4)()
    _check(lib.claire_b200_autotune(int(n), int(nbatch), _stream(), ctypes.byref(v), ms), "autotune")
    cand = fft_variant_candidates(n)
    return v.value, {c: float(ms[i]) for i, c in enumerate(cand)}


def fft_variant_candidates(n: int):
    """FFT variants the autotuner tries for n-point grids (bit 0: radix plan, bit 1: lines per CTA)."""
    if n == 150:
        return [0, 1]
    return [0, 2] if n in (16, 256) else [0, 1, 2, 3]


def read_nifti(path: str):
    """ReadWriteReg::ReadNII: the volume of a NIfTI-1 image (single file, or
    the .hdr / .img pair) as a float32 array of shape (nx[0], nx[1], nx[2]) =
    (nz, ny, nx) of the file."""
    import numpy as np
    nx = (ctypes.c_int * 3)()
    _check(lib.claire_b200_read_nifti(os.fsencode(path), nx, None, 0), "read_nifti")
    out = np.empty((nx[0], nx[1], nx[2]), dtype=np.float32)
    _check(lib.claire_b200_read_nifti(os.fsencode(path), nx, out.ctypes.data_as(ctypes.c_void_p), out.size),
           "read_nifti")
    return out


def write_nifti(path: str, arr) -> None:
    """ReadWriteReg::WriteNII: float32 NIfTI-1 (.nii, .nii.gz compressed, or
    the .hdr / .img pair)."""
    import numpy as np
    a = np.ascontiguousarray(arr, dtype=np.float32)
    if a.ndim != 3:
        raise ValueError("expected a 3D volume")
    _check(lib.claire_b200_write_nifti(os.fsencode(path), _nx(a.shape), a.ctypes.data_as(ctypes.c_void_p)),
           "write_nifti")


def read_bin(path: str, shape):
    """ReadWriteReg::ReadBIN: a PETSc binary vector of prod(shape) values (the
    grid comes from the caller, as from the options in the reference)."""
    import numpy as np
    out = np.empty(tuple(shape), dtype=np.float32)
    _check(lib.claire_b200_read_bin(os.fsencode(path), _nx(out.shape), out.ctypes.data_as(ctypes.c_void_p)),
           "read_bin")
    return out


def write_bin(path: str, arr) -> None:
    """ReadWriteReg::WriteBIN: a PETSc binary vector (big-endian doubles)."""
    import numpy as np
    a = np.ascontiguousarray(arr, dtype=np.float32)
    if a.ndim != 3:
        raise ValueError("expected a 3D volume")
    _check(lib.claire_b200_write_bin(os.fsencode(path), _nx(a.shape), a.ctypes.data_as(ctypes.c_void_p)),
           "write_bin")


def read_image(path: str, shape=None):
    """ReadWriteReg::Read (src/ReadWriteReg.cpp:440-475): by extension, NIfTI-1
    (.nii, .nii.gz, .hdr / .img) or a PETSc binary vector (.bin, needs shape)."""
    if ".bin" in os.path.basename(path):
        if shape is None:
            raise ValueError("a .bin vector holds no grid: pass shape")
        return read_bin(path, shape)
    return read_nifti(path)


def write_image(path: str, arr) -> None:
    """ReadWriteReg::Write (src/ReadWriteReg.cpp:700-745): by extension."""
    if ".bin" in os.path.basename(path):
        return write_bin(path, arr)
    return write_nifti(path, arr)


def preprocess(m, rescale: bool = True, sigma=(1.0, 1.0, 1.0)):
    """Image preparation of the file path, in place on a CUDA tensor:
    Normalize (rescale) then Gaussian smoothing with sigma grid cells
    (sigma None: no smoothing)."""
    sig = None if sigma is None else (ctypes.c_double * 3)(*[float(x) for x in sigma])
    _check(lib.claire_b200_preprocess(_dev_ptr(m), _nx(m.shape), int(bool(rescale)), sig, _stream()),
           "preprocess")
    return m


def grid_change(f, nt: int):
    """Preprocessing::Restrict / Prolong of a cubic CUDA field, or of a stack of
    them (leading dimension), to nt^3 points."""
    torch = _torch()
    ns = f.shape[-1]
    nf = 1
    for k in f.shape[:-3]:
        nf *= int(k)
    out = torch.empty(tuple(f.shape[:-3]) + (nt, nt, nt), device=f.device, dtype=torch.float32)
    _check(lib.claire_b200_grid_change(_dev_ptr(f), int(ns), _dev_ptr(out), int(nt), nf, _stream()), "grid_change")
    return out


def fft_variant(n: int) -> int:
    return int(lib.claire_b200_fft_variant(int(n)))


def set_fft_variant(n: int, variant: int) -> None:
    _check(lib.claire_b200_set_fft_variant(int(n), int(variant)), "set_fft_variant")


def kernel_launches() -> int:
    """CUDA kernel launches issued by the library since it was loaded."""
    return int(lib.claire_b200_kernel_launches())


def stage_timeouts() -> int:
    """Tile gathers on the current device whose shared-memory box copy ran out
    of its bounded wait (claire_b200_stage_timeouts)."""
    c = ctypes.c_longlong(0)
    _check(lib.claire_b200_stage_timeouts(ctypes.byref(c)), "stage_timeouts")
    return int(c.value)


def stage_wait_selftest(wait_ns: int = 1_000_000) -> None:
    """Make one bounded box-copy wait run out (claire_b200_stage_wait_selftest)."""
    _check(lib.claire_b200_stage_wait_selftest(int(wait_ns), _stream()), "stage_wait_selftest")


# ---------------------------------------------------------------------------
# tensor helpers (torch is only the device-memory / stream plumbing)
# ---------------------------------------------------------------------------

def _torch():
    import torch  # noqa: WPS433 (imported lazily: the ABI itself does not need torch)
    return torch


def _dev_ptr(t, shape_hint: str = ""):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"expected a CUDA tensor {shape_hint}")
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise TypeError(f"expected a contiguous float32 CUDA tensor {shape_hint}")
    return ctypes.c_void_p(t.data_ptr())


def _dev_ptr_bf16(t, shape_hint: str = ""):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.bfloat16 or not t.is_contiguous():
        raise TypeError(f"expected a contiguous bfloat16 CUDA tensor {shape_hint}")
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _nx(shape) -> ctypes.Array:
    return (ctypes.c_int * 3)(*[int(s) for s in shape])


# ---------------------------------------------------------------------------
# reg::RegOpt
# ---------------------------------------------------------------------------

class RegOpt:
    """Hot-path subset of reg::RegOpt; ``RegOpt(["-nx", "64", ...])`` parses CLAIRE flags."""

    def __init__(self, argv: Optional[Sequence[str]] = None, **kw):
        self.opts = Opts()
        _check(lib.claire_b200_default_opts(ctypes.byref(self.opts)), "RegOpt")
        if argv:
            arr = (ctypes.c_char_p * len(argv))(*[a.encode() for a in argv])
            _check(lib.claire_b200_parse_args(ctypes.byref(self.opts), len(argv), arr), "RegOpt.ParseArguments")
        for k, v in kw.items():
            self.set(k, v)

    def set(self, key, value):
        o = self.opts
        if key == "nx":
            vals = [value] * 3 if isinstance(value, int) else list(value)
            for i in range(3):
                o.nx[i] = int(vals[i])
        elif key == "regnorm":
            o.regnorm = NORMS[value] if isinstance(value, str) else int(value)
            o.model = MODELS["compressible"]
        elif key == "model":
            o.model = MODELS[value] if isinstance(value, str) else int(value)
        elif key == "beta":
            vals = [value] if isinstance(value, (int, float)) else list(value)
            for i, b in enumerate(vals):
                o.beta[i] = float(b)
        elif key == "krylovtol":
            o.krylovtol[0] = float(value)
        elif hasattr(o, key):
            setattr(o, key, type(getattr(o, key))(value))
        else:
            raise KeyError(key)
        return self

    @property
    def nx(self):
        return tuple(self.opts.nx)

    @property
    def nt(self):
        return int(self.opts.nt)

    def estimate_bytes(self, nbatch: int = 1) -> int:
        return int(lib.claire_b200_estimate_bytes(ctypes.byref(self.opts), nbatch))


# ---------------------------------------------------------------------------
# reg::CLAIREInterface (batched: nbatch independent problems of one size)
# ---------------------------------------------------------------------------

class CLAIREInterface:
    """Drop-in for reg::CLAIREInterface; images and velocities are NumPy arrays
    (host) or torch CUDA tensors (device, copied on set)."""

    def __init__(self, opt: RegOpt, nbatch: int = 1):
        self.opt = opt
        self.nbatch = nbatch
        self._ctx = ctypes.c_void_p()
        _check(lib.claire_b200_create(ctypes.byref(opt.opts), nbatch, ctypes.byref(self._ctx)), "CLAIREInterface")
        self.shape = opt.nx

    def close(self):
        if self._ctx:
            lib.claire_b200_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- data -----------------------------------------------------------------
    def _src(self, arr, count):
        torch = _torch()
        if isinstance(arr, torch.Tensor):
            if arr.is_cuda:
                t = arr.detach().to(torch.float32).contiguous()
                if t.numel() != count:
                    raise ValueError("size mismatch")
                return ctypes.c_void_p(t.data_ptr()), 1, t
            arr = arr.numpy()
        import numpy as np
        a = np.ascontiguousarray(arr, dtype=np.float32)
        if a.size != count:
            raise ValueError(f"size mismatch: {a.size} != {count}")
        return a.ctypes.data_as(ctypes.c_void_p), 0, a

    def _n(self):
        n1, n2, n3 = self.shape
        return n1 * n2 * n3

    def set_problem_opts(self, b: int, opt: RegOpt):
        _check(lib.claire_b200_set_problem_opts(self._ctx, b, ctypes.byref(opt.opts)), "set_problem_opts", self._ctx)

    def SetReferenceImage(self, mR, b: int = 0):
        self._mR = (b, mR)
        if getattr(self, "_mT", None) is not None and self._mT[0] == b:
            self._set_images(b)

    def SetTemplateImage(self, mT, b: int = 0):
        self._mT = (b, mT)
        if getattr(self, "_mR", None) is not None and self._mR[0] == b:
            self._set_images(b)

    def set_images(self, mR, mT, b: int = 0):
        pr, devr, keep_r = self._src(mR, self._n())
        pt, devt, keep_t = self._src(mT, self._n())
        if devr != devt:
            raise ValueError("mR and mT must both be host arrays or both CUDA tensors")
        _check(lib.claire_b200_set_images(self._ctx, b, pr, pt, devr), "SetImages", self._ctx)

    def _set_images(self, b):
        self.set_images(self._mR[1], self._mT[1], b)
        self._mR = self._mT = None

    def SetMask(self, w, b: int = 0):
        """Distance-measure weights of problem b (None removes the mask)."""
        if w is None:
            _check(lib.claire_b200_set_mask(self._ctx, b, None, 0), "SetMask", self._ctx)
            return
        p, dev, keep = self._src(w, self._n())
        _check(lib.claire_b200_set_mask(self._ctx, b, p, dev), "SetMask", self._ctx)

    def SetInitialGuess(self, v, b: int = 0):
        p, dev, keep = self._src(v, 3 * self._n())
        _check(lib.claire_b200_set_velocity(self._ctx, b, p, dev), "SetInitialGuess", self._ctx)

    def GetSolution(self, b: int = 0, out=None):
        import numpy as np
        if out is None:
            out = np.empty((3,) + tuple(self.shape), dtype=np.float32)
            _check(lib.claire_b200_get_velocity(self._ctx, b, out.ctypes.data_as(ctypes.c_void_p), 0), "GetSolution",
                   self._ctx)
            return out
        _check(lib.claire_b200_get_velocity(self._ctx, b, _dev_ptr(out), 1), "GetSolution", self._ctx)
        return out

    def GetFinalState(self, b: int = 0, out=None):
        import numpy as np
        if out is None:
            out = np.empty(tuple(self.shape), dtype=np.float32)
            _check(lib.claire_b200_get_final_state(self._ctx, b, out.ctypes.data_as(ctypes.c_void_p), 0),
                   "GetFinalState", self._ctx)
            return out
        _check(lib.claire_b200_get_final_state(self._ctx, b, _dev_ptr(out), 1), "GetFinalState", self._ctx)
        return out

    def Run(self, mask: Optional[Sequence[int]] = None):
        if mask is None:
            _check(lib.claire_b200_run(self._ctx), "Run", self._ctx)
        else:
            arr = (ctypes.c_int * self.nbatch)(*[int(x) for x in mask])
            _check(lib.claire_b200_run_masked(self._ctx, arr), "Run", self._ctx)

    def SolveForwardProblem(self, m0, b: int = 0):
        import numpy as np
        p, dev, keep = self._src(m0, self._n())
        if dev:
            torch = _torch()
            out = torch.empty_like(keep)
            _check(lib.claire_b200_forward(self._ctx, b, p, _dev_ptr(out), 1), "SolveForwardProblem", self._ctx)
            return out
        out = np.empty(tuple(self.shape), dtype=np.float32)
        _check(lib.claire_b200_forward(self._ctx, b, p, out.ctypes.data_as(ctypes.c_void_p), 0),
               "SolveForwardProblem", self._ctx)
        return out

    def ComputeDetDefGrad(self, b: int = 0, inverse: bool = False):
        """det(grad y) at the current velocity (DeformationFields::ComputeDetDefGrad, SL
        solver): (J as a host array, (min, mean, max))."""
        import numpy as np
        jac = np.empty(tuple(self.shape), dtype=np.float32)
        st = (ctypes.c_double * 3)()
        _check(lib.claire_b200_det_def_grad(self._ctx, b, int(bool(inverse)), jac.ctypes.data_as(ctypes.c_void_p), st),
               "ComputeDetDefGrad", self._ctx)
        return jac, (st[0], st[1], st[2])

    def profile(self, enable: bool = True) -> None:
        """Bracket every time-step kernel launch with CUDA events (instrumented runs)."""
        _check(lib.claire_b200_profile(self._ctx, int(bool(enable))), "profile", self._ctx)

    def profile_read(self, category: int):
        """(device ms, launches) of a timer category since the last read; resets it."""
        ms = ctypes.c_double(0.0)
        cnt = ctypes.c_longlong(0)
        _check(lib.claire_b200_profile_read(self._ctx, int(category), ctypes.byref(ms), ctypes.byref(cnt)),
               "profile_read", self._ctx)
        return float(ms.value), int(cnt.value)

    def stats(self, b: int = 0) -> dict:
        st = Stats()
        _check(lib.claire_b200_get_stats(self._ctx, b, ctypes.byref(st)), "stats", self._ctx)
        return st.as_dict()

    def footprint_bytes(self) -> int:
        return int(lib.claire_b200_footprint_bytes(self._ctx))

    def set_stream(self, stream=None):
        """Issue the context's work on a torch.cuda.Stream (None: its own stream)."""
        handle = ctypes.c_void_p(stream.cuda_stream) if stream is not None else ctypes.c_void_p()
        _check(lib.claire_b200_set_stream(self._ctx, handle), "set_stream", self._ctx)

    def synchronize(self):
        _check(lib.claire_b200_synchronize(self._ctx), "synchronize", self._ctx)

    # --- OptimizationProblem seams (host NumPy arrays) -------------------------
    def EvaluateObjective(self, v, b: int = 0):
        p, _, keep = self._src(v, 3 * self._n())
        J, D, R = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(lib.claire_b200_objective(self._ctx, b, p, ctypes.byref(J), ctypes.byref(D), ctypes.byref(R)),
               "EvaluateObjective", self._ctx)
        return J.value, D.value, R.value

    def EvaluateGradient(self, v, b: int = 0):
        import numpy as np
        p, _, keep = self._src(v, 3 * self._n())
        g = np.empty((3,) + tuple(self.shape), dtype=np.float32)
        _check(lib.claire_b200_gradient(self._ctx, b, p, g.ctypes.data_as(ctypes.c_void_p)), "EvaluateGradient",
               self._ctx)
        return g

    def HessianMatVec(self, v, vt, b: int = 0):
        import numpy as np
        p, _, keep = self._src(v, 3 * self._n())
        pt, _, keep_t = self._src(vt, 3 * self._n())
        h = np.empty((3,) + tuple(self.shape), dtype=np.float32)
        _check(lib.claire_b200_hessian_matvec(self._ctx, b, p, pt, h.ctypes.data_as(ctypes.c_void_p)),
               "HessianMatVec", self._ctx)
        return h

    def ApplyInvRegularizationOperator(self, x, b: int = 0):
        import numpy as np
        p, _, keep = self._src(x, 3 * self._n())
        out = np.empty((3,) + tuple(self.shape), dtype=np.float32)
        _check(lib.claire_b200_precond(self._ctx, b, p, out.ctypes.data_as(ctypes.c_void_p)), "Precond", self._ctx)
        return out

    def ComputeDeformationMap(self, inverse: bool = False, b: int = 0):
        """DeformationFields::ComputeDeformationMap (SL RK2) at the current
        velocity: positions y (3, n1, n2, n3) in physical coordinates."""
        import numpy as np
        y = np.empty((3,) + tuple(self.shape), dtype=np.float32)
        _check(lib.claire_b200_deformation_map(self._ctx, b, int(bool(inverse)), y.ctypes.data_as(ctypes.c_void_p)),
               "ComputeDeformationMap", self._ctx)
        return y

    def ComputeDefGrad(self, b: int = 0):
        """DeformationFields::ComputeDefGrad (SL) at the current velocity:
        (F (9, n1, n2, n3) with F_ab at 3a + b, det F, (min, mean, max))."""
        import numpy as np
        F = np.empty((9,) + tuple(self.shape), dtype=np.float32)
        det = np.empty(tuple(self.shape), dtype=np.float32)
        st = (ctypes.c_double * 3)()
        _check(lib.claire_b200_def_grad(self._ctx, b, F.ctypes.data_as(ctypes.c_void_p),
                                        det.ctypes.data_as(ctypes.c_void_p), st), "ComputeDefGrad", self._ctx)
        return F, det, (st[0], st[1], st[2])

    def ComputeDetDefGradViaDispField(self, b: int = 0):
        """det(grad y) through the displacement field (-detdefgradfromdeffield):
        (det field, (min, mean, max))."""
        import numpy as np
        jac = np.empty(tuple(self.shape), dtype=np.float32)
        st = (ctypes.c_double * 3)()
        _check(lib.claire_b200_det_def_grad_disp(self._ctx, b, jac.ctypes.data_as(ctypes.c_void_p), st),
               "ComputeDetDefGradViaDispField", self._ctx)
        return jac, (st[0], st[1], st[2])

    def ComputeDisplacementField(self, b: int = 0):
        """DeformationFields::ComputeDisplacementFieldSL at the current velocity:
        u (3, n1, n2, n3), physical units."""
        import numpy as np
        u = np.empty((3,) + tuple(self.shape), dtype=np.float32)
        _check(lib.claire_b200_displacement_field(self._ctx, b, u.ctypes.data_as(ctypes.c_void_p)),
               "ComputeDisplacementField", self._ctx)
        return u

    def GetAdjoint(self, b: int = 0):
        import numpy as np
        lam = np.empty(tuple(self.shape), dtype=np.float32)
        bf = np.empty((3,) + tuple(self.shape), dtype=np.float32)
        _check(lib.claire_b200_get_adjoint(self._ctx, b, lam.ctypes.data_as(ctypes.c_void_p),
                                           bf.ctypes.data_as(ctypes.c_void_p)), "GetAdjoint", self._ctx)
        return lam, bf


# ---------------------------------------------------------------------------
# inner operator seams on torch CUDA tensors
# ---------------------------------------------------------------------------

class SemiLagrangian:
    """ComputeTrajectory / Interpolate on device tensors (src/SemiLagrangian.cpp)."""

    def __init__(self, nt: int):
        self.nt = nt

    def ComputeTrajectory(self, v, flag: str = "state", out=None):
        torch = _torch()
        shape = v.shape[1:]
        if out is None:
            out = torch.empty_like(v)
        f = {"state": 0, "adjoint": 1}[flag]
        _check(lib.claire_b200_trajectory(_dev_ptr(v), _dev_ptr(out), _nx(shape), self.nt, f, _stream()),
               "ComputeTrajectory")
        return out

    @staticmethod
    def Interpolate(f, disp, out=None):
        torch = _torch()
        dof = 3 if f.dim() == 4 else 1
        shape = f.shape[-3:]
        if out is None:
            out = torch.empty_like(f)
        _check(lib.claire_b200_interp3(_dev_ptr(f), _dev_ptr(disp), _dev_ptr(out), _nx(shape), dof, _stream()),
               "Interpolate")
        return out

    @staticmethod
    def InterpolateBF16(f, disp, out=None):
        """Interpolate one bfloat16 volume (the -bf16images storage format)."""
        torch = _torch()
        if out is None:
            out = torch.empty_like(f)
        _check(lib.claire_b200_interp3_bf16(_dev_ptr_bf16(f), _dev_ptr(disp), _dev_ptr_bf16(out), _nx(f.shape),
                                            _stream()), "InterpolateBF16")
        return out


class Regularization:
    """Spectral regularisation operators on device tensors (src/Regularization*.cpp)."""

    def __init__(self, norm: str = "h1s", beta0: float = 1e-2, beta1: float = 1e-4):
        self.norm = norm
        self.beta = (ctypes.c_double * 2)(beta0, beta1)

    def _apply(self, v, kind, out=None):
        torch = _torch()
        if out is None:
            out = torch.empty_like(v)
        _check(lib.claire_b200_reg_apply(_dev_ptr(v), _dev_ptr(out), _nx(v.shape[1:]), NORMS[self.norm], self.beta,
                                         REG_KIND[kind], _stream()), "Regularization")
        return out

    def EvaluateGradient(self, v, out=None):
        return self._apply(v, "gradient", out)

    HessianMatVec = EvaluateGradient

    def ApplyInverse(self, v, applysqrt: bool = False, out=None):
        return self._apply(v, "sqrtinverse" if applysqrt else "inverse", out)

    def EvaluateFunctional(self, v) -> float:
        R = ctypes.c_double()
        _check(lib.claire_b200_reg_functional(_dev_ptr(v), ctypes.byref(R), _nx(v.shape[1:]), NORMS[self.norm],
                                              self.beta, _stream()), "EvaluateFunctional")
        return R.value


class Preconditioner(Regularization):
    """INVREG preconditioner: P x = (beta A)^-1 x (src/Preconditioner.cpp:549-580)."""

    def MatVec(self, x, out=None):
        return self.ApplyInverse(x, False, out)


class DistanceMeasureSL2:
    @staticmethod
    def EvaluateFunctional(mR, m1) -> float:
        D = ctypes.c_double()
        _check(lib.claire_b200_distance(_dev_ptr(mR), _dev_ptr(m1), _nx(mR.shape), ctypes.byref(D), _stream()),
               "DistanceMeasureSL2")
        return D.value


def fft_grad(f, out=None):
    torch = _torch()
    if out is None:
        out = torch.empty((3,) + tuple(f.shape), device=f.device, dtype=torch.float32)
    _check(lib.claire_b200_fft_grad(_dev_ptr(f), _dev_ptr(out), _nx(f.shape), _stream()), "fft_grad")
    return out


def fft_div(v, out=None):
    torch = _torch()
    if out is None:
        out = torch.empty(tuple(v.shape[1:]), device=v.device, dtype=torch.float32)
    _check(lib.claire_b200_fft_div(_dev_ptr(v), _dev_ptr(out), _nx(v.shape[1:]), _stream()), "fft_div")
    return out


def leray(b, model: str = "stokes", beta=(1e-2, 1e-4, 1e-4)):
    """In place: b += projection addend (CLAIREStokes / CLAIREDivReg ::ApplyProjection)."""
    arr = (ctypes.c_double * 3)(*beta)
    _check(lib.claire_b200_leray(_dev_ptr(b), _nx(b.shape[1:]), MODELS[model], arr, _stream()), "leray")
    return b


def smooth(f, sigma=(1.0, 1.0, 1.0), out=None):
    torch = _torch()
    if out is None:
        out = torch.empty_like(f)
    arr = (ctypes.c_double * 3)(*sigma)
    _check(lib.claire_b200_smooth(_dev_ptr(f), _dev_ptr(out), _nx(f.shape), arr, _stream()), "smooth")
    return out


# ---------------------------------------------------------------------------
# serving: continuous batching of registrations (claire_b200_server_*)
# ---------------------------------------------------------------------------
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = 0, 1, 2, 3, 4


class Server:
    """Registration server: requests of any supported grid / nt / norm / beta
    are queued, admitted into solver slots at GN-iteration boundaries as slots
    and HBM free up, and retired when their stopping test fires.  Images are
    host arrays (NumPy float32 or CPU tensors); results are host arrays."""

    def __init__(self, slots_per_pool: int = 4, hbm_budget_bytes: int = 0, idle_ms: int = 2000, device: int = 0,
                 batch_window_us: int = 0):
        o = ServerOpts()
        lib.claire_b200_server_default_opts(ctypes.byref(o))
        o.slots_per_pool = int(slots_per_pool)
        o.hbm_budget_bytes = int(hbm_budget_bytes)
        o.idle_ms = int(idle_ms)
        o.device = int(device)
        o.batch_window_us = int(batch_window_us)
        h = ctypes.c_void_p()
        _check(lib.claire_b200_server_create(ctypes.byref(o), ctypes.byref(h)), "Server")
        self._srv = h

    @staticmethod
    def _host(x):
        import numpy as np
        if hasattr(x, "detach"):
            x = x.detach().cpu().numpy()
        return np.ascontiguousarray(x, dtype=np.float32)

    def submit(self, opt: "RegOpt", mR, mT) -> int:
        a, b = self._host(mR), self._host(mT)
        n = opt.opts.nx[0] * opt.opts.nx[1] * opt.opts.nx[2]
        if a.size != n or b.size != n:
            raise ValueError("image size does not match the options' grid")
        rid = ctypes.c_longlong(0)
        _check(lib.claire_b200_server_submit(self._srv, ctypes.byref(opt.opts), a.ctypes.data_as(ctypes.c_void_p),
                                             b.ctypes.data_as(ctypes.c_void_p), ctypes.byref(rid)), "Server.submit")
        self._shape = tuple(opt.opts.nx)
        return int(rid.value)

    def poll(self, rid: int) -> int:
        st = ctypes.c_int(0)
        _check(lib.claire_b200_server_poll(self._srv, rid, ctypes.byref(st)), "Server.poll")
        return st.value

    def wait(self, rid: int, timeout_ms: int = -1) -> int:
        st = ctypes.c_int(0)
        _check(lib.claire_b200_server_wait(self._srv, rid, int(timeout_ms), ctypes.byref(st)), "Server.wait")
        return st.value

    def result(self, rid: int, shape):
        """(velocity (3, *shape), stats dict, submit-to-done latency ms); releases the request."""
        import numpy as np
        v = np.empty((3,) + tuple(shape), dtype=np.float32)
        st = Stats()
        lat = ctypes.c_double(0.0)
        _check(lib.claire_b200_server_result(self._srv, rid, v.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st),
                                             ctypes.byref(lat)), "Server.result")
        return v, st.as_dict(), float(lat.value)

    def cancel(self, rid: int) -> None:
        """Cancel a queued request at once, or a running one at its pool's next
        GN-iteration boundary (claire_b200_server_cancel)."""
        _check(lib.claire_b200_server_cancel(self._srv, rid), "Server.cancel")

    def info(self) -> dict:
        pools, queued = ctypes.c_int(0), ctypes.c_int(0)
        used = ctypes.c_longlong(0)
        _check(lib.claire_b200_server_info(self._srv, ctypes.byref(pools), ctypes.byref(used), ctypes.byref(queued)),
               "Server.info")
        return {"pools": pools.value, "bytes_used": used.value, "queued": queued.value}

    def close(self):
        if getattr(self, "_srv", None):
            lib.claire_b200_server_destroy(self._srv)
            self._srv = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
