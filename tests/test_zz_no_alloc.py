"""claire_b200_reg_apply_noalloc against claire_b200_reg_apply, through the C ABI.

The no-allocation entry point serves callers that cannot allocate device
memory while the operator runs (their own pool already holds the GPU budget,
or an allocation would synchronise the device or could fail mid-run).  It keeps
its FFT workspace in fixed device arrays inside the library, so these checks
make sure that shared workspace gives the same results as the allocating seam,
on consecutive calls with different inputs, and that grids above its 64^3
limit are refused before anything runs.

This file sorts last so a stop-at-first-failure run has already run every
other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5
NORMS = {"l2": 0, "h1": 1, "h1s": 2, "h2": 3, "h2s": 4, "h3": 5, "h3s": 6}
KINDS = {"gradient": 0, "inverse": 1, "sqrtinverse": 2}


def _call(lib, fn, v, out, n, norm, kind, beta, stream):
    nx = (ctypes.c_int * 3)(n, n, n)
    b = (ctypes.c_double * 2)(*beta)
    return getattr(lib, fn)(ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(out.data_ptr()), nx, NORMS[norm], b,
                            KINDS[kind], ctypes.c_void_p(stream))


def _rel(a, b):
    a = a.double()
    b = b.double()
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("n", [16, 32, 48, 64])
@pytest.mark.parametrize("norm,kind", [("h1s", "inverse"), ("h2", "gradient"), ("h1", "inverse"), ("l2", "gradient"),
                                       ("h2s", "sqrtinverse"), ("h3", "inverse"), ("h3s", "gradient"),
                                       ("h2", "sqrtinverse")])
def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(cuda, n, norm, kind):
    import torch
    import claire_b200 as cb
    lib = cb.lib
    stream = torch.cuda.current_stream().cuda_stream
    beta = (1e-2, 1e-4)
    gen = torch.Generator(device="cuda").manual_seed(n)
    for call in range(2):   # two calls in a row, different inputs
        v = torch.randn((3, n, n, n), device=cuda, generator=gen)
        ref = torch.empty_like(v)
        got = torch.full_like(v, float("nan"))
        assert _call(lib, "claire_b200_reg_apply", v, ref, n, norm, kind, beta, stream) == 0
        assert _call(lib, "claire_b200_reg_apply_noalloc", v, got, n, norm, kind, beta, stream) == 0
        torch.cuda.synchronize()
        assert torch.isfinite(got).all(), f"call {call}: output not fully written"
        assert _rel(got, ref) <= TOL, f"call {call}"


def test_noalloc_allocates_nothing(cuda):
    """After the first call on the device (its set-up, and the lazy loading of
    its kernels), further calls leave the device's free memory and the torch
    allocator's counters unchanged."""
    import torch
    import claire_b200 as cb
    n = 64
    stream = torch.cuda.current_stream().cuda_stream
    v = torch.randn((3, n, n, n), device=cuda)
    out = torch.empty_like(v)
    for kind in ("inverse", "gradient", "sqrtinverse"):
        assert _call(cb.lib, "claire_b200_reg_apply_noalloc", v, out, n, "h2", kind, (1e-3, 1e-4), stream) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0, reserved0 = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
    for _ in range(3):
        for kind in ("inverse", "gradient", "sqrtinverse"):
            assert _call(cb.lib, "claire_b200_reg_apply_noalloc", v, out, n, "h2", kind, (1e-3, 1e-4), stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0 and torch.cuda.memory_reserved() == reserved0


def test_noalloc_rejects_misaligned_buffers(cuda):
    import torch
    import claire_b200 as cb
    n = 32
    buf = torch.zeros(3 * n ** 3 + 4, device=cuda)
    v = buf[1:1 + 3 * n ** 3]            # 4-byte offset: not 16-byte aligned
    out = torch.zeros(3 * n ** 3, device=cuda)
    rc = _call(cb.lib, "claire_b200_reg_apply_noalloc", v, out, n, "h1s", "inverse", (1e-2, 1e-4),
               torch.cuda.current_stream().cuda_stream)
    assert rc == -1   # CB_ERR_ARG, before anything is launched
    torch.cuda.synchronize()
    assert float(out.abs().max()) == 0.0


def test_noalloc_rejects_grids_above_its_workspace(cuda):
    import torch
    import claire_b200 as cb
    n = 96
    v = torch.zeros((3, n, n, n), device=cuda)
    out = torch.zeros_like(v)
    rc = _call(cb.lib, "claire_b200_reg_apply_noalloc", v, out, n, "h1s", "inverse", (1e-2, 1e-4),
               torch.cuda.current_stream().cuda_stream)
    assert rc == -7   # CB_ERR_TOO_LARGE
    torch.cuda.synchronize()
    assert float(out.abs().max()) == 0.0
