"""The oracle's tricubic interpolation against the reference's own kernel.

optimized_interp3_ghost_xyz_p (src/interp3.cpp:2492-2719) is compiled from
the reference's source by oracle/build_ref.py (double and single builds; the
reference tree is needed to build them, the built libraries travel with the
repository).  The NumPy oracle and the C++ restatement must give its values
on random fields at random query points, including points that wrap around
the periodic domain more than once.
"""
import numpy as np
import pytest

from oracle import claire_ref as R
from oracle import ref_interp3
from oracle.cpu_ref import CpuRef

pytestmark = pytest.mark.skipif(not (ref_interp3.available("f64") and ref_interp3.available("f32")),
                                reason="oracle/_ref not built (needs the reference tree at build time)")


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a, np.float64) - np.asarray(b, np.float64)).ravel())
                 / np.linalg.norm(np.asarray(b, np.float64).ravel()))


@pytest.mark.parametrize("shape,span", [((16, 16, 16), 3.0), ((16, 24, 32), 3.0), ((32, 16, 48), 40.0)])
def test_oracle_interpolation_equals_reference_kernel(shape, span):
    rng = np.random.default_rng(7)
    f = rng.standard_normal(shape)
    disp = rng.uniform(-span, span, (3,) + shape)
    ref64 = ref_interp3.interp3(f, disp, "f64")
    assert rel(R.interp3(f, R.index_grid(shape) + disp), ref64) < 1e-13
    c = CpuRef(shape, 4, "h1s", 1e-2, fp64=True, threads=2)
    assert rel(c.interp(f, disp), ref64) < 1e-13
    # single builds: the reference's and the restatement's FP32 kernels (the
    # normalised query coordinates are FP32 too: ~N * 6e-8 grid units)
    ref32 = ref_interp3.interp3(f.astype(np.float32), disp, "f32")
    assert rel(ref32, ref64) < 5e-6
    c32 = CpuRef(shape, 4, "h1s", 1e-2, fp64=False, threads=2)
    assert rel(c32.interp(f.astype(np.float32), disp), ref32) < 5e-6


def test_node_values_and_cubics_through_the_reference_kernel():
    """Known answers of the Lagrange kernel itself: at integer displacements it
    returns the shifted field exactly; it reproduces trig-free cubics in the
    interior (periodic sampling of a smooth field makes the check local)."""
    shape = (16, 16, 16)
    rng = np.random.default_rng(3)
    f = rng.standard_normal(shape)
    shift = np.stack([np.full(shape, s, dtype=np.float64) for s in (2.0, -1.0, 5.0)])
    out = ref_interp3.interp3(f, shift, "f64")
    assert np.array_equal(out, np.roll(f, (-2, 1, -5), axis=(0, 1, 2)))
