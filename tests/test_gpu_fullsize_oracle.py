"""Device parity at the benchmark's own sizes against the C++ FP64 oracle.

The NumPy oracle is too slow at 128^3 and 256^3; the C++/OpenMP restatement
(oracle/cpu_ref.cpp, pinned to the NumPy oracle in tests/test_cpu_ref.py)
runs there in seconds.  On the recipe problems of the 128^3 configuration
(H2, beta 1e-3, nt 8) and of the 256^3 one (H2, beta 1e-4, nt 8), at half the
recipe velocity (displacements of ~1.3 cells per time step at 128^3, so the
gathers see the recipe's box sizes), the device's transported image,
objective, gradient, GN Hessian matvec and preconditioner agree with the FP64
oracle on the same FP32 inputs within 1e-5 relative (L2 for fields).
"""
import numpy as np
import pytest

from oracle import claire_ref as R
from oracle.cpu_ref import CpuRef

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.mark.parametrize("n,norm,beta,config", [(128, "h2", 1e-3, 1), (256, "h2", 1e-4, 3)])
def test_operators_at_full_size(cuda, n, norm, beta, config):
    import torch

    import claire_b200 as cb
    from claire_b200 import synthetic

    nt = 8
    mR_d, mT_d, v_d = synthetic.ellipsoid_problem(n, nt, config, 0, cuda)
    torch.cuda.synchronize()
    mR = mR_d.cpu().numpy()
    mT = mT_d.cpu().numpy()
    v = (0.5 * v_d).cpu().numpy()
    del mR_d, mT_d, v_d
    # a smooth direction with the recipe's spectrum (the Hessian's data term
    # is then comparable to its regularisation term)
    rng = np.random.Generator(np.random.PCG64(7))
    vt = R.velocity_random((n, n, n), rng).astype(np.float32)

    ref = CpuRef((n,) * 3, nt, norm, beta, fp64=True)
    ref.set_images(mR, mT)
    m1_ref = ref.forward(v, mT)
    J_ref, D_ref, R_ref = ref.objective(v)
    g_ref = ref.gradient(v)
    H_ref = ref.hessian_matvec(v, vt)
    P_ref = ref.precond(vt)
    ref.close()

    opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", repr(beta)])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.SetInitialGuess(v)
        m1 = ci.SolveForwardProblem(mT)
        J, D, Rv = ci.EvaluateObjective(v)
        g = ci.EvaluateGradient(v)
        H = ci.HessianMatVec(v, vt)
        P = ci.ApplyInvRegularizationOperator(vt)
    torch.cuda.empty_cache()

    assert rel(m1, m1_ref) < 1e-5
    assert abs(D - D_ref) <= 1e-5 * abs(D_ref)
    assert abs(Rv - R_ref) <= 1e-5 * abs(R_ref)
    assert abs(J - J_ref) <= 1e-5 * abs(J_ref)
    assert rel(g, g_ref) < 1e-5
    assert rel(H, H_ref) < 1e-5
    assert rel(P, P_ref) < 1e-5
