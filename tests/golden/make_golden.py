"""Generate the oracle's (FP64) registrations that the GPU tests compare with:

* tests/golden/c1_64.json: the 64^3 synthetic problem (sin^2 template, trig
  velocity v* = 0.5 (sin x3 cos x2, sin x1 cos x3, sin x2 cos x1)), nt = 4,
  H1 seminorm beta = 1e-2;
* tests/golden/c3_64.json: a 64^3 problem of the ellipsoid / random-velocity
  recipe (seeded problem 0 of the mixed-batch set), nt = 4, H1 beta = 1e-2;

* tests/golden/c1_64_2level.json: the c1 problem solved with the two-level
  preconditioner (-precond 2level: symmetric preconditioned Hessian, coarse
  solve on 32^3);

all with GN + PCG (superlinear forcing) + Armijo, gradient tolerance 1e-2, at
most 10 GN iterations, INVREG unless named.  Too slow for a test run (NumPy),
so the results are committed: iteration counts, monitor values and velocity
projections onto seeded random fields.

    python tests/golden/make_golden.py [fixture.json ...]
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import claire_ref as R  # noqa: E402


def projections(v, k=8, seed=2026):
    """<v, w_i> for k seeded standard-normal fields w_i (velocity fingerprint)."""
    rng = np.random.default_rng(seed)
    return [float(np.sum(np.asarray(v, np.float64) * rng.standard_normal(v.shape))) for _ in range(k)]


def c1_images(n, nt):
    mR, mT, _ = R.synthetic_c1(n, np.float64, nt)
    return mR, mT, "oracle.synthetic_c1, cast to float32"


def c3_images(n, nt):
    rng = np.random.Generator(np.random.PCG64(R.problem_seed(2, 0)))
    shape = (n, n, n)
    mT = R.template_ellipsoids(shape, rng)
    v = R.velocity_random(shape, rng)
    mR = R.forward_transport(mT, v, nt)
    return mR, mT, "oracle ellipsoid template and random velocity, seed problem_seed(2, 0), cast to float32"


def make(name, images, n, nt, norm, beta, maxit=10, gttol=1e-2, precond="invreg"):
    mR, mT, what = images(n, nt)
    mR = mR.astype(np.float32)
    mT = mT.astype(np.float32)
    prob = R.Problem(mR, mT, nt, R.Regularization(norm, beta))
    t = time.time()
    res = R.gauss_newton(prob, R.GNOptions(maxit=maxit, gttol=gttol, precond=precond))
    v = res["v"]
    out = {
        "problem": {"n": n, "nt": nt, "regnorm": norm, "beta": beta, "maxit": maxit, "opttol": gttol,
                    "precond": precond, "images": what},
        "gn_iterations": res["iters"],
        "pcg_iterations": res["pcg_iters"],
        "reason": res["reason"],
        "J": res["J"],
        "gnorm": res["gnorm"],
        "g0": res["g0"],
        "rel_mismatch": R.relative_mismatch(prob.mR, res["m1"], prob.mT),
        "velocity_norm": float(np.linalg.norm(v.ravel())),
        "velocity_projections": projections(v),
        "seconds_numpy": time.time() - t,
    }
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(out, f, indent=1)
    print(name, json.dumps(out))


FIXTURES = {
    "c1_64.json": lambda: make("c1_64.json", c1_images, 64, 4, "h1s", 1e-2),
    "c3_64.json": lambda: make("c3_64.json", c3_images, 64, 4, "h1", 1e-2),
    "c1_64_2level.json": lambda: make("c1_64_2level.json", c1_images, 64, 4, "h1s", 1e-2, precond="2level"),
}


def main():
    for name in sys.argv[1:] or list(FIXTURES):
        FIXTURES[name]()


if __name__ == "__main__":
    main()
