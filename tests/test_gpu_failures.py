"""Failure detection on the host side: bad inputs, memory limits, cancellation.

The reference propagates PetscErrorCode through CHKERRQ and stops TAO with
TAO_DIVERGED_NAN when the objective or the gradient norm is not finite
(src/TaoInterface.cpp:425-436).  Here every entry point returns a status
code; these tests make the failure on the host (a NaN written into a host
image, a batch too large for the device, a budget smaller than a pool, a
cancelled request) or let a bounded device wait run out on a flag nothing
sets, and check that it is reported cleanly, that the other problems of a
batch or of a server are unaffected, and that the context or server stays
usable.  No test faults, traps or hangs the GPU.
"""
import os
import time

import numpy as np
import pytest

from oracle import claire_ref as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cb(cuda):
    import claire_b200
    return claire_b200


def opt32(cb, maxit=4, **kw):
    o = cb.RegOpt(["-nx", "32", "-nt", "4", "-regnorm", "h1s", "-beta", "1e-2", "-maxit", str(maxit),
                   "-opttol", "1e-2"])
    for k, v in kw.items():
        o.set(k, v)
    return o


def c1_32():
    mR, mT, _ = R.synthetic_c1(32, np.float64, 4)
    return mR.astype(np.float32), mT.astype(np.float32)


def test_nan_input_stops_with_reason_nan_and_spares_the_batch(cb):
    mR, mT = c1_32()
    bad = mR.copy()
    bad[3, 4, 5] = np.nan
    with cb.CLAIREInterface(opt32(cb)) as alone:
        alone.set_images(mR, mT)
        alone.Run()
        v_alone = alone.GetSolution()
        st_alone = alone.stats()
    with cb.CLAIREInterface(opt32(cb), nbatch=2) as ci:
        ci.set_images(bad, mT, 0)
        ci.set_images(mR, mT, 1)
        ci.Run()  # returns normally: the NaN is a stopping reason, not an error
        st_bad = ci.stats(0)
        st_ok = ci.stats(1)
        v_ok = ci.GetSolution(1)
    assert st_bad["converged_reason"] == -1  # TAO_DIVERGED_NAN
    assert st_bad["gn_iterations"] == 0
    assert st_ok["converged_reason"] == st_alone["converged_reason"]
    assert st_ok["gn_iterations"] == st_alone["gn_iterations"]
    assert st_ok["pcg_iterations"] == st_alone["pcg_iterations"]
    assert np.array_equal(v_ok, v_alone)


def test_footprint_above_free_memory_is_refused_before_allocating(cb):
    import torch
    free0, _ = torch.cuda.mem_get_info()
    big = cb.RegOpt(["-nx", "256", "-nt", "8", "-regnorm", "h2", "-beta", "1e-3"])
    nb = int(free0 // big.estimate_bytes(1)) + 2
    with pytest.raises(cb.ClaireError) as e:
        cb.CLAIREInterface(big, nbatch=nb)
    assert e.value.code == cb.ERR_TOO_LARGE
    free1, _ = torch.cuda.mem_get_info()
    assert abs(free1 - free0) < 64 << 20  # nothing was left allocated
    # the device stays usable
    mR, mT = c1_32()
    with cb.CLAIREInterface(opt32(cb, maxit=1)) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        assert ci.stats()["gn_iterations"] == 1


def test_server_budget_smaller_than_a_pool(cb):
    mR, mT = c1_32()
    o = opt32(cb)
    need = o.estimate_bytes(2)
    with cb.Server(slots_per_pool=2, hbm_budget_bytes=need // 2) as srv:
        with pytest.raises(cb.ClaireError) as e:
            srv.submit(o, mR, mT)
        assert e.value.code == cb.ERR_TOO_LARGE
    with cb.Server(slots_per_pool=2, hbm_budget_bytes=need + (1 << 20)) as srv:
        rid = srv.submit(o, mR, mT)
        assert srv.wait(rid, 120000) == cb.REQ_DONE


def test_server_cancel_queued_and_running(cb):
    mR, mT = c1_32()
    # every GN iteration runs 49 PCG iterations (fixed Krylov tolerance 1e-30),
    # and the gradient tests never fire: a request stays running for a while
    o = opt32(cb, maxit=6, opttol=0.0, gatol=0.0, krylovfseq=0, krylovtol=1e-30)  # CB_FSEQ_NONE
    with cb.Server(slots_per_pool=1, idle_ms=60000) as srv:
        r0 = srv.submit(o, mR, mT)  # the result a request computes alone
        assert srv.wait(r0, 300000) == cb.REQ_DONE
        v_ref, st_ref, _ = srv.result(r0, (32, 32, 32))
        running = srv.submit(o, mR, mT)
        queued = srv.submit(o, mR, mT)   # same key: waits for the one slot
        after = srv.submit(o, mR, mT)
        t0 = time.time()
        while srv.poll(running) == cb.REQ_QUEUED and time.time() - t0 < 60:
            time.sleep(0.005)
        assert srv.poll(running) == cb.REQ_RUNNING
        assert srv.poll(queued) == cb.REQ_QUEUED
        srv.cancel(queued)
        assert srv.poll(queued) == cb.REQ_CANCELLED
        srv.cancel(running)
        assert srv.wait(running, 300000) == cb.REQ_CANCELLED
        for rid in (queued, running):
            with pytest.raises(cb.ClaireError) as e:
                srv.result(rid, (32, 32, 32))
            assert e.value.code == cb.ERR_CANCELLED
        # the freed slot serves the next request, which computes what it computes alone
        assert srv.wait(after, 300000) == cb.REQ_DONE
        v, st, _ = srv.result(after, (32, 32, 32))
        assert st["gn_iterations"] == st_ref["gn_iterations"]
        assert st["pcg_iterations"] == st_ref["pcg_iterations"]
        assert np.array_equal(v, v_ref)
        with pytest.raises(cb.ClaireError):
            srv.cancel(after)  # already finished and released


def test_idle_pools_are_reaped(cb):
    mR, mT = c1_32()
    o = opt32(cb, maxit=1)
    tasks = lambda: len(os.listdir("/proc/self/task"))  # noqa: E731
    with cb.Server(slots_per_pool=1, idle_ms=20) as srv:
        rid = srv.submit(o, mR, mT)
        assert srv.wait(rid, 120000) == cb.REQ_DONE
        srv.result(rid, (32, 32, 32))
        time.sleep(0.5)
        srv.info()
        base = tasks()
        for _ in range(5):
            rid = srv.submit(o, mR, mT)
            assert srv.wait(rid, 120000) == cb.REQ_DONE
            srv.result(rid, (32, 32, 32))
            time.sleep(0.3)  # the pool idles out and its worker exits
        # info() joins and drops exited pools; a worker that is still
        # releasing its memory finishes within a few seconds
        deadline = time.time() + 10.0
        info = srv.info()
        while info["bytes_used"] != 0 and time.time() < deadline:
            time.sleep(0.05)
            info = srv.info()
        assert info["pools"] == 0
        assert info["bytes_used"] == 0
        assert tasks() <= base


def test_box_copy_wait_runs_out_cleanly(cb):
    """The tile gathers wait for their shared-memory box copies with a bounded
    wait.  The self-test arms a barrier for a copy that is never issued, so the
    wait (1 ms here) runs out: the count of timeouts grows by one, the kernel
    returns, and the device keeps computing correct gathers afterwards."""
    import torch
    before = cb.stage_timeouts()
    cb.stage_wait_selftest(1_000_000)
    torch.cuda.synchronize()
    assert cb.stage_timeouts() == before + 1
    n = 32
    rng = np.random.default_rng(9)
    f = rng.standard_normal((n, n, n)).astype(np.float32)
    disp = rng.uniform(-2.5, 2.5, size=(3, n, n, n)).astype(np.float32)
    out = cb.SemiLagrangian.Interpolate(torch.from_numpy(f).cuda(), torch.from_numpy(disp).cuda()).cpu().numpy()
    ref = R.interp3(f.astype(np.float64), R.index_grid((n, n, n)) + disp.astype(np.float64))
    assert np.linalg.norm((out - ref).ravel()) <= 1e-5 * np.linalg.norm(ref.ravel())
    assert cb.stage_timeouts() == before + 1  # real copies complete within the limit
