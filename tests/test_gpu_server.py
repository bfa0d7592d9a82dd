"""Serving: continuous batching of registrations (claire_b200_server_*).

Each request's result must be the result of a plain CLAIREInterface::Run on
the same inputs, whether it runs alone or admitted into a pool next to other
requests (of the same key, or of other grids / norms / weights running
concurrently in other pools).  The slots of a pool share no data, so the
comparison is exact.
"""
import numpy as np
import pytest

from oracle import claire_ref as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cb(cuda):
    import claire_b200
    return claire_b200


def opt_for(cb, n, nt, norm, beta, maxit=4):
    return cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", str(beta), "-maxit", str(maxit),
                      "-opttol", "1e-2"])


def sin2(n, nt, v0=0.5):
    shape = (n, n, n)
    mT = R.rescale(R.template_sin2(shape))
    v = R.velocity_trig(shape, v0, reference_case=False)
    mR = R.rescale(R.forward_transport(mT, v, nt))
    return mR.astype(np.float32), mT.astype(np.float32)


def ellipsoids(n, nt, idx):
    shape = (n, n, n)
    rng = np.random.Generator(np.random.PCG64(R.problem_seed(3, idx)))
    mT = R.template_ellipsoids(shape, rng)
    v = R.velocity_random(shape, rng)
    mR = R.forward_transport(mT, v, nt)
    return mR.astype(np.float32), mT.astype(np.float32)


def plain_run(cb, opt, mR, mT):
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        return np.asarray(ci.GetSolution()), ci.stats()


def test_request_alone_equals_plain_run(cb):
    n, nt = 32, 4
    mR, mT = sin2(n, nt)
    opt = opt_for(cb, n, nt, "h1s", 1e-2)
    v_ref, st_ref = plain_run(cb, opt, mR, mT)
    with cb.Server(slots_per_pool=2, idle_ms=100) as srv:
        rid = srv.submit(opt, mR, mT)
        assert srv.wait(rid, 120000) == cb.REQ_DONE
        v, st, lat = srv.result(rid, (n, n, n))
    assert np.array_equal(v, v_ref)
    assert st["gn_iterations"] == st_ref["gn_iterations"] and st["pcg_iterations"] == st_ref["pcg_iterations"]
    assert st["rel_mismatch"] == st_ref["rel_mismatch"]
    assert lat > 0


def test_request_in_a_mix_equals_alone(cb):
    """A 32^3 h1s request alone, then the same request submitted among
    requests of another norm and weight (same pool), of another grid (48^3,
    its own pool, concurrent) and more requests than slots (queueing)."""
    n, nt = 32, 4
    mR, mT = sin2(n, nt)
    opt = opt_for(cb, n, nt, "h1s", 1e-2)
    with cb.Server(slots_per_pool=2, idle_ms=100) as srv:
        rid = srv.submit(opt, mR, mT)
        assert srv.wait(rid, 120000) == cb.REQ_DONE
        v_alone, st_alone, _ = srv.result(rid, (n, n, n))

    others = []
    e1 = ellipsoids(32, nt, 1)
    others.append((opt_for(cb, 32, nt, "h2s", 1e-3), e1, (32, 32, 32)))
    others.append((opt_for(cb, 32, nt, "h1", 5e-3), ellipsoids(32, nt, 2), (32, 32, 32)))
    others.append((opt_for(cb, 48, nt, "h1s", 1e-2), ellipsoids(48, nt, 3), (48, 48, 48)))
    others.append((opt_for(cb, 32, nt, "h1s", 1e-2), e1, (32, 32, 32)))
    with cb.Server(slots_per_pool=2, idle_ms=100) as srv:
        ids = [srv.submit(o, im[0], im[1]) for o, im, _ in others[:2]]
        mine = srv.submit(opt, mR, mT)          # third request of the 32^3 pool: queued behind two
        ids += [srv.submit(o, im[0], im[1]) for o, im, _ in others[2:]]
        assert srv.wait(mine, 300000) == cb.REQ_DONE
        v_mix, st_mix, _ = srv.result(mine, (n, n, n))
        results = []
        for rid, (o, im, shape) in zip(ids, others):
            assert srv.wait(rid, 300000) == cb.REQ_DONE
            results.append(srv.result(rid, shape))
    assert np.array_equal(v_mix, v_alone)
    assert st_mix["gn_iterations"] == st_alone["gn_iterations"]
    assert st_mix["pcg_iterations"] == st_alone["pcg_iterations"]
    # every other request equals its plain run too
    for (o, im, shape), (v, st, _) in zip(others, results):
        v_ref, st_ref = plain_run(cb, o, im[0], im[1])
        assert np.array_equal(v, v_ref), shape
        assert st["pcg_iterations"] == st_ref["pcg_iterations"]


def test_budget_admission_releases_idle_pools(cb):
    """A budget that holds one pool at a time: requests of a second grid wait
    until the first pool idles out and releases its memory."""
    nt = 4
    o32 = opt_for(cb, 32, nt, "h1s", 1e-2, maxit=2)
    o48 = opt_for(cb, 48, nt, "h1s", 1e-2, maxit=2)
    need32 = o32.estimate_bytes(2)
    need48 = o48.estimate_bytes(2)
    budget = max(need32, need48) + min(need32, need48) // 2
    a = sin2(32, nt)
    b = ellipsoids(48, nt, 4)
    with cb.Server(slots_per_pool=2, hbm_budget_bytes=budget, idle_ms=50) as srv:
        r1 = srv.submit(o32, *a)
        r2 = srv.submit(o48, *b)
        assert srv.wait(r1, 120000) == cb.REQ_DONE
        assert srv.wait(r2, 120000) == cb.REQ_DONE
        v1, _, _ = srv.result(r1, (32, 32, 32))
        v2, _, _ = srv.result(r2, (48, 48, 48))
        assert srv.info()["bytes_used"] <= budget
    assert np.array_equal(v1, plain_run(cb, o32, *a)[0])
    assert np.array_equal(v2, plain_run(cb, o48, *b)[0])


def test_unsupported_grid_fails_cleanly(cb):
    opt = opt_for(cb, 40, 4, "h1s", 1e-2)  # no FFT plan for 40
    mR = np.zeros((40, 40, 40), np.float32)
    with cb.Server(slots_per_pool=1, idle_ms=50) as srv:
        rid = srv.submit(opt, mR, mR)
        assert srv.wait(rid, 60000) == cb.REQ_FAILED
        with pytest.raises(cb.ClaireError):
            srv.result(rid, (40, 40, 40))


def test_scheduler_places_whole_requests(cb):
    """The multi-GPU scheduler over the devices this run has (one here): a
    request placed by it computes what the device's own server computes."""
    import torch
    from claire_b200.scheduler import Scheduler
    n, nt = 32, 4
    mR, mT = sin2(n, nt)
    o = opt_for(cb, n, nt, "h1s", 1e-2)
    with cb.Server(slots_per_pool=2) as srv:
        rid = srv.submit(o, mR, mT)
        assert srv.wait(rid, 120000) == cb.REQ_DONE
        v_ref, st_ref, _ = srv.result(rid, (n, n, n))
    devices = list(range(torch.cuda.device_count()))
    with Scheduler(devices, slots_per_pool=2) as sch:
        gids = [sch.submit(o, mR, mT) for _ in range(2 * len(devices))]
        assert sorted(sch.device_of(g) for g in gids) == sorted(devices * 2)
        for g in gids:
            assert sch.wait(g, 120000) == cb.REQ_DONE
            v, st, _ = sch.result(g, (n, n, n))
            assert st["gn_iterations"] == st_ref["gn_iterations"]
            assert np.array_equal(v, v_ref)
        assert all(x == 0 for x in sch.outstanding.values())


def test_burst_beyond_page_locked_blocks(cb):
    """A burst of requests larger than the pool's page-locked blocks (slots
    per pool 1: 2 input and 2 result blocks): the later requests arrive with
    pageable inputs that the stager moves into recycled blocks, every
    velocity comes back on the pool's copy stream, and one queued request is
    cancelled in the middle.  Each result equals the plain run of its inputs."""
    n, nt = 32, 4
    probs = [ellipsoids(n, nt, 20 + i) for i in range(6)]
    opt = opt_for(cb, n, nt, "h1s", 1e-2, maxit=2)
    refs = [plain_run(cb, opt, mR, mT) for mR, mT in probs]
    with cb.Server(slots_per_pool=1, idle_ms=200) as srv:
        ids = [srv.submit(opt, mR, mT) for mR, mT in probs]
        srv.cancel(ids[3])  # still queued behind the single slot
        for i, rid in enumerate(ids):
            st = srv.wait(rid, 300000)
            if i == 3:
                assert st == cb.REQ_CANCELLED
                with pytest.raises(cb.ClaireError):
                    srv.result(rid, (n, n, n))
                continue
            assert st == cb.REQ_DONE
            v, stats, _ = srv.result(rid, (n, n, n))
            v_ref, st_ref = refs[i]
            assert stats["gn_iterations"] == st_ref["gn_iterations"]
            assert stats["pcg_iterations"] == st_ref["pcg_iterations"]
            assert np.array_equal(v, v_ref)
