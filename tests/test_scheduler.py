"""Host-side placement of whole registrations on GPUs (claire_b200.scheduler).

Runs without a GPU: fake per-device servers record what they receive.  The
placement rule is footprint-aware least-loaded: a request goes to the device
whose outstanding footprint, with the request added, is the smallest share of
that device's budget.
"""
import pytest

from claire_b200.scheduler import Scheduler


class FakeServer:
    def __init__(self, dev):
        self.dev = dev
        self.got = []
        self.cancelled = []
        self.closed = False

    def submit(self, opt, mR, mT):
        self.got.append(opt)
        return len(self.got)

    def poll(self, rid):
        return 2

    def wait(self, rid, timeout_ms=-1):
        return 2

    def result(self, rid, shape):
        return ("v", {"dev": self.dev, "rid": rid}, 1.0)

    def cancel(self, rid):
        self.cancelled.append(rid)

    def close(self):
        self.closed = True


def make(devices, budget=1000):
    return Scheduler(devices, hbm_budget_bytes=budget, server_factory=FakeServer, footprint=lambda opt: opt)


def test_equal_requests_spread_round_robin():
    s = make([0, 1, 2, 3])
    ids = [s.submit(100, None, None) for _ in range(8)]
    assert [s.device_of(i) for i in ids] == [0, 1, 2, 3, 0, 1, 2, 3]
    assert all(s.outstanding[d] == 200 for d in range(4))


def test_footprint_aware_placement():
    s = make([0, 1])
    big = s.submit(600, None, None)       # -> 0
    small = [s.submit(100, None, None) for _ in range(5)]
    assert s.device_of(big) == 0
    # device 1 takes the small ones until its share passes device 0's
    assert [s.device_of(i) for i in small] == [1, 1, 1, 1, 1]
    assert s.outstanding == {0: 600, 1: 500}
    assert s.device_of(s.submit(100, None, None)) == 1  # 0.7 on 0 vs 0.6 on 1


def test_release_on_result_and_forwarding():
    s = make([0, 1])
    a = s.submit(300, None, None)
    b = s.submit(300, None, None)
    v, st, lat = s.result(a, (4, 4, 4))
    assert st["dev"] == 0 and s.outstanding[0] == 0
    s.cancel(b)
    assert s.servers[1].cancelled == [1]
    assert s.poll(b) == 2 and s.wait(b) == 2
    s.close()


def test_budgets_per_device():
    s = make([0, 1], budget=0)
    s.budget = {0: 1000, 1: 4000}
    placed = [s.device_of(s.submit(500, None, None)) for _ in range(5)]
    # device 1 has four times the room: it takes four of the five
    assert placed.count(1) == 4 and placed.count(0) == 1


def test_needs_a_device():
    with pytest.raises(ValueError):
        Scheduler([], server_factory=FakeServer)
