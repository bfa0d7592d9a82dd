"""Multi-GPU request scheduler: whole registrations placed on GPUs by HBM footprint.

A registration does not shard across GPUs (the reference's MPI pencil
decomposition is out of scope), but independent registrations do: this host
scheduler keeps one registration server (claire_b200_server, continuous
batching) per device and places each request, whole, on the device whose
outstanding footprint (the claire_b200_estimate_bytes of its queued and
running requests) is smallest relative to that device's budget.  There is no
collective on the data path: images go to one device and the velocity comes
back from it.  The reference has no counterpart (one CLAIREInterface::Run,
src/CLAIREInterface.cpp:709-885, per process and problem).

``server_factory(device)`` builds a server for one device; it defaults to
``claire_b200.Server``, and tests substitute a fake to check the placement on
a host without GPUs.
"""
from __future__ import annotations

import threading
from typing import Callable, Dict, Optional, Sequence, Tuple


class Scheduler:
    def __init__(self, devices: Sequence[int], slots_per_pool: int = 4, hbm_budget_bytes: int = 0,
                 idle_ms: int = 2000, server_factory: Optional[Callable[[int], object]] = None,
                 footprint: Optional[Callable[[object], int]] = None):
        if not devices:
            raise ValueError("at least one device")
        if server_factory is None:
            import claire_b200 as cb

            def server_factory(dev):
                return cb.Server(slots_per_pool=slots_per_pool, hbm_budget_bytes=hbm_budget_bytes,
                                 idle_ms=idle_ms, device=dev)
        # bytes one request of these options needs on a device (a pool's share)
        self._footprint = footprint or (lambda opt: int(opt.estimate_bytes(1)))
        self.devices = list(devices)
        self.servers = {d: server_factory(d) for d in self.devices}
        self.budget = {d: (hbm_budget_bytes or self._device_budget(d)) for d in self.devices}
        self.outstanding: Dict[int, int] = {d: 0 for d in self.devices}
        self._req: Dict[int, Tuple[int, int, int]] = {}  # global id -> (device, server id, bytes)
        self._next = 1
        self._lock = threading.Lock()

    def _device_budget(self, dev: int) -> int:
        try:
            import torch
            free, _ = torch.cuda.mem_get_info(dev)
            return int(0.9 * free)
        except Exception:
            return 1 << 40

    def place(self, nbytes: int) -> int:
        """Device for a request of nbytes: smallest outstanding share of the
        budget after adding it (ties: the first listed device)."""
        return min(self.devices, key=lambda d: ((self.outstanding[d] + nbytes) / max(1, self.budget[d]),
                                                self.devices.index(d)))

    def submit(self, opt, mR, mT) -> int:
        nbytes = self._footprint(opt)
        with self._lock:
            dev = self.place(nbytes)
            rid = self.servers[dev].submit(opt, mR, mT)
            gid = self._next
            self._next += 1
            self._req[gid] = (dev, rid, nbytes)
            self.outstanding[dev] += nbytes
        return gid

    def device_of(self, gid: int) -> int:
        return self._req[gid][0]

    def poll(self, gid: int) -> int:
        dev, rid, _ = self._req[gid]
        return self.servers[dev].poll(rid)

    def wait(self, gid: int, timeout_ms: int = -1) -> int:
        dev, rid, _ = self._req[gid]
        return self.servers[dev].wait(rid, timeout_ms)

    def _release(self, gid: int):
        with self._lock:
            dev, _, nbytes = self._req.pop(gid)
            self.outstanding[dev] -= nbytes

    def result(self, gid: int, shape):
        """(velocity, stats, latency ms) from the request's device; releases it."""
        dev, rid, _ = self._req[gid]
        try:
            return self.servers[dev].result(rid, shape)
        finally:
            self._release(gid)

    def cancel(self, gid: int) -> None:
        dev, rid, _ = self._req[gid]
        self.servers[dev].cancel(rid)

    def close(self):
        for s in self.servers.values():
            s.close()
        self.servers = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
