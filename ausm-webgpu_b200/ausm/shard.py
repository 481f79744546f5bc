"""Request sharding across devices (no counterpart in the reference, which runs one
grid in one browser tab).

Solves are independent, so several GPUs serve a request stream by placing whole
requests on devices; there is no data-path collective and no device reads another's
memory.  Placement is by HBM budget and work: a request goes to the device with the
least work placed on it so far (cells x steps limit), among the devices whose budget
holds the request; ties go to the lower device index, so every process that places the
same stream gets the same placement (a multi-process launch needs no communication to
agree on it).

  place_requests   static placement of a stream (one process per GPU: each rank serves
                   the requests placed on it)
  ShardedServer    one continuous-batching Server per device in one process; submit
                   places each request on the device with the least work in flight
"""
from __future__ import annotations

from .solver import Server, request_bytes, set_device


def request_work(r) -> float:
    """Work estimate of a request: cells x its step limit."""
    return float(r.M) * float(r.N) * float(r.max_steps)


def place_requests(bytes_per_request, work_per_request, n_devices: int, budget: float) -> list[int]:
    """Device index of each request, in stream order (greedy, deterministic).  Raises
    ValueError for a request whose bytes exceed the per-device budget."""
    if n_devices < 1:
        raise ValueError("need at least one device")
    load = [0.0] * n_devices
    out = []
    for k, (b, w) in enumerate(zip(bytes_per_request, work_per_request)):
        if b > budget:
            raise ValueError(f"request {k} needs {b:.3e} bytes, above the per-device budget {budget:.3e}")
        d = min(range(n_devices), key=lambda i: (load[i], i))
        load[d] += w
        out.append(d)
    return out


class ShardedServer:
    """Servers on several devices behind one submit / poll interface.  Request ids are
    (device slot, server id) pairs; a request's result does not depend on its device or
    on what else that device serves."""

    def __init__(self, devices, hbm_budget_bytes: float = 160e9, max_active: int = 256, chunk_steps: int = 100,
                 plain: bool = False):
        self.devices = list(devices)
        self.budget = float(hbm_budget_bytes)
        self.servers = []
        for d in self.devices:
            set_device(d)
            self.servers.append(Server(hbm_budget_bytes, max_active, chunk_steps, plain=plain))
        self.inflight = [0.0] * len(self.devices)  # work placed and not yet polled as done
        self._work = {}

    def start(self):
        for d, s in zip(self.devices, self.servers):
            set_device(d)  # a server's worker binds to the device current at start
            s.start()

    def submit(self, r):
        b = request_bytes(r)
        if b > self.budget:
            raise ValueError(f"request needs {b:.3e} bytes, above the per-device budget {self.budget:.3e}")
        k = min(range(len(self.servers)), key=lambda i: (self.inflight[i], i))
        set_device(self.devices[k])
        rid = self.servers[k].submit(r)
        w = request_work(r)
        self.inflight[k] += w
        self._work[(k, rid)] = w
        return (k, rid)

    def poll(self, gid, with_cp: bool = True) -> dict:
        k, rid = gid
        d = self.servers[k].poll(rid, with_cp)
        d["device"] = self.devices[k]
        if d["state"] not in (1, 2) and gid in self._work:  # finished: release its work
            self.inflight[k] -= self._work.pop(gid)
        return d

    def drain(self):
        for s in self.servers:
            s.drain()

    def stats(self) -> list[dict]:
        return [s.stats() for s in self.servers]

    def close(self):
        for d, s in zip(self.devices, self.servers):
            set_device(d)
            s.stop()
            s.close()
        self.servers = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
