"""Serving loop: continuous batching of AMEn solve requests on one GPU.

Requests are admitted into the :class:`~ttnumpy_b200.batched.BatchEngine`
as they arrive, as long as the device has memory for them (free HBM from
the CUDA driver, minus a reserve), and leave it as they finish; admitted
solves keep their cores and environments resident on the device and
advance together, one grouped operation per tick.  Latency is measured per
request from arrival to completion on the host clock.
"""

from __future__ import annotations

import heapq
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import torch

from .batched import BatchEngine, SolveState


def estimate_bytes(A, b, max_rank: int = 64) -> int:
    """Device memory a solve may hold: cores of x and z at ``max_rank``,
    the five environment families, and the largest local system's work
    (Krylov vectors and the operator's intermediates)."""
    d = len(A)
    n = max(A.row_modes)
    R = max(A.bonds)
    r = max_rank
    cores = d * r * n * r * 8 * 3
    envs = d * (2 * r * R * r + 3 * r * r) * 8 * 2
    local = (12 * r * n * r + 2 * r * n * R * r) * 8
    return int(cores + envs + local)


@dataclass(order=True)
class Request:
    arrival: float
    rid: int
    A: object = field(compare=False)
    b: object = field(compare=False)
    x0: object = field(compare=False, default=None)
    kwargs: dict = field(compare=False, default_factory=dict)
    state: Optional[SolveState] = field(compare=False, default=None)
    done_at: Optional[float] = field(compare=False, default=None)


class Server:
    """Continuous-batching AMEn server on the current CUDA device.

    ``reserve_bytes`` of device memory are never handed to requests;
    ``max_active`` caps the number of concurrently admitted solves.
    """

    def __init__(self, reserve_bytes: int = 4 << 30, max_active: int = 512,
                 rank_guess: int = 64):
        self.engine = BatchEngine()
        self.reserve = reserve_bytes
        self.max_active = max_active
        self.rank_guess = rank_guess
        self.waiting: List[Request] = []
        self.admitted: List[Request] = []
        self.completed: List[Request] = []
        self.held = 0

    def submit(self, req: Request) -> None:
        heapq.heappush(self.waiting, req)

    def _can_admit(self, need: int) -> bool:
        if len(self.engine.active) >= self.max_active:
            return False
        free, _ = torch.cuda.mem_get_info()
        cached = torch.cuda.memory_reserved() - torch.cuda.memory_allocated()
        return free + cached - self.reserve - self.held >= need or not self.engine.active

    def step(self, now: float) -> List[Request]:
        """Admit what has arrived and fits, run one tick, retire finished
        requests; returns the requests that finished in this tick."""
        while self.waiting and self.waiting[0].arrival <= now:
            req = self.waiting[0]
            need = estimate_bytes(req.A, req.b, self.rank_guess)
            if not self._can_admit(need):
                break
            heapq.heappop(self.waiting)
            req.state = self.engine.admit(req.A, req.b, req.x0, rid=req.rid, **req.kwargs)
            req.need = need
            self.held += need
            self.admitted.append(req)
        if not self.engine.active:
            return []
        finished = self.engine.tick()
        out = []
        if finished:
            t = time.perf_counter()
            ids = {id(s) for s in finished}
            keep = []
            for req in self.admitted:
                if id(req.state) in ids:
                    req.done_at = t
                    self.held -= req.need
                    out.append(req)
                else:
                    keep.append(req)
            self.admitted = keep
            self.completed.extend(out)
        return out

    def idle(self) -> bool:
        return not self.waiting and not self.engine.active

    def run(self, clock: Callable[[], float] = time.perf_counter) -> List[Request]:
        """Serve until every submitted request finished.  Arrival times are
        on ``clock``; the loop sleeps only when nothing is admitted."""
        while not self.idle():
            now = clock()
            self.step(now)
            if not self.engine.active and self.waiting:
                delay = self.waiting[0].arrival - clock()
                if delay > 0:
                    time.sleep(min(delay, 0.01))
        return self.completed


def serve_batch(dev_reqs: Sequence, kwargs_fn: Callable, download: bool = False):
    """Admit every ``(A, b, x0, problem)`` at once and serve them to
    completion; returns ``([(x, info)], latencies_ms)`` in request order."""
    srv = Server()
    t0 = time.perf_counter()
    reqs = []
    for i, (A, b, x0, p) in enumerate(dev_reqs):
        r = Request(t0, i, A, b, x0, kwargs_fn(p))
        srv.submit(r)
        reqs.append(r)
    srv.run()
    results, lat = [], []
    for r in reqs:
        s = r.state
        if s.error is not None:
            raise s.error
        x = s.x
        if download:
            x.to_numpy()
        results.append((x, s.info))
        lat.append(1e3 * (r.done_at - r.arrival))
    return results, lat
