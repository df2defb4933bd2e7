"""Continuous batching on the persistent whole-solve kernel.

Requests arrive over time.  Whenever one of ``streams`` CUDA streams is
free and requests are waiting, the waiting requests (at most ``max_batch``,
longest first) are packed into one persistent launch on that stream
(``ttb_amen_persistent``: one thread block per solve).  Launches on
different streams run concurrently, so the blocks of a new launch take the
SMs that finished solves of earlier launches leave idle: a short request
does not wait for the longest solve of an earlier batch.  Each launch copies
its requests' inputs from host memory on its own stream and the solutions
are read back when its completion event has fired.

Each request starts at a slot capacity chosen from its mode sizes
(``initial_rmax``); one whose bonds outgrow it (status -4) is queued again
with twice the capacity, as ``amen_persistent`` does.  Requests with mode
sizes of 64 and up run on clusters of four thread blocks (``cluster_size``),
the others on one.  A launch takes requests of one capacity and cluster
size, those of the oldest waiting request.

With ``light_streams``, requests whose estimated cost is at most
``light_cost`` (the 2-D QTT Poisson problems of the serving mix) wait in a
queue of their own and launch on streams of the highest priority, so that a
burst of long solves does not hold them back.

Requests are admitted by device memory: with ``mem_budget`` set, a launch
takes waiting requests only while the work areas (slabs) of all launches in
flight stay within the budget, so a burst of arrivals queues on the host
instead of exhausting HBM.  A request larger than the whole budget is
launched alone once nothing else is in flight.
Latency is measured per request on the host clock, from arrival to the
moment its launch is found complete.
"""

from __future__ import annotations

import time
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

import torch

from . import kernels as K
from .persistent import (PersistentBatch, Result, _cost, _Prepared, cluster_size, initial_rmax,
                         slab_doubles)


def admit(sizes: Sequence[int], room: Optional[int], idle: bool) -> List[int]:
    """Indices of the waiting requests (given oldest first, by work-area
    bytes) that one launch takes under a device-memory budget: the longest
    prefix, in arrival order, whose bytes fit in ``room`` (``room`` None: no
    budget, all of them).  The first request that does not fit stops the
    launch, so later, smaller arrivals never overtake it and an old large
    request cannot starve.  When none fits and nothing is in flight
    (``idle``), the oldest is taken alone, so a request larger than the
    whole budget still runs."""
    if room is None:
        return list(range(len(sizes)))
    out, used = [], 0
    for i, b in enumerate(sizes):
        if used + b > room:
            break
        out.append(i)
        used += b
    if not out and idle and sizes:
        out = [0]
    return out


@dataclass
class Job:
    rid: int
    arrival: float
    prep: _Prepared
    rmax: int
    cluster: int = 1  # thread blocks of its solve
    lane: int = 1     # 0: light requests (own queue, high-priority streams), 1: the rest
    result: Optional[Result] = None
    slab_bytes: int = 0  # work area at the current slot capacity
    done_at: Optional[float] = None
    host_cores: Optional[list] = None  # the solution's cores read back to the host

    @property
    def latency(self) -> Optional[float]:
        return None if self.done_at is None else self.done_at - self.arrival


class PersistentServer:
    """Serve AMEn requests with concurrent persistent launches.

    ``streams`` bounds the launches in flight, ``max_batch`` the requests of
    one launch; a launch is issued at most every ``min_interval`` seconds
    unless ``max_batch`` requests are waiting, so arrivals in a burst share
    a launch.
    """

    def __init__(self, streams: int = 16, max_batch: int = 1024, rmax: Optional[int] = None,
                 max_rmax: int = 256, min_interval: float = 0.005, download: bool = True,
                 mem_budget: Optional[int] = None, resident: bool = False,
                 cluster_for: Optional[Callable[[_Prepared], int]] = cluster_size,
                 time_limit: Optional[float] = None, light_streams: int = 0,
                 light_cost: float = 1e5):
        K.device_ok()
        # lane 1: ``streams`` streams of normal priority; lane 0 (with
        # ``light_streams``): requests of estimated cost at most
        # ``light_cost`` in their own queue, launched on streams of the
        # highest priority, so the block scheduler gives them the next free
        # SMs instead of leaving them behind long solves
        # (a priority beyond the device's range maps to its highest)
        self.streams = ([torch.cuda.Stream(priority=-10) for _ in range(light_streams)]
                        + [torch.cuda.Stream() for _ in range(streams)])
        self.lane_of = [0] * light_streams + [1] * streams
        self.free = {0: list(range(light_streams)),
                     1: list(range(light_streams, light_streams + streams))}
        self.light_cost = light_cost if light_streams > 0 else -1.0
        self.max_batch = max_batch
        self.rmax = rmax
        self.max_rmax = max_rmax
        self.min_interval = min_interval
        self.download = download
        self.mem_budget = mem_budget
        self.resident = resident  # inputs uploaded before submission (no copy per launch)
        self.cluster_for = cluster_for  # thread blocks per solve (None: one)
        self.time_limit = time_limit    # per-solve device-time limit (s), status -6 past it
        self.inflight_bytes = 0
        self.peak_bytes = 0
        self.queues = {0: [], 1: []}  # waiting requests per lane, oldest first
        self.inflight = []  # (stream index, batch, event, jobs, slab bytes)
        self.completed: List[Job] = []
        self.launches = 0
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        self._last_launch = {0: -1e30, 1: -1e30}

    def submit(self, rid: int, arrival: float, A, b, x0=None, kwargs: Optional[dict] = None) -> Job:
        """Validate a request on the host and queue it (``amen`` arguments)."""
        return self.submit_prepared(rid, arrival, _Prepared(A, b, x0, dict(kwargs or {})))

    def submit_prepared(self, rid: int, arrival: float, prep: _Prepared) -> Job:
        """Queue an already validated request; it starts at the server's
        slot capacity, or at ``initial_rmax`` for its mode sizes."""
        job = Job(rid, arrival, prep, self.rmax or initial_rmax(prep),
                  self.cluster_for(prep) if self.cluster_for else 1,
                  0 if _cost(prep) <= self.light_cost else 1)
        job.slab_bytes = 8 * slab_doubles(job.prep, job.rmax)
        self.queues[job.lane].append(job)
        return job

    @property
    def queue(self) -> List[Job]:
        """Every waiting request (both lanes)."""
        return self.queues[0] + self.queues[1]

    def _launch(self, now: float) -> bool:
        return any([self._launch_lane(lane, now) for lane in (0, 1)])

    def _launch_lane(self, lane: int, now: float) -> bool:
        queue, free = self.queues[lane], self.free[lane]
        if not queue or not free:
            return False
        if len(queue) < self.max_batch and now - self._last_launch[lane] < self.min_interval:
            return False
        # one slot capacity per launch: the oldest waiting request's, so that
        # requests of every capacity are launched in arrival order
        rmax, cl = queue[0].rmax, queue[0].cluster
        take = [j for j in queue if j.rmax == rmax and j.cluster == cl][: self.max_batch]
        room = None if self.mem_budget is None else self.mem_budget - self.inflight_bytes
        idx = admit([j.slab_bytes for j in take], room, not self.inflight)
        if not idx:
            return False
        take = [take[i] for i in idx]
        taken = set(id(j) for j in take)
        self.queues[lane] = [j for j in queue if id(j) not in taken]
        take.sort(key=lambda j: -_cost(j.prep))
        si = free.pop()
        s = self.streams[si]
        with torch.cuda.stream(s):
            batch = PersistentBatch([j.prep for j in take], rmax, resident=self.resident,
                                    cluster=cl, time_limit=self.time_limit)
            batch.launch(s)
            ev = torch.cuda.Event()
            ev.record(s)
        self.h2d_bytes += batch.h2d_bytes
        nbytes = sum(j.slab_bytes for j in take)
        self.inflight_bytes += nbytes
        self.peak_bytes = max(self.peak_bytes, self.inflight_bytes)
        self.inflight.append((si, batch, ev, take, nbytes))
        self.launches += 1
        self._last_launch[lane] = now
        return True

    def _collect(self, now: float) -> bool:
        done_any = False
        still = []
        for si, batch, ev, jobs, nbytes in self.inflight:
            if not ev.query():
                still.append((si, batch, ev, jobs, nbytes))
                continue
            done_any = True
            self.inflight_bytes -= nbytes
            with torch.cuda.stream(self.streams[si]):
                results = batch.collect()
                for job, res in zip(jobs, results):
                    if res.status == -4 and job.rmax < self.max_rmax:
                        job.rmax = min(2 * job.rmax, self.max_rmax)
                        job.slab_bytes = 8 * slab_doubles(job.prep, job.rmax)
                        self.queues[job.lane].append(job)
                        continue
                    job.result = res
                    if self.download and res.x is not None:
                        job.host_cores = res.x.to_numpy()
                        self.d2h_bytes += sum(c.nbytes for c in job.host_cores)
                    job.done_at = now
                    self.completed.append(job)
            batch.release()
            self.free[self.lane_of[si]].append(si)
        self.inflight = still
        return done_any

    def step(self, now: float) -> bool:
        """Collect finished launches, then issue new ones; True if anything
        happened."""
        a = self._collect(now)
        b = False
        while self._launch(now):
            b = True
        return a or b

    def idle(self) -> bool:
        return not self.queues[0] and not self.queues[1] and not self.inflight

    def serve(self, requests: Sequence, arrivals: Sequence[float],
              clock: Callable[[], float] = time.perf_counter) -> List[Job]:
        """Submit ``requests`` [(A, b, x0, kwargs)], or requests already
        prepared (``_Prepared``), at ``arrivals`` (seconds from the start) and
        serve them to completion; returns the jobs in request order.
        Requests arriving at the same time are queued in the order given."""
        order = sorted(range(len(requests)), key=lambda i: arrivals[i])
        jobs: List[Optional[Job]] = [None] * len(requests)
        t0 = clock()
        nxt = 0
        while nxt < len(order) or not self.idle():
            now = clock() - t0
            while nxt < len(order) and arrivals[order[nxt]] <= now:
                i = order[nxt]
                if isinstance(requests[i], _Prepared):
                    jobs[i] = self.submit_prepared(i, arrivals[i], requests[i])
                else:
                    A, b, x0, kw = requests[i]
                    jobs[i] = self.submit(i, arrivals[i], A, b, x0, kw)
                nxt += 1
            if not self.step(clock() - t0):
                time.sleep(0.0005)
        return jobs
