"""Serving loop: continuous batching of solve requests on one GPU.

Requests (a grid, a scheme, a first dt and a step count) arrive over time.
The server keeps every admitted request's state resident in one device pool
(:class:`gpluto_dev_b200.batch.Batch`) and advances all of them together in
chunks of ``chunk`` steps -- per RK stage one persistent sweep launch and
one persistent EMF/finish launch over all active requests, replayed from a
captured CUDA graph.  Between chunks it

1. retires requests whose step budget is spent (downloads the result, frees
   the slot and its pool space),
2. admits waiting requests while slots and pool memory are free -- first
   come first served, but a request that does not fit does not block
   smaller ones behind it -- so that requests arriving while others are on
   the GPU join the running mix at the next chunk,
3. records the queue depth.

Each request advances exactly as it would alone (every slot has its own dt
sequence and budget; the kernels do not mix slots), so its result does not
depend on what else is in the mix.  Latency = completion time - arrival
time, on the host clock.
"""
from __future__ import annotations

import collections
import dataclasses
import time

from . import api, autotune
from . import batch as gb


@dataclasses.dataclass
class Job:
    rid: int
    arrival: float
    state: object           # ics.PrimState
    scheme: api.Scheme
    nsteps: int
    dt0: float = 1e-4
    # filled in by the server
    slot: int = -1
    admitted: float = -1.0
    finished: float = -1.0
    result: tuple = None    # (V, U, Bs) after nsteps
    status: object = None   # batch.SlotStatus at retirement

    @property
    def cells(self) -> int:
        return int(self.state.ncells)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Server:
    """Continuous-batching server over one device pool.

    ``batch`` may be given (tests pass a stand-in); otherwise a
    :class:`~gpluto_dev_b200.batch.Batch` of ``pool_bytes`` with
    ``max_slots`` slots is created.  ``table`` is an autotuner table (tile
    shapes per size bin).  ``keep_results`` downloads every finished state.
    """

    def __init__(self, pool_bytes: int = 150 * 10 ** 9, max_slots: int = 1024, chunk: int = 25,
                 table: dict | None = None, batch=None, slot_bytes=None, clock=None,
                 keep_results: bool = False, stream=None):
        self.batch = batch if batch is not None else gb.Batch(pool_bytes, max_slots, stream=stream)
        self.slot_bytes = slot_bytes or gb.slot_bytes
        self.pool_bytes = pool_bytes
        self.max_slots = max_slots
        self.chunk = chunk
        self.table = table or autotune.default_table()
        self.clock = clock or time.perf_counter
        self.keep_results = keep_results
        self.pending = collections.deque()
        self.active = {}          # slot -> Job
        self.done = []
        self.used_bytes = 0
        self.depth = []           # (time, pending, active) per scheduling round
        self.zone_updates = 0

    # -- bookkeeping --------------------------------------------------------
    def submit(self, job: Job):
        self.pending.append(job)

    def _fits(self, job: Job) -> bool:
        return (len(self.active) < self.max_slots and
                self.used_bytes + self.slot_bytes(job.state, job.scheme) <= self.pool_bytes)

    def admit(self, now: float) -> int:
        """Admit waiting jobs that fit; returns how many were admitted."""
        n = 0
        keep = collections.deque()
        while self.pending:
            job = self.pending.popleft()
            if not self._fits(job):
                keep.append(job)
                continue
            shape = autotune.shape_for(self.table, job.state.ndim, job.cells)
            try:
                job.slot = self.batch.add(job.state, job.scheme, job.dt0, job.nsteps, shape)
            except api.GPError as e:
                if e.code == -4:          # pool fragmented or full: retry later
                    keep.append(job)
                    continue
                raise
            job.admitted = now
            self.used_bytes += self.slot_bytes(job.state, job.scheme)
            self.active[job.slot] = job
            n += 1
        self.pending = keep
        return n

    def retire(self, now: float) -> int:
        n = 0
        for slot in list(self.active):
            st = self.batch.status(slot)
            if st.steps_left > 0:
                continue
            job = self.active.pop(slot)
            job.status = st
            if self.keep_results:
                job.result = self.batch.download(slot)
            self.batch.remove(slot)
            self.used_bytes -= self.slot_bytes(job.state, job.scheme)
            self.zone_updates += job.cells * st.steps_done
            job.finished = now
            self.done.append(job)
            n += 1
        return n

    def round(self):
        """One scheduling round: admit, run one chunk, retire."""
        self.admit(self.clock())
        self.depth.append((self.clock(), len(self.pending), len(self.active)))
        if self.active:
            self.batch.advance(self.chunk)
            self.batch.wait()
        self.retire(self.clock())

    # -- a stream of timed arrivals -----------------------------------------
    def serve(self, jobs, t0: float | None = None, sleep=time.sleep):
        """Serve ``jobs`` (Job.arrival in seconds after t0) until all finish.

        Returns the finished jobs in completion order."""
        future = collections.deque(sorted(jobs, key=lambda j: j.arrival))
        t0 = self.clock() if t0 is None else t0
        for j in future:
            j.arrival += t0
        while future or self.pending or self.active:
            now = self.clock()
            while future and future[0].arrival <= now:
                self.submit(future.popleft())
            if not self.pending and not self.active:
                if future:
                    sleep(max(0.0, future[0].arrival - self.clock()))
                continue
            before = len(self.active)
            self.round()
            if before == 0 and not self.active and self.pending:
                raise RuntimeError("a waiting request can never be admitted (larger than the pool)")
        for j in jobs:
            j.arrival -= t0
            j.finished -= t0
            if j.admitted >= 0:
                j.admitted -= t0
        return self.done

    def close(self):
        if hasattr(self.batch, "close"):
            self.batch.close()


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return float("nan")
    k = (len(xs) - 1) * q / 100.0
    f = int(k)
    c = min(f + 1, len(xs) - 1)
    return xs[f] + (xs[c] - xs[f]) * (k - f)


def summary(jobs, depth, makespan: float) -> dict:
    lat = [j.latency for j in jobs]
    zu = sum(j.cells * j.nsteps for j in jobs)
    return {"requests": len(jobs), "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99),
            "mean_s": sum(lat) / max(1, len(lat)), "makespan_s": makespan,
            "Mzone_updates_per_s": zu / makespan / 1e6,
            "queue_depth_mean": sum(d[1] for d in depth) / max(1, len(depth)),
            "queue_depth_max": max((d[1] for d in depth), default=0),
            "active_mean": sum(d[2] for d in depth) / max(1, len(depth))}
