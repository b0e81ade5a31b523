"""Scheduling logic of the serving loop, on the CPU with a stand-in batch.

The stand-in keeps per-slot step budgets like the device does (a chunk of
K steps advances every slot with budget left by min(K, left)) and refuses
admissions beyond its slot count, so admission, retirement, memory
accounting and the continuous-batching order can be checked without a GPU.
"""
import dataclasses

import pytest

from gpluto_dev_b200 import api, serve


@dataclasses.dataclass
class FakeState:
    ndim: int
    ncells: int


class FakeBatch:
    def __init__(self, max_slots):
        self.max_slots = max_slots
        self.left = {}
        self.done = {}
        self.advances = []

    def add(self, st, scheme, dt0, nsteps, shape=None):
        free = [s for s in range(self.max_slots) if s not in self.left]
        if not free:
            raise api.GPError(-4, "slot table full")
        s = free[0]
        self.left[s], self.done[s] = nsteps, 0
        return s

    def status(self, slot):
        from gpluto_dev_b200.batch import SlotStatus
        return SlotStatus(self.done[slot], self.left[slot], 0, 1e-4, 0.0)

    def remove(self, slot):
        del self.left[slot]
        del self.done[slot]

    def advance(self, k):
        self.advances.append(sorted(self.left))
        for s in self.left:
            d = min(k, self.left[s])
            self.left[s] -= d
            self.done[s] += d

    def wait(self):
        pass

    def download(self, slot):
        return ("state", slot, self.done[slot])


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.01          # every clock read advances 10 ms
        return self.t

    def sleep(self, dt):
        self.t += dt


def job(rid, arrival, cells, nsteps, ndim=2):
    return serve.Job(rid, arrival, FakeState(ndim, cells), api.Scheme(), nsteps)


def make_server(pool, slots=8, chunk=5, keep=False):
    clk = FakeClock()
    srv = serve.Server(pool_bytes=pool, max_slots=slots, chunk=chunk, batch=FakeBatch(slots),
                       slot_bytes=lambda st, sch: st.ncells * 100, clock=clk, keep_results=keep)
    return srv, clk


def test_every_request_runs_exactly_its_steps():
    srv, clk = make_server(pool=10 ** 9, keep=True)
    jobs = [job(i, 0.05 * i, 1000 * (i + 1), 3 + 4 * i) for i in range(6)]
    done = srv.serve(jobs, sleep=clk.sleep)
    assert sorted(j.rid for j in done) == list(range(6))
    for j in done:
        assert j.status.steps_done == j.nsteps
        assert j.result[2] == j.nsteps
        assert j.finished >= j.admitted >= j.arrival >= 0
    assert srv.used_bytes == 0 and not srv.active and not srv.pending


def test_late_arrivals_join_the_running_mix():
    """A request arriving while a long one runs is admitted before the long
    one finishes (continuous batching, not a queue)."""
    srv, clk = make_server(pool=10 ** 9, chunk=2)
    long_job = job(0, 0.0, 1000, 40)
    short = job(1, 0.1, 1000, 4)
    srv.serve([long_job, short], sleep=clk.sleep)
    assert short.admitted < long_job.finished
    assert short.finished < long_job.finished
    both = [a for a in srv.batch.advances if len(a) == 2]
    assert both, "the two requests never shared a chunk"


def test_memory_budget_and_skip_ahead():
    """The pool holds 3000 cells' worth; a big request waits while smaller
    ones behind it that fit are admitted; nothing exceeds the budget."""
    srv, clk = make_server(pool=3000 * 100, chunk=3)
    a = job(0, 0.0, 2000, 9)
    big = job(1, 0.0, 2500, 3)      # does not fit while a runs
    small = job(2, 0.0, 800, 3)     # fits beside a
    peak = []
    orig_round = srv.round

    def round_and_check():
        orig_round()
        peak.append(srv.used_bytes)
        assert srv.used_bytes <= srv.pool_bytes
    srv.round = round_and_check
    srv.serve([a, big, small], sleep=clk.sleep)
    assert small.admitted < big.admitted
    assert big.admitted >= a.finished
    assert max(peak) <= 3000 * 100
    assert max(d[1] for d in srv.depth) >= 1      # the big one waited


def test_request_larger_than_pool_is_reported():
    srv, clk = make_server(pool=1000)
    with pytest.raises(RuntimeError):
        srv.serve([job(0, 0.0, 50, 3)], sleep=clk.sleep)


def test_percentiles_and_summary():
    assert serve.percentile([1, 2, 3, 4], 50) == 2.5
    assert serve.percentile([5], 99) == 5
    srv, clk = make_server(pool=10 ** 9)
    jobs = [job(i, 0.02 * i, 500, 5) for i in range(4)]
    done = srv.serve(jobs, sleep=clk.sleep)
    s = serve.summary(done, srv.depth, makespan=1.0)
    assert s["requests"] == 4 and s["p99_s"] >= s["p50_s"] > 0
    assert s["Mzone_updates_per_s"] == pytest.approx(4 * 500 * 5 / 1e6)
