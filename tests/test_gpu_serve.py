"""Serving loop on the GPU: requests of different physics, dimensionality,
size, step count and precision arrive while others run, share the device
in the same launches, and each result is the same as the request run alone.

Tolerance: none.  A request alone in the batch and the same request in the
mix run the same code on the same slot data, so the results must be
bit-identical in both precision forms; FP64 requests must also be
bit-identical to the single-grid entry point (Solver.run).
"""
import numpy as np
import pytest

from gpluto_dev_b200 import api, ics, serve
from gpluto_dev_b200 import batch as gb
from gpluto_dev_b200.workloads import scheme_for

pytestmark = pytest.mark.gpu


def make_jobs():
    spec = [  # (physics, shape, nsteps, precision, arrival s)
        (api.MHD, (48, 40), 37, api.FP64, 0.000),
        (api.HD, (12, 10, 8), 9, api.MIXED, 0.000),
        (api.MHD, (16, 12, 10), 12, api.FP64, 0.000),
        (api.HD, (40, 40), 25, api.FP64, 0.001),
        (api.MHD, (32, 64), 6, api.MIXED, 0.002),
        (api.MHD, (10, 10, 10), 21, api.MIXED, 0.003),
        (api.HD, (64, 20), 4, api.FP64, 0.004),
        (api.MHD, (24, 24), 30, api.FP64, 0.005),
        (api.HD, (14, 14, 14), 7, api.FP64, 0.006),
        (api.MHD, (20, 16, 12), 11, api.FP64, 0.007),
    ]
    jobs = []
    for i, (phys, shape, n, prec, t) in enumerate(spec):
        if phys == api.MHD:
            st = (ics.mhd2d_turbulence(n=shape, seed=900 + i) if len(shape) == 2
                  else ics.mhd3d_turbulence(n=shape, seed=900 + i))
        else:
            st = ics.hd_turbulence(n=shape, seed=900 + i)
        jobs.append(serve.Job(i, t, st, scheme_for(phys, prec, st.gamma), n))
    return jobs


def alone_in_batch(job):
    b = gb.Batch(gb.slot_bytes(job.state, job.scheme) + (1 << 20), 1)
    s = b.add(job.state, job.scheme, job.dt0, job.nsteps)
    b.advance(job.nsteps)
    b.wait()
    out = b.download(s), b.status(s)
    b.close()
    return out


def same(a, b):
    Va, Ua, Ba = a
    Vb, Ub, Bb = b
    return (np.array_equal(Va, Vb) and np.array_equal(Ua, Ub) and len(Ba) == len(Bb)
            and all(np.array_equal(x, y) for x, y in zip(Ba, Bb)))


def test_results_are_the_same_alone_and_in_the_mix():
    jobs = make_jobs()
    srv = serve.Server(pool_bytes=1 << 30, max_slots=6, chunk=2, keep_results=True)
    done = srv.serve(jobs)
    srv.close()
    assert len(done) == len(jobs)
    # requests shared the device: several were active in one chunk, and a
    # request was admitted while an earlier one was still running
    assert max(d[2] for d in srv.depth) >= 3
    assert any(a.admitted < b.admitted < a.finished for a in done for b in done)
    for j in done:
        assert j.status.steps_done == j.nsteps, j.rid
        ref, st = alone_in_batch(j)
        assert st.steps_done == j.nsteps
        assert st.dt == j.status.dt, j.rid
        assert same(j.result, ref), f"request {j.rid} differs alone vs in the mix"
        if j.scheme.precision == api.FP64:
            s = api.Solver.from_state(j.state, j.scheme)
            s.run(j.nsteps, j.dt0)
            assert same(j.result, s.download()), f"request {j.rid} differs from Solver.run"
            s.close()


def test_pool_budget_limits_admission():
    """A pool that holds two of these grids never runs more than two."""
    st = ics.mhd2d_turbulence(n=(64, 64), seed=950)
    sch = scheme_for(api.MHD, api.FP64, st.gamma)
    per = gb.slot_bytes(st, sch)
    srv = serve.Server(pool_bytes=2 * per + 4096, max_slots=8, chunk=3)
    jobs = [serve.Job(i, 0.0, st, sch, 6) for i in range(5)]
    done = srv.serve(jobs)
    srv.close()
    assert len(done) == 5
    assert max(d[2] for d in srv.depth) == 2
    assert max(d[1] for d in srv.depth) >= 3
