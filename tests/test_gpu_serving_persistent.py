"""Continuous batching on the persistent kernel (``PersistentServer``).

* Requests arriving over time are served by concurrent launches; every
  solve converges and meets its tolerance (checked by the host oracle).
* A solve's result does not depend on which launch it lands in or what it
  shares the GPU with: the served cores are bit-identical to the same
  request solved alone in one launch.
"""

import numpy as np
import pytest

from oracle import tt_oracle as O
from ttnumpy_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def srv_mod():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ttnumpy_b200 import persistent, persistent_serving

    return persistent, persistent_serving


KW = dict(residual_tol=1e-8, symmetric=True, max_sweeps=20, seed=0, stagnation_factor=None)


def _problems():
    rng = np.random.default_rng(3)
    out = []
    for i in range(10):
        if i % 2 == 0:
            out.append(P.qtt_poisson_2d(3 + i // 2))
        else:
            out.append(P.parametric_diffusion(4, 16, rng.uniform(-1, 1, size=4)))
    return out


@pytest.mark.parametrize("light_streams", [0, 2])
def test_staggered_arrivals_match_alone(srv_mod, light_streams):
    """With light_streams, the QTT requests (the light ones) are served from
    their own queue on high-priority streams; results are the same either
    way."""
    pers, ps = srv_mod
    probs = _problems()
    reqs = [(p.A, p.b, None, KW) for p in probs]
    arrivals = [0.0, 0.0, 0.01, 0.02, 0.02, 0.05, 0.08, 0.08, 0.12, 0.2]
    server = ps.PersistentServer(streams=4, min_interval=0.002, light_streams=light_streams)
    jobs = server.serve(reqs, arrivals)
    assert server.launches >= 2
    lanes = [j.lane for j in jobs]
    if light_streams:
        assert lanes == [0 if i % 2 == 0 else 1 for i in range(len(jobs))]
    else:
        assert set(lanes) == {1}
    for p, job in zip(probs, jobs):
        res = job.result
        assert res.status == 0 and res.info.converged, (p.name, res.info)
        assert job.latency is not None and job.latency >= 0.0
        host = O.relative_residual(O.Train(p.A), O.Train(p.b), O.Train(job.host_cores))
        assert host <= 1.05e-8, (p.name, host)
        (alone,) = pers.amen_persistent([(p.A, p.b, None, KW)])
        assert alone.info.residuals == res.info.residuals, p.name
        assert all(np.array_equal(u, v) for u, v in zip(alone.x.to_numpy(), job.host_cores))


def test_memory_budget_admission(srv_mod):
    """With a device-memory budget the server never holds more slab bytes
    in flight than the budget (a request larger than the budget runs alone),
    and the results are those of the unconstrained server."""
    pers, ps = srv_mod
    probs = _problems()
    reqs = [(p.A, p.b, None, KW) for p in probs]
    arrivals = [0.0] * len(reqs)  # one burst: everything queued at once
    sizes = [8 * pers.slab_doubles(pers.prepare([r])[0], 64) for r in reqs]
    budget = 2 * max(sizes)
    server = ps.PersistentServer(streams=4, min_interval=0.0, mem_budget=budget)
    jobs = server.serve(reqs, arrivals)
    assert server.peak_bytes <= budget
    assert server.launches >= 2  # the burst did not fit in one launch
    free = ps.PersistentServer(streams=4, min_interval=0.0).serve(reqs, arrivals)
    for p, a, b in zip(probs, jobs, free):
        assert a.result.status == 0 and a.result.info.converged, p.name
        assert a.result.info.residuals == b.result.info.residuals, p.name
        assert all(np.array_equal(u, v) for u, v in zip(a.host_cores, b.host_cores))
    tiny = ps.PersistentServer(streams=2, min_interval=0.0, mem_budget=1)
    (job,) = tiny.serve(reqs[:1], [0.0])
    assert job.result.status == 0 and tiny.launches == 1
