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


def test_staggered_arrivals_match_alone(srv_mod):
    pers, ps = srv_mod
    probs = _problems()
    reqs = [(p.A, p.b, None, KW) for p in probs]
    arrivals = [0.0, 0.0, 0.01, 0.02, 0.02, 0.05, 0.08, 0.08, 0.12, 0.2]
    server = ps.PersistentServer(streams=4, min_interval=0.002)
    jobs = server.serve(reqs, arrivals)
    assert server.launches >= 2
    for p, job in zip(probs, jobs):
        res = job.result
        assert res.status == 0 and res.info.converged, (p.name, res.info)
        assert job.latency is not None and job.latency >= 0.0
        host = O.relative_residual(O.Train(p.A), O.Train(p.b), O.Train(job.host_cores))
        assert host <= 1.05e-8, (p.name, host)
        (alone,) = pers.amen_persistent([(p.A, p.b, None, KW)])
        assert alone.info.residuals == res.info.residuals, p.name
        assert all(np.array_equal(u, v) for u, v in zip(alone.x.to_numpy(), job.host_cores))
