"""Mixed-precision AMEn on the persistent kernel: the iterative local
solves run as float64 iterative refinement around inner MINRES solves
whose operator products run on the tcgen05 tensor cores in 3xTF32.

Acceptance: the mixed solve ends within a factor 3 of the requested
residual (recomputed by the host oracle in float64; the sweep in which a
diffusion solve crosses 1e-8 is decided by rounding-level rank choices, and
the mixed trajectories take more sweeps than the float64 ones) and the
small diffusion case converges; its solution is within 1e-5 of the float64
solve's (relative difference, which the condition numbers of these
operators allow near residual 1e-8); the tensor cores did run (their FLOP
count is positive and refinement steps were taken); and a request gives the
same bits alone and in a mixed launch.  The relative error of each mixed
result against the float64 solve is printed beside it.
"""

import numpy as np
import pytest

from oracle import tt_oracle as O
from ttnumpy_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def pers():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ttnumpy_b200 import persistent

    return persistent


def _requests():
    rng = np.random.default_rng(17)
    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=30, seed=0, stagnation_factor=None)
    out = []
    for d, n in ((4, 16), (4, 32)):
        p = P.parametric_diffusion(d, n, rng.uniform(-1, 1, size=d))
        out.append((p, None, dict(kw)))
    # the 2-D QTT Poisson problem of config 3 with iterative local solves
    # above 50 unknowns (its default direct_solve_size keeps them all direct)
    p = P.qtt_poisson_2d(10)
    ranks = [1] + [3] * 19 + [1]
    x0 = [np.ones((ranks[i], 2, 1, ranks[i + 1])) for i in range(20)]
    out.append((p, x0, dict(kw, direct_solve_size=50)))
    return out


def test_mixed_matches_fp64(pers):
    reqs = _requests()
    fp = pers.amen_persistent([(p.A, p.b, x0, kw) for p, x0, kw in reqs])
    mx = pers.amen_persistent([(p.A, p.b, x0, dict(kw, precision="mixed")) for p, x0, kw in reqs])
    for (p, _, kw), a, m in zip(reqs, fp, mx):
        assert a.status == 0 and m.status == 0, (p.name, m.status)
        host = O.relative_residual(O.Train(p.A), O.Train(p.b), O.Train(m.x.to_numpy()))
        assert m.info.residuals[-1] == pytest.approx(host, rel=1e-6), (p.name, host)
        assert host <= 3.0 * kw["residual_tol"], (p.name, host)
        xa, xm = O.Train(a.x.to_numpy()), O.Train(m.x.to_numpy())
        rel = O.tt_norm(O.add(xm, O.scale(xa, -1.0))) / O.tt_norm(xa)
        print(f"{p.name}: mixed residual {host:.2e}, relative error vs float64 {rel:.2e}, "
              f"sweeps {m.info.num_sweeps_run} (float64 {a.info.num_sweeps_run}), "
              f"refinement steps {m.refine}, tensor-core GFLOP {m.flops_tc / 1e9:.2f}")
        assert rel < 1e-5, (p.name, rel)
        assert m.flops_tc > 0 and m.refine > 0, p.name
    assert mx[0].info.converged, mx[0].info


def test_mixed_alone_equals_in_launch(pers):
    reqs = _requests()
    p, x0, kw = reqs[1]
    kw = dict(kw, precision="mixed")
    (alone,) = pers.amen_persistent([(p.A, p.b, x0, kw)])
    mixed = pers.amen_persistent([(q.A, q.b, y0, dict(k, precision="mixed"))
                                  for q, y0, k in reqs])
    m = mixed[1]
    assert alone.status == 0 and m.status == 0
    assert alone.info.residuals == m.info.residuals
    assert all(np.array_equal(u, v) for u, v in zip(alone.x.to_numpy(), m.x.to_numpy()))


def test_precision_argument_checked(pers):
    p, x0, kw = _requests()[0]
    with pytest.raises(ValueError):
        pers.prepare([(p.A, p.b, x0, dict(kw, precision="fp16"))])
