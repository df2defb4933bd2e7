"""Batched engine and serving loop on the GPU.

* Every solve of a batch meets its tolerance (checked by the host oracle)
  and agrees with the one-at-a-time drop-in ``amen``: same sweeps and bonds,
  solutions within 1e-10 relative.
* A solve's result does not depend on what it is batched with: alone, in a
  mix, and admitted while others are running, the cores are bit-identical
  (every kernel gives each problem its own thread blocks and fixed-order
  reductions).
"""

import time

import numpy as np
import pytest

from conftest import golden_train, load_golden
from oracle import tt_oracle as O
from ttnumpy_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def tt():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ttnumpy_b200

    return ttnumpy_b200


def otrain(t):
    return O.Train(t.to_numpy(), t.orth_center)


def rel_tt(a, b):
    return O.tt_norm(O.add(a, O.scale(b, -1.0))) / O.tt_norm(b)


def golden_problem(tt, case):
    data = load_golden(case)
    A_c, _ = golden_train(data, "A")
    b_c, b_oc = golden_train(data, "b")
    x0 = None
    if "x0_n" in data:
        c, oc = golden_train(data, "x0")
        x0 = tt.TensorTrain(c, orth_center=oc)
    return (tt.TensorTrain(A_c), tt.TensorTrain(b_c, orth_center=b_oc), x0, dict(data["args"]),
            (A_c, b_c, b_oc))


CASES = ["amen_qtt_lap1d_o6", "amen_lap4_minres", "amen_cfg3", "amen_diffusion_0",
         "amen_nonsym_o5"]


def test_batch_matches_plain(tt):
    from ttnumpy_b200.batched import BatchEngine

    probs = [golden_problem(tt, c) for c in CASES]
    eng = BatchEngine()
    states = [eng.admit(A, b, x0, **args) for A, b, x0, args, _ in probs]
    eng.run()
    for case, s, (A, b, x0, args, host) in zip(CASES, states, probs):
        assert s.error is None, (case, s.error)
        x_plain, info_plain = tt.amen(A, b, x0=x0, return_info=True, **args)
        assert s.info.converged, (case, s.info)
        assert s.info.num_sweeps_run == info_plain.num_sweeps_run
        assert s.x.bonds == x_plain.bonds
        assert rel_tt(otrain(s.x), otrain(x_plain)) < 1e-10
        A_c, b_c, b_oc = host
        res = O.relative_residual(O.Train(A_c), O.Train(b_c, b_oc), otrain(s.x))
        assert res <= args["residual_tol"] * 1.05


def _diffusion(seed, d=4, n=16):
    theta = np.random.default_rng(seed).uniform(-1, 1, size=d)
    return P.parametric_diffusion(d, n, theta)


def test_alone_equals_mixed(tt):
    from ttnumpy_b200.batched import BatchEngine

    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=12, seed=0, stagnation_factor=None)
    target = _diffusion(5)
    others = [P.qtt_poisson_2d(4), _diffusion(6), P.qtt_poisson_2d(6), _diffusion(7, 5, 16)]

    def run(with_others, stagger):
        eng = BatchEngine()
        states = []
        if with_others:
            states += [eng.admit(tt.TensorTrain(p.A), tt.TensorTrain(p.b), **kw)
                       for p in others[:2]]
        for _ in range(stagger):
            eng.tick()
        s = eng.admit(tt.TensorTrain(target.A), tt.TensorTrain(target.b), **kw)
        if with_others:
            for _ in range(3):
                eng.tick()
            states += [eng.admit(tt.TensorTrain(p.A), tt.TensorTrain(p.b), **kw)
                       for p in others[2:]]
        eng.run()
        assert all(t.error is None for t in states + [s])
        return s

    alone = run(False, 0)
    mixed = run(True, 7)
    assert alone.info.converged and mixed.info.converged
    assert alone.info.residuals == mixed.info.residuals
    a, m = alone.x.to_numpy(), mixed.x.to_numpy()
    assert all(np.array_equal(u, v) for u, v in zip(a, m))


def test_server_staggered_arrivals(tt):
    from ttnumpy_b200.serving import Request, Server

    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=12, seed=0, stagnation_factor=None)
    probs = [P.qtt_poisson_2d(3 + (i % 5)) if i % 2 == 0 else _diffusion(10 + i)
             for i in range(8)]
    srv = Server()
    t0 = time.perf_counter()
    for i, p in enumerate(probs):
        srv.submit(Request(t0 + 0.02 * i, i, tt.TensorTrain(p.A), tt.TensorTrain(p.b), None, kw))
    done = srv.run()
    assert len(done) == len(probs)
    for req in done:
        assert req.state.error is None
        assert req.state.info.converged
        assert req.done_at >= req.arrival
        p = probs[req.rid]
        res = O.relative_residual(O.Train(p.A), O.Train(p.b), otrain(req.state.x))
        assert res <= 1.05e-8
