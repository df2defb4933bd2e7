"""Whole AMEn solves in one persistent launch (one thread block per solve)
against the reference's results and the one-at-a-time drop-in.

Same acceptance as the drop-in (``test_gpu_amen.py``): convergence, the final
residual recomputed by the host oracle within ``residual_tol``, and the
distance to the reference solution below 1e-6; plus: a solve gives
bit-identical results alone and launched with others.
"""

import numpy as np
import pytest

from conftest import golden_train, load_golden
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


def otrain(t):
    return O.Train(t.to_numpy(), t.orth_center)


def rel_tt(a, b):
    return O.tt_norm(O.add(a, O.scale(b, -1.0))) / O.tt_norm(b)


CASES = ["amen_qtt_lap1d_o6", "amen_lap4_minres", "amen_cfg3", "amen_diffusion_0",
         "amen_diffusion_1", "amen_nonsym_o5"]


def golden_request(case):
    import ttnumpy_b200 as tt

    data = load_golden(case)
    A_c, _ = golden_train(data, "A")
    b_c, b_oc = golden_train(data, "b")
    x0 = None
    if "x0_n" in data:
        c, oc = golden_train(data, "x0")
        x0 = tt.TensorTrain(c, orth_center=oc)
    b = tt.TensorTrain(b_c, orth_center=b_oc)
    return (A_c, b, x0, dict(data["args"])), data


# The reference converges this case at 9.94e-9 (0.6 % below the tolerance)
# with stagnation_factor="auto": rounding-level differences in the rank
# decisions decide between "converged" and "stagnated" a hair above the
# tolerance, so it is held to the tolerance within a factor 2.
BORDERLINE = {"amen_diffusion_1"}


def test_golden_cases_one_launch(pers):
    reqs, datas = zip(*[golden_request(c) for c in CASES])
    out = pers.amen_persistent(list(reqs))
    for case, res, req, data in zip(CASES, out, reqs, datas):
        assert res.status == 0, (case, pers.STATUS.get(res.status))
        A_c, b, _, args = req
        b_c, b_oc = golden_train(data, "b")
        host = O.relative_residual(O.Train(A_c), O.Train(b_c, b_oc), otrain(res.x))
        if case in BORDERLINE:
            assert str(res.info.stop_reason) in ("converged", "stagnated"), (case, res.info)
            assert host <= args["residual_tol"] * 2.0, (case, host)
            assert res.info.residuals[-1] == pytest.approx(host, rel=1e-6)
            ref = O.Train(golden_train(data, "x")[0])
            assert rel_tt(otrain(res.x), ref) < 1e-5, case
            continue
        assert res.info.converged, (case, res.info)
        assert host <= args["residual_tol"] * 1.05, (case, host)
        assert res.info.residuals[-1] == pytest.approx(host, rel=1e-6, abs=1e-3 * args["residual_tol"])
        ref = O.Train(golden_train(data, "x")[0])
        assert rel_tt(otrain(res.x), ref) < 1e-6, case
        assert abs(res.info.num_sweeps_run - int(data["num_sweeps_run"])) <= 1, case
        assert len(res.info.max_bonds) == res.info.num_sweeps_run


def test_gmres_local_solves(pers):
    """A non-symmetric system with local solves forced onto GMRES
    (direct_solve_size 4): the persistent kernel's restarted GMRES against
    the reference's run."""
    req, data = golden_request("amen_nonsym_gmres")
    (res,) = pers.amen_persistent([req])
    assert res.status == 0, pers.STATUS.get(res.status)
    A_c, b, _, args = req
    b_c, b_oc = golden_train(data, "b")
    host = O.relative_residual(O.Train(A_c), O.Train(b_c, b_oc), otrain(res.x))
    assert res.info.converged, res.info
    assert host <= args["residual_tol"] * 1.05
    assert res.info.residuals[-1] == pytest.approx(host, rel=1e-6, abs=1e-3 * args["residual_tol"])
    ref = O.Train(golden_train(data, "x")[0])
    assert rel_tt(otrain(res.x), ref) < 1e-6
    assert abs(res.info.num_sweeps_run - int(data["num_sweeps_run"])) <= 1
    assert res.info.local_solves == int(data["local_solves"])


def test_threshold_mode_case(pers):
    req, data = golden_request("amen_lap5_threshold")
    (res,) = pers.amen_persistent([req])
    assert res.status == 0
    assert str(res.info.stop_reason) == str(data["stop_reason"])
    assert res.info.num_sweeps_run == int(data["num_sweeps_run"])
    got, ref = np.asarray(res.info.residuals), np.asarray(data["residuals"])
    assert np.all(got <= 2.0 * ref) and np.all(got >= 0.5 * ref)
    assert max(res.x.bonds) <= 7


def _diffusion(seed, d=4, n=16):
    theta = np.random.default_rng(seed).uniform(-1, 1, size=d)
    return P.parametric_diffusion(d, n, theta)


def test_alone_equals_in_launch(pers):
    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=12, seed=0, stagnation_factor=None)
    target = _diffusion(5)
    others = [P.qtt_poisson_2d(4), _diffusion(6), P.qtt_poisson_2d(6), _diffusion(7, 5, 16)]
    (alone,) = pers.amen_persistent([(target.A, target.b, None, kw)])
    mixed = pers.amen_persistent([(p.A, p.b, None, kw) for p in others[:2]]
                                 + [(target.A, target.b, None, kw)]
                                 + [(p.A, p.b, None, kw) for p in others[2:]])
    assert all(r.status == 0 and r.info.converged for r in mixed)
    m = mixed[2]
    assert alone.info.residuals == m.info.residuals
    assert all(np.array_equal(u, v) for u, v in zip(alone.x.to_numpy(), m.x.to_numpy()))
    for p, r in zip(others[:2] + [target] + others[2:], mixed):
        res = O.relative_residual(O.Train(p.A), O.Train(p.b), otrain(r.x))
        assert res <= 1.05e-8


def test_cluster_equals_lone_block(pers):
    """A solve on a cluster of four blocks (the leader's larger products
    shared out by output tile and row) gives the lone block's bits."""
    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=6, seed=0, stagnation_factor=None)
    probs = [_diffusion(8, 4, 64), _diffusion(10, 5, 32), P.qtt_poisson_2d(6)]
    reqs = [(p.A, p.b, None, kw) for p in probs]
    lone = pers.amen_persistent(reqs, rmax=96)
    clus = pers.amen_persistent(reqs, rmax=96, cluster=4)
    for p, a, b in zip(probs, lone, clus):
        assert a.status == 0 and b.status == 0, (p.name, b.status)
        assert a.info.residuals == b.info.residuals, p.name
        assert all(np.array_equal(u, v) for u, v in zip(a.x.to_numpy(), b.x.to_numpy())), p.name


def test_graph_replay_equals_launch(pers):
    """The batch's launch captured in a CUDA graph and replayed re-solves
    every request with the same bits, lone blocks and clusters alike."""
    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=8, seed=0, stagnation_factor=None)
    probs = [_diffusion(12, 4, 32), P.qtt_poisson_2d(5)]
    for cluster in (1, 2):
        batch = pers.PersistentBatch(pers.prepare([(p.A, p.b, None, kw) for p in probs]), 64,
                                     cluster=cluster)
        first = batch.run()
        graph = batch.capture()
        graph.replay()
        torch.cuda.synchronize()
        again = batch.collect()
        for a, b in zip(first, again):
            assert a.status == 0 and b.status == 0
            assert a.info.residuals == b.info.residuals
            assert all(np.array_equal(u, v) for u, v in zip(a.x.to_numpy(), b.x.to_numpy()))


def test_matches_dropin(pers):
    import ttnumpy_b200 as tt

    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=12, seed=0, stagnation_factor=None)
    p = _diffusion(9, 5, 16)
    (res,) = pers.amen_persistent([(p.A, p.b, None, kw)])
    x, info = tt.amen(tt.TensorTrain(p.A), tt.TensorTrain(p.b), return_info=True, **kw)
    # the rank search applies the operator term by term instead of as one
    # matmat, so the trajectories agree to rounding only: same acceptance
    assert res.info.converged and info.converged
    assert abs(res.info.num_sweeps_run - info.num_sweeps_run) <= 1
    assert rel_tt(otrain(res.x), otrain(x)) < 1e-6


def test_rank1_factorisation_self_check(pers):
    """The rank search applies the operator to each rank-one term through
    its factorisation over the operator bond; in debug mode the kernel also
    applies it in full and records the worst relative gap (rounding only)."""
    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=4, seed=0, stagnation_factor=None)
    reqs = [(p.A, p.b, None, kw) for p in (_diffusion(3, 4, 16), P.qtt_poisson_2d(5))]
    batch = pers.PersistentBatch(pers.prepare(reqs), 64, debug=True)
    out = batch.run()
    assert all(r.status == 0 for r in out)
    checks = [row["check"] for row in batch.breakdown()]
    assert max(checks) < 1e-11, checks
    assert checks[0] > 0.0  # the diffusion solve truncated with residual-budget ranks


def test_chunked_rank_search_matches_term_by_term(pers):
    """Outside debug mode the rank search forms the applied rank-one terms
    eight at a time (three GEMMs per chunk, the rank-R contraction fused
    into the running-sum loop); debug mode keeps the term-by-term search.
    Both must take the same rank decisions: same bonds and sweeps, residuals
    and solutions equal to rounding."""
    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=4, seed=0, stagnation_factor=None)
    reqs = [(p.A, p.b, None, kw) for p in (_diffusion(3, 4, 16), _diffusion(4, 3, 32),
                                           P.qtt_poisson_2d(5))]
    runs = []
    for debug in (True, False):
        batch = pers.PersistentBatch(pers.prepare(reqs), 64, debug=debug)
        out = batch.run()
        assert all(r.status == 0 for r in out)
        runs.append(out)
    for a, b in zip(*runs):
        assert a.x.bonds == b.x.bonds
        assert a.info.num_sweeps_run == b.info.num_sweeps_run
        np.testing.assert_allclose(a.info.residuals, b.info.residuals, rtol=1e-6, atol=1e-14)
        assert rel_tt(otrain(a.x), otrain(b.x)) < 1e-9


def test_two_level_qr_self_check(pers):
    """The residual-norm sweep factorises tall matrices (rows >= 4 x columns,
    more than 64 columns) with the two-level blocked R-only QR; in debug mode
    each such factorisation is repeated with the one-level blocked QR and the
    worst relative gap of R is recorded (rounding only)."""
    kw = dict(residual_tol=1e-8, symmetric=True, max_sweeps=6, seed=0, stagnation_factor=None)
    reqs = [(p.A, p.b, None, kw) for p in (_diffusion(4, 4, 32), _diffusion(5, 5, 16))]
    batch = pers.PersistentBatch(pers.prepare(reqs), 64, debug=True)
    out = batch.run()
    assert all(r.status == 0 for r in out)
    rows = batch.breakdown()
    assert sum(row["n_qr2"] for row in rows) > 0
    # Householder QR is backward stable with ||dR|| <= c m eps ||A||; for
    # m ~ 2000-7000 rows the two orders of summation differ by ~1e-12
    assert max(row["check_qr"] for row in rows) < 1e-10, rows
