"""The CPU oracle against the reference's own outputs (golden fixtures).

These pin the oracle before it is trusted as the checker of the CUDA path.
"""

import numpy as np
import pytest

from conftest import golden_train, load_golden
from oracle import tt_oracle as O
from ttnumpy_b200 import problems as P

AMEN_CASES = [
    "amen_qtt_lap1d_o6",
    "amen_nonsym_o5",
    "amen_nonsym_gmres",
    "amen_lap4_minres",
    "amen_lap5_threshold",
    "amen_cfg1_literal",
    "amen_cfg3",
    "amen_diffusion_0",
    "amen_diffusion_1",
]


def _train(data, name):
    cores, oc = golden_train(data, name)
    return O.Train([c.copy() for c in cores], oc)


#: Cases whose trajectory the reference itself does not reproduce from run to
#: run (one unconverged sweep of MINRES solves over rank-deficient QR
#: factors): only the rank trace and the residual's size are compared.
CHAOTIC = {"amen_cfg1_literal"}


@pytest.mark.parametrize("case", AMEN_CASES)
def test_oracle_amen_matches_reference(case):
    data = load_golden(case)
    A, b = _train(data, "A"), _train(data, "b")
    x0 = _train(data, "x0") if "x0_n" in data else None
    x, info = O.amen(A, b, x0=x0, **data["args"])
    ref_x = _train(data, "x")
    assert info.num_sweeps_run == int(data["num_sweeps_run"])
    assert info.stop_reason == str(data["stop_reason"])
    assert x.bonds == list(data["bonds"])
    assert info.local_solves == int(data["local_solves"])
    diff = O.tt_norm(O.add(x, O.scale(ref_x, -1.0))) / O.tt_norm(ref_x)
    if case in CHAOTIC:
        np.testing.assert_allclose(info.residuals, data["residuals"], rtol=0.25)
        assert diff < 0.05
        return
    # same algorithm, same LAPACK calls: the trajectories agree to rounding
    tol = data["args"].get("residual_tol") or 1e-8
    np.testing.assert_allclose(info.residuals, data["residuals"], rtol=1e-6, atol=1e-3 * tol)
    assert diff <= 1e-9


ALS_CASES = ["als_qtt_lap1d_o6", "als_lap4_minres", "als_nonsym_gmres"]


@pytest.mark.parametrize("case", ALS_CASES)
def test_oracle_als_matches_reference(case):
    """ALS (``solvers/als.py``): fixed ranks, same local solves as AMEn."""
    data = load_golden(case)
    A, b = _train(data, "A"), _train(data, "b")
    x0 = _train(data, "x0") if "x0_n" in data else None
    x, info = O.als(A, b, x0=x0, **data["args"])
    ref_x = _train(data, "x")
    assert info.num_sweeps_run == int(data["num_sweeps_run"])
    assert info.stop_reason == str(data["stop_reason"])
    assert x.bonds == list(data["bonds"])
    assert info.local_solves == int(data["local_solves"])
    np.testing.assert_allclose(info.residuals, data["residuals"], rtol=1e-6, atol=1e-14)
    diff = O.tt_norm(O.add(x, O.scale(ref_x, -1.0))) / O.tt_norm(ref_x)
    assert diff <= 1e-9


MALS_CASES = ["mals_qtt_lap1d_o6", "mals_lap4_minres", "mals_qtt_cap3", "mals_nonsym_gmres"]


@pytest.mark.parametrize("case", MALS_CASES)
def test_oracle_mals_matches_reference(case):
    """MALS (``solvers/mals.py``, ``two_site.py``): two-site solves and
    splits, the same sweeps, stop reason, bonds and residual trace as the
    reference."""
    data = load_golden(case)
    A, b = _train(data, "A"), _train(data, "b")
    x0 = _train(data, "x0") if "x0_n" in data else None
    x, info = O.mals(A, b, x0=x0, **data["args"])
    ref_x = _train(data, "x")
    assert info.num_sweeps_run == int(data["num_sweeps_run"])
    assert info.stop_reason == str(data["stop_reason"])
    assert x.bonds == list(data["bonds"])
    assert info.max_bonds == list(data["max_bonds"])
    assert info.local_solves == int(data["local_solves"])
    # residuals at round-off level (below 1e-12) agree only to that level
    np.testing.assert_allclose(info.residuals, data["residuals"], rtol=1e-6, atol=1e-12)
    diff = O.tt_norm(O.add(x, O.scale(ref_x, -1.0))) / O.tt_norm(ref_x)
    assert diff <= 1e-9


@pytest.mark.parametrize("case", ["truncate_pair_u", "truncate_pair_g", "truncate_pair_maxrank",
                                  "truncate_pair_d16"])
def test_oracle_truncate_matches_reference(case):
    data = load_golden(case)
    args = data["args"]
    pairs = 1 if case.endswith("d16") else 3
    d, r = (16, 32) if case.endswith("d16") else (8, 8)
    for pair in range(pairs):
        if args["gaussian"]:
            p, q = _train(data, f"p{pair}"), _train(data, f"q{pair}")
        else:
            p = O.Train(P.random_tt([4] * d, r, 2 * pair))
            q = O.Train(P.random_tt([4] * d, r, 2 * pair + 1))
        s = O.add(p, q)
        out = O.truncate(s, args["error"], args["max_rank"])
        assert out.bonds == list(data[f"bonds{pair}"])
        ref = _train(data, f"out{pair}")
        rel = O.tt_norm(O.add(out, O.scale(ref, -1.0))) / O.tt_norm(ref)
        assert rel < 1e-12


def test_oracle_truncate_canonical():
    data = load_golden("truncate_canonical")
    t = _train(data, "t")
    for canon in ("auto", "left", "right"):
        out = O.truncate(t, 1e-3, None, canonical=canon)
        ref = _train(data, f"out_{canon}")
        assert out.bonds == ref.bonds
        assert out.orth_center == ref.orth_center
        np.testing.assert_allclose(out.full(), ref.full(), atol=1e-12)


def test_oracle_dot_and_residual():
    data = load_golden("dot_residual")
    A, x, b = _train(data, "A"), _train(data, "x"), _train(data, "b")
    y = O.dot(A, x)
    assert y.bonds == _train(data, "y").bonds
    np.testing.assert_allclose(y.full(), data["y_full"], rtol=1e-12, atol=1e-12)
    assert O.relative_residual(A, b, x) == pytest.approx(float(data["residual"]), rel=1e-12)
    assert O.tt_norm(b) == pytest.approx(float(data["b_norm"]), rel=1e-14)


def test_oracle_dense_solution_qtt_laplacian():
    """The reference test's own dense check (solution vs np.linalg.solve)."""
    data = load_golden("amen_qtt_lap1d_o6")
    A, b = _train(data, "A"), _train(data, "b")
    x, info = O.amen(A, b, x0=_train(data, "x0"), **data["args"])
    exact = np.linalg.solve(A.full(), b.full())
    assert info.stop_reason == "converged"
    assert np.linalg.norm(x.full() - exact) / np.linalg.norm(exact) < 1e-8


def test_problem_builders_dense():
    """Config builders against dense assembly on small sizes."""
    A = O.Train(P.laplacian_nd(3, 5))
    h = 1 / 6
    L = (2 * np.eye(5) - np.eye(5, k=1) - np.eye(5, k=-1)) / h**2
    I = np.eye(5)
    dense = np.kron(np.kron(L, I), I) + np.kron(np.kron(I, L), I) + np.kron(np.kron(I, I), L)
    np.testing.assert_allclose(A.full(), dense, rtol=1e-12, atol=1e-9)
    # diffusion operator: compare with a direct assembly of -div(a grad u)
    d, n = 3, 5
    theta = np.array([0.3, -0.7, 0.5])
    A = O.Train(P.diffusion_operator(d, n, theta, 0.2))
    nodes = (np.arange(n) + 1) * h
    mids = (np.arange(n + 1) + 0.5) * h
    grids = np.meshgrid(nodes, nodes, nodes, indexing="ij")
    N = n**3
    M = np.zeros((N, N))
    idx = np.arange(N).reshape(n, n, n)

    def a_at(pt):
        return 1 + sum(0.2 * theta[k] * np.sin((k + 1) * np.pi * pt[k]) for k in range(d))

    for p in np.ndindex(n, n, n):
        i = idx[p]
        for ax in range(d):
            for s in (-1, 1):
                q = list(p)
                q[ax] += s
                pt = [nodes[p[k]] for k in range(d)]
                pt[ax] = mids[p[ax] + (1 if s == 1 else 0)]
                c = a_at(pt) / h**2
                M[i, i] += c
                if 0 <= q[ax] < n:
                    M[i, idx[tuple(q)]] -= c
    np.testing.assert_allclose(A.full(), M, rtol=1e-11, atol=1e-8)


def test_oracle_randomized_truncate_matches_reference():
    """``truncate(method="randomized")`` (``tensor_train.py:913-937``,
    ``utils.py:139-236``): same Gaussian draws, same QRs and SVDs."""
    data = load_golden("truncate_randomized")
    for name, kw in data["args"]["cases"]:
        src = _train(data, "A" if name == "ttm" else "s")
        out = O.truncate(src, method="randomized", **kw)
        ref = _train(data, f"out_{name}")
        assert out.bonds == ref.bonds, name
        diff = O.tt_norm(O.add(out, O.scale(ref, -1.0))) / O.tt_norm(ref)
        assert diff <= 1e-12, (name, diff)
        assert out.orth_center == ref.orth_center, name


def test_oracle_tt_svd_matches_reference():
    """``tt_svd`` (``tensor_train.py:1138-1247``): same bonds, same train
    (the same LAPACK gesvd, so the same signs) and the same centre."""
    data = load_golden("tt_svd")
    for name, src, kw in data["args"]["cases"]:
        kw = dict(kw)
        if "physical_indexes" in kw:
            kw["physical_indexes"] = [tuple(p) if isinstance(p, list) else p
                                      for p in kw["physical_indexes"]]
        out = O.tt_svd(data[src], **kw)
        ref = _train(data, f"out_{name}")
        assert out.bonds == ref.bonds, name
        assert all(np.allclose(a, b, rtol=1e-10, atol=1e-12) for a, b in zip(out.cores, ref.cores)), name
        assert out.orth_center == ref.orth_center == len(ref) - 1


def test_oracle_tt_to_qtt_matches_reference():
    """``tt_to_qtt`` (``tensor_train.py:942-1066``): same bonds, same cores
    (same LAPACK calls), centre on the last core."""
    data = load_golden("tt_to_qtt")
    for name, src, kw in data["args"]["cases"]:
        out = O.tt_to_qtt(_train(data, src), **kw)
        ref = _train(data, f"out_{name}")
        assert out.bonds == ref.bonds, name
        assert all(np.allclose(a, b, rtol=1e-9, atol=1e-12) for a, b in zip(out.cores, ref.cores)), name
        assert out.orth_center == ref.orth_center == len(ref) - 1


def test_oracle_qtt_to_tt_matches_reference():
    """``qtt_to_tt`` (``tensor_train.py:1072-1135``): regroupings of the
    quantised trains of the fixture, TTM pairs and a group of 40 cores most
    of mode 1; same bonds and cores as the reference."""
    data = load_golden("tt_to_qtt")
    for name, src, idx, kw in data["args"]["back"]:
        idx = [tuple(p) if isinstance(p, list) else p for p in idx]
        out = O.qtt_to_tt(_train(data, src), idx, **kw)
        ref = _train(data, f"back_{name}")
        assert out.bonds == ref.bonds, name
        assert all(np.allclose(a, b, rtol=1e-9, atol=1e-12) for a, b in zip(out.cores, ref.cores)), name
        assert out.orth_center == ref.orth_center


def test_oracle_qtt_round_trip_and_errors():
    """Quantise and merge back returns the train; mismatched indexes raise
    (``tests/test_tensor_train.py:592-620`` of the reference)."""
    t = O.Train([np.random.default_rng(3).standard_normal(s) for s in
                 [(1, 4, 1, 3), (3, 4, 1, 3), (3, 4, 1, 1)]])
    q = O.tt_to_qtt(t, error=1e-13)
    assert [c.shape[1] for c in q.cores] == [2] * 6
    back = O.qtt_to_tt(q, [4, 4, 4], error=1e-13)
    assert np.allclose(back.full(), t.full(), rtol=1e-11, atol=1e-12)
    for bad in ([4, 4], [8, 8, 8], [3, 8, 8]):
        with pytest.raises(ValueError):
            O.qtt_to_tt(q, bad)


def test_oracle_multiply_matches_reference():
    """Element-wise product of two trains (``tensor_train.py:327-407``):
    plain, direct rounding, and HaTT-1 randomized rounding
    (``utils.py:262-333``) with exact and lossy sketches and a TTM pair;
    the same random draws, so the same cores up to rounding."""
    data = load_golden("hadamard")
    for name, a, b, kw in data["args"]["cases"]:
        kw = dict(kw)
        tr = kw.pop("truncate", False)
        out = O.multiply(_train(data, a), _train(data, b), tr, **kw)
        ref = _train(data, f"out_{name}")
        assert out.bonds == ref.bonds, name
        assert all(np.allclose(x, y, rtol=1e-8, atol=1e-10) for x, y in zip(out.cores, ref.cores)), name
        assert out.orth_center == ref.orth_center, name


def _dense_ttm(matrix, order):
    return O.tt_svd(matrix.reshape([2] * 2 * order), error=0.0,
                    physical_indexes=[(2, 2)] * order, ttm=True)


def test_oracle_mals_solves_toeplitz_from_either_guess():
    """MALS behaviour the reference's tests pin (``tests/test_mals.py:53-79``):
    a symmetric Toeplitz system of size 256 solved to 1e-7 in one sweep from
    a rank-5 ones or random guess with the rank capped at 10."""
    import scipy.linalg as sla

    order, size = 8, 256
    mat = sla.toeplitz(np.arange(1, size + 1), np.arange(1, size + 1)).astype(float)
    A = _dense_ttm(mat, order)
    b = O.ones([2] * order)
    ref = np.linalg.solve(mat, np.ones(size))
    guesses = [O.orthonormalize(O.ones([2] * order, ranks=5), "right"),
               O.Train(P.random_tt([2] * order, 5, 153))]
    for x0 in guesses:
        x, _ = O.mals(A, b, x0=x0, error_threshold=1e-7, max_rank=10, max_sweeps=1)
        v = x.full().reshape(-1)
        assert np.linalg.norm(v - ref) / np.linalg.norm(ref) < 1e-7
        assert O.relative_residual(A, b, x) < 1e-7


def test_oracle_mals_nonsymmetric_default_guess():
    """A dense random operator solved from the default guess in two sweeps
    (``tests/test_mals.py:81-101``)."""
    order, size = 8, 256
    mat = np.random.default_rng(31).random((size, size))
    A = _dense_ttm(mat, order)
    ref = np.linalg.solve(mat, np.ones(size))
    b = O.tt_svd((mat @ ref).reshape([2] * order), error=0.0)
    x, _ = O.mals(A, b, error_threshold=1e-7, max_sweeps=2)
    v = x.full().reshape(-1)
    assert np.linalg.norm(v - ref) / np.linalg.norm(ref) < 1e-7
    assert O.relative_residual(A, b, x) < 1e-7


def test_oracle_qtt_reference_behaviours():
    """``tt_to_qtt`` behaviours the reference's tests pin
    (``tests/test_tensor_train.py:473-536``): the error stays within
    ``error * ||A||``, bonds floor at 1 under a huge error, and cores that
    need no split (mode 2) or modes like 243 = 3^5 are handled."""
    dense = np.random.default_rng(0).standard_normal((8, 8, 8))
    t = O.tt_svd(dense)
    for err in (3e-1, 1e-1, 1e-2, 1e-4):
        q = O.tt_to_qtt(t, error=err)
        assert np.linalg.norm(q.full().reshape(8, 8, 8) - dense) <= err * np.linalg.norm(dense)
    t16 = O.Train(P.random_tt([16, 16], 4, 120))
    assert O.tt_to_qtt(t16, error=1e2).bonds == [1] * 9
    for modes, base, seed in (([2, 8], 2, 121), ([243, 3], 3, 122)):
        t = O.Train(P.random_tt(modes, 2, seed))
        q = O.tt_to_qtt(t, mode_size=base, error=1e-12)
        assert all(c.shape[1] == base for c in q.cores)
        assert np.allclose(q.full().reshape(-1), t.full().reshape(-1), rtol=1e-10, atol=1e-12)


def test_canonical_cores_match_reference():
    """``canonical_tt`` (``tensor_train.py:1390-1446``): the host cores the
    device constructor uploads equal the reference's, with its centre."""
    from ttnumpy_b200.tensor_train import canonical_cores

    data = load_golden("canonical_tt")
    for name, dims, rank in data["args"]["cases"]:
        cores, center = canonical_cores(dims, rank)
        ref = _train(data, f"out_{name}")
        assert len(cores) == len(ref.cores), name
        assert all(np.array_equal(a, b) for a, b in zip(cores, ref.cores)), name
        assert center == ref.orth_center, name
