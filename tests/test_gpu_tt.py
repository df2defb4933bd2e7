"""Device TensorTrain (truncate, dot, add, norms, canonical forms) and the
batched rounding kernel against the golden fixtures and the oracle.

Rounded trains are compared as reconstructions (SVD/QR signs are
ambiguous): relative difference below 1e-12 for exact operations, below the
requested truncation error for rounding, and identical bonds.
"""

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


def rel_tt(a: O.Train, b: O.Train) -> float:
    return O.tt_norm(O.add(a, O.scale(b, -1.0))) / O.tt_norm(b)


@pytest.mark.parametrize("case", ["truncate_pair_u", "truncate_pair_g", "truncate_pair_maxrank",
                                  "truncate_pair_d16"])
def test_truncate_matches_reference(tt, case):
    data = load_golden(case)
    args = data["args"]
    pairs = 1 if case.endswith("d16") else 3
    d, r = (16, 32) if case.endswith("d16") else (8, 8)
    for pair in range(pairs):
        if args["gaussian"]:
            p, _ = golden_train(data, f"p{pair}")
            q, _ = golden_train(data, f"q{pair}")
        else:
            p, q = P.random_tt([4] * d, r, 2 * pair), P.random_tt([4] * d, r, 2 * pair + 1)
        s = tt.TensorTrain(p) + tt.TensorTrain(q)
        out = s.truncate(error=args["error"], max_rank=args["max_rank"])
        ref_cores, _ = golden_train(data, f"out{pair}")
        assert out.bonds == [c.shape[0] for c in ref_cores] + [1]
        ref = O.Train(ref_cores)
        assert rel_tt(otrain(out), ref) < 1e-10
        # rounding error against the untruncated sum is within the request
        # (a max_rank cap may exceed it, as in the reference)
        if args["max_rank"] is None:
            err = rel_tt(otrain(out), O.add(O.Train(p), O.Train(q)))
            assert err <= args["error"] * 1.0001 + 1e-14


def test_truncate_canonical_and_centres(tt):
    data = load_golden("truncate_canonical")
    cores, oc = golden_train(data, "t")
    t = tt.TensorTrain(cores, orth_center=oc)
    for canon in ("auto", "left", "right"):
        out = t.truncate(error=1e-3, canonical=canon)
        ref_cores, ref_oc = golden_train(data, f"out_{canon}")
        assert out.bonds == [c.shape[0] for c in ref_cores] + [1]
        assert out.orth_center == ref_oc
        np.testing.assert_allclose(out.get_full_tensor(), O.Train(ref_cores).full().reshape(
            out.get_full_tensor().shape), atol=1e-11)


def test_dot_norm_residual(tt):
    data = load_golden("dot_residual")
    A = tt.TensorTrain(golden_train(data, "A")[0])
    x = tt.TensorTrain(golden_train(data, "x")[0])
    b = tt.TensorTrain(golden_train(data, "b")[0])
    y = A.dot(x)
    assert y.bonds == list(O.Train(golden_train(data, "y")[0]).bonds)
    np.testing.assert_allclose(y.get_full_tensor().reshape(-1), data["y_full"], rtol=1e-12,
                               atol=1e-12)
    assert (A @ x).bonds == y.bonds
    assert tt.relative_residual(A, b, x) == pytest.approx(float(data["residual"]), rel=1e-11)
    assert b.tt_norm() == pytest.approx(float(data["b_norm"]), rel=1e-13)


def test_orthonormalize_and_errors(tt):
    rng = np.random.default_rng(3)
    cores = [rng.standard_normal(s) for s in [(1, 3, 1, 4), (4, 3, 1, 5), (5, 3, 1, 1)]]
    t = tt.TensorTrain(cores)
    full = t.get_full_tensor()
    left = t.orthonormalize("left")
    assert left.orth_center == 2
    np.testing.assert_allclose(left.get_full_tensor(), full, atol=1e-12)
    c0 = left.cores[0].cpu().numpy().reshape(-1, left.bonds[1])
    np.testing.assert_allclose(c0.T @ c0, np.eye(c0.shape[1]), atol=1e-13)
    right = t.orthonormalize("right")
    assert right.orth_center == 0
    assert right.tt_norm() == pytest.approx(np.linalg.norm(full), rel=1e-13)
    assert t.tt_norm() == pytest.approx(np.linalg.norm(full), rel=1e-13)
    with pytest.raises(tt.DimensionMismatch):
        t + tt.TensorTrain([rng.standard_normal(s) for s in [(1, 2, 1, 1), (1, 3, 1, 1),
                                                             (1, 3, 1, 1)]])
    with pytest.raises(tt.WrongTTFormat):
        tt.TensorTrain([rng.standard_normal((2, 3, 1, 1)), rng.standard_normal((1, 3, 1, 1))])
    with pytest.raises(TypeError):
        t.dot(3)
    with pytest.raises(ValueError):
        t.truncate(canonical="mix")
    with pytest.raises(tt.DimensionMismatch):
        t.dot(t)
    with pytest.raises(ValueError):
        tt.eye([3, 3, 3]).dot(t, error=1e-3)


@pytest.mark.parametrize("d,n,r,err,mr,gauss", [(6, 4, 6, 1e-6, None, False),
                                               (8, 4, 8, 1e-6, None, True),
                                               (8, 4, 8, 1e-4, 5, True),
                                               (16, 4, 32, 1e-6, None, False),
                                               (7, 2, 20, 1e-8, None, True)])
def test_round_batch_matches_oracle(tt, d, n, r, err, mr, gauss):
    from ttnumpy_b200.rounding import PackedTrains, round_sum_batch

    pairs = 5
    rng = np.random.default_rng(d * 100 + r)
    ranks = [1] + [r] * (d - 1) + [1]
    if gauss:
        ps = [[rng.standard_normal((ranks[k], n, 1, ranks[k + 1])) for k in range(d)]
              for _ in range(pairs)]
        qs = [[rng.standard_normal((ranks[k], n, 1, ranks[k + 1])) for k in range(d)]
              for _ in range(pairs)]
    else:
        ps = [P.random_tt([n] * d, r, 2 * i) for i in range(pairs)]
        qs = [P.random_tt([n] * d, r, 2 * i + 1) for i in range(pairs)]
    res = round_sum_batch(PackedTrains.from_numpy(ps), PackedTrains.from_numpy(qs), err, mr)
    assert (res.status.cpu().numpy() >= 0).all()
    for i in range(pairs):
        s = O.add(O.Train(ps[i]), O.Train(qs[i]))
        want = O.truncate(s, err, mr)
        got = otrain(res.train(i))
        assert got.bonds == want.bonds
        assert rel_tt(got, want) < max(1e-10, 0.01 * err)


def test_randomized_truncate_matches_reference(tt):
    """``truncate(method="randomized")`` against the reference's results:
    the same Gaussian sketch (drawn on the host from the seed), QRs and SVD
    sweep on the device; bonds, orthogonality centre and the rounded train
    (TT difference, 1e-10 relative) agree, including a lossy sketch and a
    TTM train."""
    data = load_golden("truncate_randomized")
    for name, kw in data["args"]["cases"]:
        key = "A" if name == "ttm" else "s"
        cores, oc = golden_train(data, key)
        src = tt.TensorTrain(cores, orth_center=oc)
        out = src.truncate(method="randomized", **kw)
        ref_c, ref_oc = golden_train(data, f"out_{name}")
        ref = O.Train(ref_c)
        assert out.bonds == ref.bonds, name
        assert out.orth_center == ref_oc, name
        got = O.Train(out.to_numpy())
        diff = O.tt_norm(O.add(got, O.scale(ref, -1.0))) / O.tt_norm(ref)
        assert diff < 1e-10, (name, diff)


def test_randomized_truncate_errors(tt):
    t = tt.TensorTrain(P.random_tt([3] * 4, 3, seed=1))
    with pytest.raises(ValueError):
        t.truncate(method="randomized")  # needs max_rank
    with pytest.raises(ValueError):
        t.truncate(method="randomized", max_rank=2, options={"bogus": 1})
    with pytest.raises(ValueError):
        t.truncate(method="randomized", max_rank=2, options={"oversampling": -1})
    with pytest.raises(ValueError):
        t.truncate(method="sketch")


def test_randomized_rounding_of_products(tt):
    """``dot(..., truncate=True, method="randomized")`` rounds the product
    exactly as ``truncate`` of the product does with the same seed."""
    A = tt.TensorTrain(P.laplacian_nd(4, 5))
    x = tt.TensorTrain(P.random_tt([5] * 4, 3, seed=2))
    direct = A.dot(x).truncate(method="randomized", max_rank=4, seed=9)
    fused = A.dot(x, truncate=True, max_rank=4, method="randomized", seed=9)
    assert direct.bonds == fused.bonds
    assert all(np.array_equal(u, v) for u, v in zip(direct.to_numpy(), fused.to_numpy()))


def test_tt_svd_matches_reference(tt):
    """``tt_svd`` on the device against the reference's trains: the same
    bonds and centre, and the same tensor (dense comparison; the SVD signs
    may differ, the product may not)."""
    data = load_golden("tt_svd")
    for name, src, kw in data["args"]["cases"]:
        kw = dict(kw)
        if "physical_indexes" in kw:
            kw["physical_indexes"] = [tuple(p) if isinstance(p, list) else p
                                      for p in kw["physical_indexes"]]
        dense = np.asarray(data[src])
        for inp in (dense, torch.from_numpy(dense).cuda()):
            out = tt.tt_svd(inp, **kw)
            ref_c, ref_oc = golden_train(data, f"out_{name}")
            assert out.bonds == O.Train(ref_c).bonds, name
            assert out.orth_center == ref_oc
            got, want = O.Train(out.to_numpy()).full(), O.Train(ref_c).full()
            assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want), name


def test_tt_svd_errors(tt):
    with pytest.raises(tt.AmbiguousFormat):
        tt.tt_svd(np.ones(8))
    with pytest.raises(tt.AmbiguousFormat):
        tt.tt_svd(np.ones((2, 2)), ttm=True)


def _dense_close(out_cores, ref_cores, rel=1e-10):
    got, want = O.Train(out_cores).full(), O.Train(ref_cores).full()
    return np.linalg.norm(got - want) <= rel * np.linalg.norm(want)


def test_tt_to_qtt_matches_reference(tt):
    """``tt_to_qtt`` on the device against the reference's quantised trains
    (``tensor_train.py:942-1066``): same bonds, modes and centre, the same
    tensor, left-orthonormal cores, and the source left untouched."""
    data = load_golden("tt_to_qtt")
    for name, src, kw in data["args"]["cases"]:
        src_c, _ = golden_train(data, src)
        ref_c, ref_oc = golden_train(data, f"out_{name}")
        t = tt.TensorTrain(src_c)
        out = t.tt_to_qtt(**kw)
        assert out.bonds == O.Train(ref_c).bonds, name
        assert out.orth_center == ref_oc == len(ref_c) - 1, name
        assert out.physical_dims() == [(c.shape[1], c.shape[2]) if c.shape[2] > 1 else c.shape[1]
                                       for c in ref_c], name
        cores = out.to_numpy()
        assert _dense_close(cores, ref_c), name
        for c in cores[:-1]:
            m = c.reshape(-1, c.shape[-1])
            assert np.allclose(m.T @ m, np.eye(m.shape[1]), atol=1e-12), name
        assert all(np.array_equal(a, b) for a, b in zip(src_c, t.to_numpy())), name
        assert t.orth_center is None


def test_qtt_to_tt_matches_reference(tt):
    """``qtt_to_tt`` on the device (``tensor_train.py:1072-1135``):
    regroupings, TTM pairs and a 40-core group mostly of mode 1 against the
    reference's merged and rounded trains."""
    data = load_golden("tt_to_qtt")
    for name, src, idx, kw in data["args"]["back"]:
        idx = [tuple(p) if isinstance(p, list) else p for p in idx]
        src_c, _ = golden_train(data, src)
        ref_c, ref_oc = golden_train(data, f"back_{name}")
        out = tt.TensorTrain(src_c).qtt_to_tt(idx, **kw)
        assert out.bonds == O.Train(ref_c).bonds, name
        assert out.orth_center == ref_oc, name
        assert out.physical_dims() == idx, name
        assert _dense_close(out.to_numpy(), ref_c), name


def test_qtt_cycles_and_error_bound(tt):
    """Five quantise/merge cycles keep the tensor; the quantisation error
    stays within ``error * ||A||`` (reference tests/test_tensor_train.py:
    458-481)."""
    t = tt.rand([8] * 4, ranks=8, seed=118)
    want = O.Train(t.to_numpy()).full()
    for _ in range(5):
        t = t.tt_to_qtt(error=1e-12).qtt_to_tt([8] * 4, error=1e-12)
    assert np.linalg.norm(O.Train(t.to_numpy()).full() - want) <= 1e-10 * np.linalg.norm(want)
    dense = np.random.default_rng(0).standard_normal((8, 8, 8))
    src = tt.tt_svd(dense)
    for err in (3e-1, 1e-1, 1e-2, 1e-4):
        q = src.tt_to_qtt(error=err)
        got = O.Train(q.to_numpy()).full().reshape(8, 8, 8)
        assert np.linalg.norm(got - dense) <= err * np.linalg.norm(dense)
    assert tt.rand([16, 16], ranks=4, seed=120).tt_to_qtt(error=1e2).bonds == [1] * 9


def test_qtt_errors(tt):
    t = tt.rand([4, 4], ranks=2, seed=123)
    with pytest.raises(ValueError):
        t.tt_to_qtt(max_rank=0)
    with pytest.raises(ValueError):
        t.tt_to_qtt(mode_size=1)
    with pytest.raises(tt.DimensionMismatch):
        t.tt_to_qtt(mode_size=3)
    with pytest.raises(tt.DimensionMismatch):
        tt.rand([(4, 2), (4, 2)], ranks=2, seed=124).tt_to_qtt()
    q = tt.rand([4, 4, 4], ranks=3, seed=125).tt_to_qtt(error=1e-12)
    for bad in ([4, 4], [8, 8, 8], [3, 8, 8]):
        with pytest.raises(tt.DimensionMismatch):
            q.qtt_to_tt(bad)
    qm = tt.rand([(4, 4), (4, 4)], ranks=3, seed=126).tt_to_qtt(error=1e-12)
    with pytest.raises(tt.DimensionMismatch):
        qm.qtt_to_tt([(4, 2), (4, 8)])


def test_multiply_matches_reference(tt):
    """Element-wise product of two trains on the device against the
    reference's results (``tensor_train.py:327-407``): the plain product
    (``ttb_hadamard`` cores, exact), its direct rounding, and HaTT-1
    randomized rounding (``utils.py:262-333``) with exact and lossy
    sketches, an error bound and a TTM pair, drawn from the same seeds."""
    data = load_golden("hadamard")
    for name, a, b, kw in data["args"]["cases"]:
        ac, _ = golden_train(data, a)
        bc, _ = golden_train(data, b)
        ref_c, ref_oc = golden_train(data, f"out_{name}")
        out = tt.TensorTrain(ac).multiply(tt.TensorTrain(bc), **kw)
        assert out.bonds == O.Train(ref_c).bonds, name
        assert out.orth_center == ref_oc, name
        if name == "plain":
            assert all(np.array_equal(x, y) for x, y in zip(out.to_numpy(), ref_c)), name
        got, want = O.Train(out.to_numpy()).full(), O.Train(ref_c).full()
        assert np.linalg.norm(got - want) <= 1e-9 * np.linalg.norm(want), name


def test_hattt_equals_sketch_of_formed_product(tt):
    """HaTT-1 without the product cores gives the randomized left
    orthonormalisation of the formed product train (same draws)."""
    from ttnumpy_b200 import tensor_train as T

    p = tt.rand([3] * 6, ranks=4, seed=1)
    q = tt.rand([3] * 6, ranks=5, seed=2)
    formed = [tt.kernels.hadamard(a, b) for a, b in zip(p.cores, q.cores)]
    ref = T.randomized_left_orth(list(formed), 9, np.random.default_rng(7))
    got = T.randomized_hadamard(p.cores, q.cores, 9, np.random.default_rng(7))
    assert [c.shape for c in got] == [c.shape for c in ref]
    a = O.Train([c.cpu().numpy() for c in got]).full()
    b = O.Train([c.cpu().numpy() for c in ref]).full()
    assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)
    for c in got[:-1]:
        m = c.reshape(-1, c.shape[-1]).cpu().numpy()
        assert np.allclose(m.T @ m, np.eye(m.shape[1]), atol=1e-12)


def test_multiply_errors(tt):
    p = tt.rand([3] * 4, ranks=2, seed=1)
    with pytest.raises(tt.DimensionMismatch):
        p.multiply(tt.rand([2] * 4, ranks=2, seed=1))
    with pytest.raises(ValueError):
        p.multiply(p, method="randomized")
    with pytest.raises(ValueError):
        p.multiply(p, truncate=True, method="randomized", max_rank=0)
    with pytest.raises(TypeError):
        p.multiply("x")


def test_canonical_tt_matches_reference(tt):
    """``canonical_tt`` on the device: the reference's cores and centre."""
    data = load_golden("canonical_tt")
    for name, dims, rank in data["args"]["cases"]:
        t = tt.canonical_tt(dims, rank)
        ref_c, ref_oc = golden_train(data, f"out_{name}")
        assert t.orth_center == ref_oc, name
        assert all(np.array_equal(a, b) for a, b in zip(t.to_numpy(), ref_c)), name
    with pytest.raises(tt.WrongTTFormat):
        tt.canonical_tt([4], 2)


def test_element_matricize_transpose(tt):
    """``get_element``, ``matricize``, ``transpose`` and ``conj``
    (``tensor_train.py:556-703``) against the dense tensors of the host
    cores, for a TT and a TTM (reference tests/test_tensor_train.py:60-145)."""
    rng = np.random.default_rng(7)
    ranks = [1, 2, 3, 1]
    tcores = [rng.standard_normal((ranks[k], 3, 1, ranks[k + 1])) for k in range(3)]
    mcores = [rng.standard_normal((ranks[k], 2, 3, ranks[k + 1])) for k in range(3)]
    t, m = tt.TensorTrain(tcores), tt.TensorTrain(mcores)
    vec_t = O.Train(tcores).full()  # the reference's matricize order
    dense_t = vec_t.reshape(3, 3, 3)
    assert t.get_element([2, 0, 1]) == pytest.approx(dense_t[2, 0, 1], rel=1e-13)
    assert t.get_element([(1, 0), (2, 0), (0, 0)]) == pytest.approx(dense_t[1, 2, 0], rel=1e-13)
    with pytest.raises(tt.DimensionMismatch):
        t.get_element([0, 0])
    np.testing.assert_allclose(t.matricize(), vec_t, rtol=1e-13, atol=1e-14)
    # TTM: the (rows x columns) operator, entries indexed (rows..., cols...)
    mat_m = O.Train(mcores).full()
    dense_m = mat_m.reshape(2, 2, 2, 3, 3, 3)
    assert m.get_element([(1, 2), (0, 0), (1, 1)]) == pytest.approx(dense_m[1, 0, 1, 2, 0, 1],
                                                                   rel=1e-13)
    np.testing.assert_allclose(m.matricize(), mat_m, rtol=1e-13, atol=1e-14)
    mt = m.transpose()
    assert mt.row_modes == [3, 3, 3] and mt.col_modes == [2, 2, 2]
    np.testing.assert_allclose(mt.matricize(), mat_m.T, rtol=1e-13, atol=1e-14)
    part = m.transpose([0])
    assert np.array_equal(part.to_numpy()[0], mcores[0].transpose(0, 2, 1, 3))
    assert np.array_equal(part.to_numpy()[1], mcores[1])
    assert np.array_equal(m.to_numpy()[0], mcores[0])  # not in place
    back = mt.transpose(conjugate=True).conj()
    assert all(np.array_equal(a, b) for a, b in zip(back.to_numpy(), mcores))
    col = t.transpose()
    assert col.is_ttm() and col.col_modes == [3, 3, 3]
