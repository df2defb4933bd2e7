"""GPU MALS (the drop-in ``mals``) against the reference's own results
(golden fixtures made by running ``ttnumpy.solvers.mals.mals``) and the
oracle.

MALS adapts every bond at each split, so the bonds are compared exactly;
the trajectory (sweeps, stop reason, per-sweep maximum bond, local solve
count, residual history) matches to rounding and the solution to 1e-8
relative (TT difference).
"""

import numpy as np
import pytest

from conftest import golden_train, load_golden
from oracle import tt_oracle as O
from ttnumpy_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = ["mals_qtt_lap1d_o6", "mals_lap4_minres", "mals_qtt_cap3", "mals_nonsym_gmres"]

# The GMRES case holds its local solves to 0.1 * residual_tol and stops at a
# global residual of ~9e-11, the same level: restarted GMRES here and
# SciPy's stop at different iterates within that tolerance, so the residual
# history agrees to 50 % and the solution to 1e-6.
LOOSE = {"mals_nonsym_gmres"}

# The default initial guess (ones with the bonds of b) is rank-deficient, so
# its right QR sweep leaves the trailing basis vectors of each bond to the
# QR's own choices, and the right environments of the first forward pass
# differ with them.  Under a binding rank cap the first sweep's residual
# depends on that basis (a 1e-14 perturbation of the guess moves it by
# 2e-5 relative in the oracle); from the second sweep on, and for the
# solution, the basis no longer matters.
FREE_START = {"mals_qtt_cap3"}


@pytest.fixture(scope="module")
def tt():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ttnumpy_b200

    return ttnumpy_b200


def _dist(x, ref_cores) -> float:
    ref = O.Train(ref_cores)
    got = O.Train(x.to_numpy())
    return O.tt_norm(O.add(got, O.scale(ref, -1.0))) / O.tt_norm(ref)


@pytest.mark.parametrize("case", CASES)
def test_mals_matches_reference(tt, case):
    data = load_golden(case)
    A_c, _ = golden_train(data, "A")
    b_c, b_oc = golden_train(data, "b")
    args = dict(data["args"])
    x, info = tt.mals(tt.TensorTrain(A_c), tt.TensorTrain(b_c, orth_center=b_oc),
                      return_info=True, **args)
    assert x.bonds == [int(v) for v in data["bonds"]]
    assert info.num_sweeps_run == int(data["num_sweeps_run"])
    assert str(info.stop_reason) == str(data["stop_reason"])
    assert info.max_bonds == [int(v) for v in data["max_bonds"]]
    assert info.local_solves == int(data["local_solves"])
    dist = _dist(x, golden_train(data, "x")[0])
    if case in LOOSE:
        np.testing.assert_allclose(info.residuals, data["residuals"], rtol=0.5)
        assert dist < 1e-6
    else:
        first = 1 if case in FREE_START else 0
        if first:
            assert info.residuals[0] == pytest.approx(float(data["residuals"][0]), rel=1e-3)
        np.testing.assert_allclose(info.residuals[first:], data["residuals"][first:], rtol=1e-5,
                                   atol=1e-13)
        assert dist < 1e-8
    assert x.orth_center == 0
    host = O.relative_residual(O.Train(A_c), O.Train(b_c), O.Train(x.to_numpy()))
    assert info.residuals[-1] == pytest.approx(host, rel=1e-6, abs=1e-12)


@pytest.mark.parametrize("kw", [
    dict(residual_tol=1e-8, symmetric=True, max_sweeps=4, direct_solve_size=200),
    dict(error_threshold=1e-4, max_sweeps=2, local_solver="direct"),
    dict(residual_tol=1e-6, max_rank=4, max_sweeps=3, symmetric=True, local_solver="minres",
         direct_solve_size=50),
])
def test_mals_matches_oracle(tt, kw):
    """A 4-D Laplacian with a rank-3 right-hand side and a random rank-2
    guess, under residual, threshold and capped MINRES truncation."""
    A_c, b_c = P.laplacian_nd(4, 6), P.random_tt([6] * 4, 3, seed=11)
    x0_c = P.random_tt([6] * 4, 2, seed=12)
    x, info = tt.mals(tt.TensorTrain(A_c), tt.TensorTrain(b_c), x0=tt.TensorTrain(x0_c),
                      return_info=True, **kw)
    xo, io = O.mals(O.Train(A_c), O.Train(b_c), x0=O.Train(x0_c), **kw)
    assert x.bonds == xo.bonds
    assert info.num_sweeps_run == io.num_sweeps_run
    assert str(info.stop_reason) == str(io.stop_reason)
    assert info.max_bonds == io.max_bonds
    np.testing.assert_allclose(info.residuals, io.residuals, rtol=1e-4, atol=1e-13)
    assert _dist(x, xo.cores) < 1e-6


def test_mals_small_trains_and_inputs(tt):
    """Two cores (only the backward pass solves), the inputs untouched and
    ``inplace``."""
    A_c, b_c = P.laplacian_nd(2, 5), P.random_tt([5] * 2, 2, seed=3)
    A, b = tt.TensorTrain(A_c), tt.TensorTrain(b_c)
    x0 = tt.ones([5, 5], ranks=2)
    before = [c.copy() for c in x0.to_numpy()]
    x, info = tt.mals(A, b, x0=x0, residual_tol=1e-10, max_sweeps=2, return_info=True)
    assert all(np.array_equal(u, v) for u, v in zip(before, x0.to_numpy()))
    assert all(np.array_equal(u, v) for u, v in zip(b_c, b.to_numpy()))
    assert info.converged and info.residuals[-1] <= 1e-10
    xo, io = O.mals(O.Train(A_c), O.Train(b_c), x0=O.Train(x0.to_numpy()), residual_tol=1e-10,
                    max_sweeps=2)
    assert x.bonds == xo.bonds and info.num_sweeps_run == io.num_sweeps_run
    y = tt.mals(A, b, x0=x0, inplace=True, max_sweeps=1)
    assert y is x0


def test_mals_errors(tt):
    A, b = tt.TensorTrain(P.laplacian_nd(3, 4)), tt.TensorTrain(P.random_tt([4] * 3, 2, seed=1))
    with pytest.raises(ValueError):
        tt.mals(A, b, max_rank=0)
    with pytest.raises(ValueError):
        tt.mals(A, b, residual_damp=0.5)
    with pytest.raises(ValueError):
        tt.mals(A, b, residual_tol=-1.0)
    with pytest.raises(tt.WrongTTType):
        tt.mals(b, b)
    with pytest.raises(tt.DimensionMismatch):
        tt.mals(A, tt.TensorTrain(P.random_tt([4] * 2, 2, seed=1)))


def _dense_ttm(matrix, order):
    return O.tt_svd(matrix.reshape([2] * 2 * order), error=0.0,
                    physical_indexes=[(2, 2)] * order, ttm=True)


def test_mals_reference_behaviours(tt):
    """Systems the reference's MALS tests solve (``tests/test_mals.py:53-101``),
    on the device: a Toeplitz system of size 256 in one sweep from a rank-5
    ones or random guess (rank cap 10), and a dense random operator from the
    default guess in two sweeps, each to 1e-7 in solution and residual."""
    import scipy.linalg as sla

    order, size = 8, 256
    mat = sla.toeplitz(np.arange(1, size + 1), np.arange(1, size + 1)).astype(float)
    A = _dense_ttm(mat, order)
    ref = np.linalg.solve(mat, np.ones(size))
    for x0 in (tt.ones([2] * order, ranks=5).orthonormalize("right"),
               tt.TensorTrain(P.random_tt([2] * order, 5, 153))):
        x = tt.mals(tt.TensorTrain(A.cores), tt.ones([2] * order), x0=x0, error_threshold=1e-7,
                    max_rank=10, max_sweeps=1)
        v = O.Train(x.to_numpy()).full().reshape(-1)
        assert np.linalg.norm(v - ref) / np.linalg.norm(ref) < 1e-7
        assert O.relative_residual(A, O.ones([2] * order), O.Train(x.to_numpy())) < 1e-7
    mat = np.random.default_rng(31).random((size, size))
    A = _dense_ttm(mat, order)
    ref = np.linalg.solve(mat, np.ones(size))
    b = O.tt_svd((mat @ ref).reshape([2] * order), error=0.0)
    x = tt.mals(tt.TensorTrain(A.cores), tt.TensorTrain(b.cores), error_threshold=1e-7,
                max_sweeps=2)
    v = O.Train(x.to_numpy()).full().reshape(-1)
    assert np.linalg.norm(v - ref) / np.linalg.norm(ref) < 1e-7
    assert O.relative_residual(A, b, O.Train(x.to_numpy())) < 1e-7
