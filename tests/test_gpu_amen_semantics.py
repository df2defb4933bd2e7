"""AMEn behaviours the reference's own tests pin (ttnumpy tests/test_amen.py),
on the drop-in and on the persistent whole-solve kernel:

* ``max_rank`` caps every bond, and a cap above the needed rank still
  converges (test_amen.py:364-441); the capped solve's bonds equal the
  oracle's.
* With ``residual_tol`` set, truncation follows the residual budget and
  ignores ``error_threshold``: identical bonds and cores (:443-478).
* The inputs are not modified and the global NumPy random state is
  untouched (:508-533).
* The reported final residual equals the host recomputation (:388-415).
"""

import numpy as np
import pytest

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


def _problem():
    return P.laplacian_nd(4, 8), P.random_tt([8] * 4, 3, seed=11)


KW = dict(residual_tol=1e-8, symmetric=True, max_sweeps=12, seed=5, direct_solve_size=40)


@pytest.mark.parametrize("cap", [3, 6])
def test_max_rank_cap(tt, cap):
    A_c, b_c = _problem()
    x, info = tt.amen(tt.TensorTrain(A_c), tt.TensorTrain(b_c), max_rank=cap, return_info=True,
                      **KW)
    assert max(x.bonds) <= cap
    xo, io = O.amen(O.Train(A_c), O.Train(b_c), max_rank=cap, **KW)
    assert x.bonds == xo.bonds
    assert info.num_sweeps_run == io.num_sweeps_run
    assert str(info.stop_reason) == str(io.stop_reason)
    from ttnumpy_b200.persistent import amen_persistent

    (r,) = amen_persistent([(A_c, b_c, None, dict(KW, max_rank=cap))])
    assert r.status == 0 and max(r.x.bonds) <= cap


def test_cap_above_needed_rank_converges(tt):
    A_c, b_c = _problem()
    x, info = tt.amen(tt.TensorTrain(A_c), tt.TensorTrain(b_c), max_rank=40, return_info=True,
                      **KW)
    assert info.converged
    assert O.relative_residual(O.Train(A_c), O.Train(b_c), O.Train(x.to_numpy())) <= 1.05e-8


def test_residual_mode_ignores_error_threshold(tt):
    A_c, b_c = _problem()
    outs = []
    for eth in (1e-3, 1e-12):
        x = tt.amen(tt.TensorTrain(A_c), tt.TensorTrain(b_c), error_threshold=eth, **KW)
        outs.append(x)
    assert outs[0].bonds == outs[1].bonds
    assert all(np.array_equal(a, b) for a, b in zip(outs[0].to_numpy(), outs[1].to_numpy()))
    from ttnumpy_b200.persistent import amen_persistent

    r1, r2 = amen_persistent([(A_c, b_c, None, dict(KW, error_threshold=e)) for e in (1e-3, 1e-12)])
    assert r1.x.bonds == r2.x.bonds
    assert all(np.array_equal(a, b) for a, b in zip(r1.x.to_numpy(), r2.x.to_numpy()))


def test_inputs_and_global_rng_untouched(tt):
    A_c, b_c = _problem()
    A, b = tt.TensorTrain(A_c), tt.TensorTrain(b_c)
    x0 = tt.ones(b.physical_dims(), ranks=2)
    a_before = [c.copy() for c in A.to_numpy()]
    b_before = [c.copy() for c in b.to_numpy()]
    x0_before = [c.copy() for c in x0.to_numpy()]
    np.random.seed(1234)
    state = np.random.get_state()
    x, info = tt.amen(A, b, x0=x0, return_info=True, **KW)
    after = np.random.get_state()
    assert state[0] == after[0] and np.array_equal(state[1], after[1]) and state[2:] == after[2:]
    assert all(np.array_equal(u, v) for u, v in zip(a_before, A.to_numpy()))
    assert all(np.array_equal(u, v) for u, v in zip(b_before, b.to_numpy()))
    assert all(np.array_equal(u, v) for u, v in zip(x0_before, x0.to_numpy()))
    assert x is not x0


def test_final_residual_matches_report(tt):
    A_c, b_c = _problem()
    x, info = tt.amen(tt.TensorTrain(A_c), tt.TensorTrain(b_c), return_info=True, **KW)
    host = O.relative_residual(O.Train(A_c), O.Train(b_c), O.Train(x.to_numpy()))
    assert info.residuals[-1] == pytest.approx(host, rel=1e-6)
    from ttnumpy_b200.persistent import amen_persistent

    (r,) = amen_persistent([(A_c, b_c, None, KW)])
    host = O.relative_residual(O.Train(A_c), O.Train(b_c), O.Train(r.x.to_numpy()))
    assert r.info.residuals[-1] == pytest.approx(host, rel=1e-6)
