"""GPU ALS (the drop-in ``als``) against the reference's own results
(golden fixtures made by running ``ttnumpy.solvers.als.als``).

ALS keeps the bonds of its initial guess, so bonds are compared exactly;
the trajectory (sweeps, stop reason, local solve count, residual history)
matches to rounding, and the solution to 1e-8 relative (TT difference).
"""

import numpy as np
import pytest

from conftest import golden_train, load_golden
from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = ["als_qtt_lap1d_o6", "als_lap4_minres", "als_nonsym_gmres"]

# The GMRES case runs its local solves to the default local tolerance
# (1e-8) and its global residual (~4.5e-9) sits at that level: restarted
# GMRES here and SciPy's stop at different iterates within the tolerance, so
# the residual history agrees to 10 % and the solution to 1e-6.
LOOSE = {"als_nonsym_gmres"}


@pytest.fixture(scope="module")
def tt():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ttnumpy_b200

    return ttnumpy_b200


@pytest.mark.parametrize("case", CASES)
def test_als_matches_reference(tt, case):
    data = load_golden(case)
    A_c, _ = golden_train(data, "A")
    b_c, b_oc = golden_train(data, "b")
    x0 = None
    if "x0_n" in data:
        c, oc = golden_train(data, "x0")
        x0 = tt.TensorTrain(c, orth_center=oc)
    args = dict(data["args"])
    x, info = tt.als(tt.TensorTrain(A_c), tt.TensorTrain(b_c, orth_center=b_oc), x0=x0,
                     return_info=True, **args)
    assert x.bonds == [int(v) for v in data["bonds"]]
    assert info.num_sweeps_run == int(data["num_sweeps_run"])
    assert str(info.stop_reason) == str(data["stop_reason"])
    assert info.local_solves == int(data["local_solves"])
    ref = O.Train(golden_train(data, "x")[0])
    got = O.Train(x.to_numpy())
    dist = O.tt_norm(O.add(got, O.scale(ref, -1.0))) / O.tt_norm(ref)
    if case in LOOSE:
        np.testing.assert_allclose(info.residuals, data["residuals"], rtol=0.1)
        assert dist < 1e-6
    else:
        np.testing.assert_allclose(info.residuals, data["residuals"], rtol=1e-5, atol=1e-13)
        assert dist < 1e-8
    assert x.orth_center == 0


def test_als_keeps_inputs(tt):
    data = load_golden("als_lap4_minres")
    A_c, _ = golden_train(data, "A")
    b_c, _ = golden_train(data, "b")
    c, oc = golden_train(data, "x0")
    x0 = tt.TensorTrain(c, orth_center=oc)
    before = [v.copy() for v in x0.to_numpy()]
    x = tt.als(tt.TensorTrain(A_c), tt.TensorTrain(b_c), x0=x0, max_sweeps=1)
    assert all(np.array_equal(u, v) for u, v in zip(before, x0.to_numpy()))
    assert x.bonds == x0.bonds
