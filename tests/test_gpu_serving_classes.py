"""AMEn on the request classes of the serving mix at their full sizes, on
the persistent kernel, against runs of the reference itself
(``tests/golden/amen_c5_*.npz``, made by ``make_golden.py serving``):
parametric diffusion with mode size 64 and d up to 12, and the large class
(d = 24, n = 64, random rank-8 right-hand side, on which the reference's
own local solves all stop inexact and the residual stalls near 0.13).

The inputs are regenerated from the stored draw (``problems.py``).  The
solutions are compared through quantities that do not depend on QR/SVD
signs: their norm and inner products with seeded probe trains, beside the
per-sweep residual history, the bonds and the stop reason; the final
residual is recomputed by the host oracle.  Runs below convergence
(``max_sweeps`` smaller than the solve needs) compare a prefix of the
reference's trajectory.

At these sizes the sweep's rank decisions sit on flat residual-budget
thresholds, and the trajectory depends on rounding: the reference itself,
re-run on theta perturbed by one part in 1e15, moves its first-sweep
residual of the d = 8, n = 64 case from 0.066 to 0.080, and two runs of it
that differ only in memory alignment (OpenBLAS kernels) gave 0.066 and 0.062.
So the comparison is by outcome, not step by step: the same stop reason and
sweep count, residuals of the same size sweep by sweep (within a factor 3),
bonds within a quarter of the reference's, and solutions whose norm and
probe inner products agree far more closely than their residuals.
"""

import numpy as np
import pytest

from conftest import load_golden
from oracle import tt_oracle as O
from ttnumpy_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = ["amen_c5_diffusion_d4_n64", "amen_c5_diffusion_d8_n64", "amen_c5_diffusion_d12_n32",
         "amen_c5_large"]


@pytest.fixture(scope="module")
def pers():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ttnumpy_b200 import persistent

    return persistent


def golden_problem(case):
    data = load_golden(case)
    args = dict(data["args"])
    kind, d, n = args.pop("kind"), args.pop("d"), args.pop("n")
    theta = np.asarray(data["theta"])
    assert len(theta) == d
    if kind == "diffusion":
        p = P.parametric_diffusion(d, n, theta)
    else:
        p = P.large_diffusion(theta, int(data["rhs_seed"]), n)
    return p, args, data


def fingerprint(x_cores, data, modes):
    """Norm and probe inner products of a solution, relative gaps to the
    reference's."""
    norm = np.sqrt(O.inner(x_cores, x_cores))
    probes = np.array([O.inner(x_cores, P.random_tt(modes, 2, seed=int(s)))
                       for s in data["probe_seeds"]])
    ref = np.asarray(data["probes"])
    return (abs(norm - float(data["x_norm"])) / float(data["x_norm"]),
            float(np.max(np.abs(probes - ref) / np.abs(ref))))


@pytest.mark.parametrize("case", CASES)
def test_serving_class_matches_reference(pers, case):
    p, args, data = golden_problem(case)
    res = pers.amen_persistent([(p.A, p.b, None, args)], rmax=96)[0]
    assert res.status == 0, pers.STATUS.get(res.status)
    info = res.info
    ref = np.asarray(data["residuals"])
    modes = [c.shape[1] for c in p.b]
    xs = res.x.to_numpy()
    d_norm, d_probe = fingerprint(xs, data, modes)
    host = O.relative_residual(O.Train(p.A), O.Train(p.b), O.Train(xs))
    print(f"{case}: sweeps {info.num_sweeps_run}/{int(data['num_sweeps_run'])} "
          f"residuals {np.array(info.residuals)} ref {ref} bonds {res.x.bonds} ref "
          f"{list(data['bonds'])} norm gap {d_norm:.2e} probe gap {d_probe:.2e} host {host:.3e}")
    # the device's reported final residual is the host oracle's
    assert info.residuals[-1] == pytest.approx(host, rel=1e-6)
    assert str(info.stop_reason) == str(data["stop_reason"])
    if str(data["stop_reason"]) == "converged":
        assert host <= args["residual_tol"] * 1.05
        assert abs(info.num_sweeps_run - int(data["num_sweeps_run"])) <= 1
        assert d_norm < 1e-6 and d_probe < 1e-5
        return
    assert info.num_sweeps_run == int(data["num_sweeps_run"])
    ratio = np.asarray(info.residuals) / ref
    assert np.all(ratio < 3.0) and np.all(ratio > 1.0 / 3.0), ratio
    bonds, rbonds = np.array(res.x.bonds), np.asarray(data["bonds"])
    assert np.all(np.abs(bonds - rbonds) <= np.maximum(2, rbonds // 4)), (bonds, rbonds)
    # solutions of a run stopped early differ by about their residual
    tol = 1e-3 + 10.0 * float(ref[-1])
    assert d_norm < tol and d_probe < tol, (d_norm, d_probe)
