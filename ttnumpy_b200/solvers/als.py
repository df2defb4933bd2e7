"""Alternating least squares (ALS) on the GPU, a drop-in for the reference
``als`` (``ttnumpy/solvers/als.py:57-212``).

One-site sweeps with the local solves and centre shifts of ``amen``
(environments, local right-hand side, direct or Krylov local solve, QR
shifts: the same C-ABI kernels) but without the residual train, enrichment
or truncation, so the bonds of ``x0`` never change.  Arguments, defaults,
errors, the stop rule and ``SolverInfo`` are the reference's.
"""

from __future__ import annotations

import logging
import time
from typing import Optional, Tuple, Union

from .. import tensor_train
from ..tensor_train import TensorTrain
from .amen import _Stats, _Sweeper
from .common import (
    LocalSolver,
    SolverInfo,
    StopReason,
    _SolverSettings,
    _validate_solver_inputs,
    relative_residual,
)

logger = logging.getLogger("ttnumpy")

_ENVS = ("A", "b")


def als(A: TensorTrain, b: TensorTrain, x0: Optional[TensorTrain] = None, inplace: bool = False,
        max_sweeps: int = 4, residual_tol: Optional[float] = None,
        stagnation_factor: Union[float, str, None] = "auto",
        local_solver: Union[str, LocalSolver] = "auto", direct_solve_size: int = 1000,
        local_rtol: Optional[float] = None, allow_dense_fallback: bool = False,
        symmetric: bool = False, return_info: bool = False,
        ) -> Union[TensorTrain, Tuple[TensorTrain, SolverInfo]]:
    """ALS for ``A x = b`` on the GPU: the reference ``als``
    (``ttnumpy/solvers/als.py:57-212``) with every contraction and
    factorisation on the device."""
    settings = _SolverSettings.resolve(
        max_sweeps=max_sweeps, residual_tol=residual_tol, stagnation_factor=stagnation_factor,
        local_solver=local_solver, symmetric=symmetric, direct_solve_size=direct_solve_size,
        return_info=return_info, local_rtol=local_rtol,
        allow_dense_fallback=allow_dense_fallback)
    if x0 is None:
        x0 = tensor_train.ones(b.physical_dims(), ranks=b.bonds)
    _validate_solver_inputs(A, b, x0)
    x = x0 if inplace else x0.copy()
    if x.orth_center != 0:
        x.orthonormalize(canonical="right", inplace=True)

    sw = _Sweeper(A, b, x, None, settings, 1, 0.0, None, 1.0)
    d = sw.d
    for i in range(d - 1, -1, -1):  # als.py:144-146
        sw.build_right(i, _ENVS)

    info = SolverInfo()
    b_norm = b.tt_norm() if settings.track_residual else None
    stats = _Stats()
    started = time.perf_counter()
    for sweep in range(settings.max_sweeps):
        for k in range(d - 1):  # als.py:153-170
            sw.build_left(k, _ENVS)
            u, _ = sw.solve_local(k, stats)
            sw.shift_right(x, k, u)
        sw.build_left(d - 1, _ENVS)  # als.py:172-175
        for k in range(d - 1, -1, -1):  # als.py:177-201
            sw.build_right(k, _ENVS)
            u, _ = sw.solve_local(k, stats)
            if k == 0:
                x.cores[0] = u.reshape(u.shape[0], u.shape[1], 1, u.shape[2])
                x.orth_center = 0
            else:
                sw.shift_left(x, k, u)
        sw.check_lu()
        info.num_sweeps_run = sweep + 1
        info.max_bonds.append(max(x.bonds))
        info.local_solves += stats.local_solves
        info.local_fallbacks += stats.local_fallbacks
        info.local_inexact += stats.local_inexact
        stats = _Stats()
        if not settings.track_residual:
            continue
        res = relative_residual(A, b, x, b_norm=b_norm)
        info.residuals.append(res)
        logger.debug("ALS sweep %d/%d: relative residual %.3e, %.3fs", sweep + 1,
                     settings.max_sweeps, res, time.perf_counter() - started)
        if settings.residual_tol is not None and res <= settings.residual_tol:
            info.stop_reason = StopReason.CONVERGED
            break
        if (settings.stagnation_factor is not None and len(info.residuals) >= 2
                and info.residuals[-1] > settings.stagnation_factor * info.residuals[-2]):
            info.stop_reason = StopReason.STAGNATED
            logger.warning("ALS stagnated at sweep %d: relative residual %.3e vs %.3e previous",
                           sweep + 1, info.residuals[-1], info.residuals[-2])
            break
    if return_info:
        return x, info
    return x
