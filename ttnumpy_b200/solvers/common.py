"""Solver vocabulary, settings and the relative residual.

The enums, ``SolverInfo`` and the option rules restate
``ttnumpy/solvers/common.py:36-400`` so that callers see the same names,
values and errors; ``relative_residual`` runs in TT arithmetic on the GPU
(``ttnumpy/solvers/common.py:118-146``).
"""

from __future__ import annotations

import logging
from dataclasses import dataclass, field
from enum import Enum
from typing import List, Optional, Union

import numpy as np

from .. import tensor_train

logger = logging.getLogger("ttnumpy")


class StopReason(str, Enum):
    """Why an iterative TT solve stopped (``common.py:36-53``)."""

    CONVERGED = "converged"
    STAGNATED = "stagnated"
    MAX_SWEEPS = "max_sweeps"

    def __str__(self) -> str:
        return str.__str__(self)


class LocalSolver(str, Enum):
    """Local-system solver selection (``common.py:56-69``)."""

    AUTO = "auto"
    DIRECT = "direct"
    MINRES = "minres"
    GMRES = "gmres"

    def __str__(self) -> str:
        return str.__str__(self)


class TruncationMode(str, Enum):
    """Rule for truncating a solved core (``common.py:72-82``)."""

    RESIDUAL = "residual"
    THRESHOLD = "threshold"

    def __str__(self) -> str:
        return str.__str__(self)


@dataclass
class SolverInfo:
    """Per-solve record with the reference's fields (``common.py:85-115``)."""

    residuals: List[float] = field(default_factory=list)
    num_sweeps_run: int = 0
    stop_reason: StopReason = StopReason.MAX_SWEEPS
    max_bonds: List[int] = field(default_factory=list)
    local_solves: int = 0
    local_fallbacks: int = 0
    local_inexact: int = 0

    @property
    def converged(self) -> bool:
        return self.stop_reason == StopReason.CONVERGED


def relative_residual(A, b, x, b_norm: Optional[float] = None) -> float:
    """``||A x - b|| / ||b||`` in TT arithmetic on the device: Kronecker
    cores of ``A x``, the block sum with ``-b`` and a right QR sweep for the
    norm (``common.py:118-146``)."""
    residual = A.dot(x).add(b.multiply(-1))
    if b_norm is None:
        b_norm = b.tt_norm()
    rn = residual.tt_norm()
    if b_norm == 0.0:
        return rn
    return rn / b_norm


_LOCAL_TOL_FACTOR = 0.1
_DEFAULT_LOCAL_RTOL = 1e-8
_MAX_LOCAL_RESTARTS = 4
_RESTART_RTOL_SHRINK = 1e-2
_DEFAULT_STAGNATION_FACTOR = 0.9
_LOCAL_RATE_REPORT_SHARE = 0.5


@dataclass(frozen=True)
class _SolverSettings:
    """Validated and derived options (``common.py:244-400``)."""

    max_sweeps: int
    residual_tol: Optional[float]
    stagnation_factor: Optional[float]
    iterative_solver: Optional[LocalSolver]
    direct_solve_size: int
    track_residual: bool
    local_rtol: Optional[float]
    allow_dense_fallback: bool = False
    truncation_steps: int = 1

    @property
    def truncation_mode(self) -> TruncationMode:
        return TruncationMode.RESIDUAL if self.residual_tol is not None else TruncationMode.THRESHOLD

    @property
    def truncation_tol(self) -> Optional[float]:
        if self.residual_tol is None:
            return None
        return self.residual_tol / np.sqrt(self.truncation_steps)

    def use_iterative(self, size: int) -> bool:
        return self.iterative_solver is not None and size > self.direct_solve_size

    @classmethod
    def resolve(cls, *, max_sweeps, residual_tol, stagnation_factor, local_solver, symmetric,
                direct_solve_size, return_info, local_rtol=None, allow_dense_fallback=False,
                truncation_steps=1) -> "_SolverSettings":
        if residual_tol is not None and residual_tol <= 0.0:
            raise ValueError(f"residual_tol must be positive, got {residual_tol}")
        if truncation_steps < 1:
            raise ValueError(f"truncation_steps must be positive, got {truncation_steps}")
        if isinstance(stagnation_factor, str):
            if stagnation_factor != "auto":
                raise ValueError("stagnation_factor must be a float in (0, 1], None or "
                                 f"'auto', got {stagnation_factor!r}")
            stagnation_factor = (_DEFAULT_STAGNATION_FACTOR
                                 if residual_tol is not None or return_info else None)
        if stagnation_factor is not None and not 0.0 < stagnation_factor <= 1.0:
            raise ValueError(f"stagnation_factor must be in (0, 1], got {stagnation_factor}")
        track_residual = (return_info or residual_tol is not None
                          or (stagnation_factor is not None and max_sweeps > 1))
        if local_rtol is not None and local_rtol <= 0.0:
            raise ValueError(f"local_rtol must be positive, got {local_rtol}")
        try:
            local_solver = LocalSolver(local_solver)
        except ValueError as exc:
            allowed = ", ".join(repr(m.value) for m in LocalSolver)
            raise ValueError(f"local_solver must be one of {allowed}, got {local_solver!r}") from exc
        if local_solver is LocalSolver.AUTO:
            iterative = LocalSolver.MINRES if symmetric else LocalSolver.GMRES
        elif local_solver is LocalSolver.DIRECT:
            iterative = None
        else:
            iterative = local_solver
        if iterative is None:
            lr = None
        elif local_rtol is not None:
            lr = local_rtol
        elif residual_tol is not None:
            lr = _LOCAL_TOL_FACTOR * residual_tol
        else:
            lr = _DEFAULT_LOCAL_RTOL
        if lr is not None and residual_tol is not None and lr > 0.5 * residual_tol:
            logger.warning("local_rtol %.2e exceeds half of residual_tol %.2e: the local "
                           "solves may be too loose to drive the truncation budget", lr,
                           residual_tol)
        return cls(max_sweeps=max_sweeps, residual_tol=residual_tol,
                   stagnation_factor=stagnation_factor, iterative_solver=iterative,
                   direct_solve_size=direct_solve_size, track_residual=track_residual,
                   local_rtol=lr, allow_dense_fallback=allow_dense_fallback,
                   truncation_steps=truncation_steps)


def _validate_solver_inputs(A, b, x0) -> None:
    """Structural checks of ``A x = b`` (``common.py:684-726``)."""
    if x0.is_ttm():
        raise tensor_train.WrongTTType("Initial guess x0 must be a TensorTrain, not a TTM.")
    if b.is_ttm():
        raise tensor_train.WrongTTType("Right-hand side b must be a TensorTrain, not a TTM.")
    if not A.is_ttm():
        raise tensor_train.WrongTTType("Matrix A must be a TTM, not a TensorTrain.")
    if not len(A) == len(b) == len(x0):
        raise tensor_train.DimensionMismatch(
            "A, b and x0 must have the same number of cores, "
            f"got {len(A)}, {len(b)} and {len(x0)}")
    if A.row_modes != A.col_modes:
        raise tensor_train.DimensionMismatch(
            f"Solver requires a square operator, got row modes {A.row_modes} "
            f"and column modes {A.col_modes}")
    if A.row_modes != b.row_modes:
        raise tensor_train.DimensionMismatch(
            "Row modes of A must match physical dimensions of b: "
            f"{A.row_modes} != {b.row_modes}")
    if A.col_modes != x0.row_modes:
        raise tensor_train.DimensionMismatch(
            "Column modes of A must match physical dimensions of x0: "
            f"{A.col_modes} != {x0.row_modes}")
