"""Modified alternating least squares (MALS) on the GPU, a drop-in for the
reference ``mals`` (``ttnumpy/solvers/mals.py:61-292`` with the two-site
algebra of ``ttnumpy/solvers/two_site.py:28-241``).

Each step solves the projected system of the supercore of sites (k, k+1)
and splits the solution by SVD, which adapts the shared bond.  The
two-site operator ``Psi . A_k . A_{k+1} . Phi`` is the one-site operator of
the merged operator core ``A_k A_{k+1}`` (row modes and column modes of the
pair merged, one device GEMM per pair, cached for the solve), so every
local step runs on the one-site kernels: ``ttb_project`` for the right-hand
side with the merged ``b`` core, ``ttb_local_matrix`` + ``ttb_lu_solve`` or
``ttb_minres`` / ``ttb_gmres`` for the solve, ``ttb_svd`` for the split and
``ttb_local_apply`` + ``ttb_rank_residual`` (or ``ttb_rank_threshold``)
for the rank.  Arguments, defaults, errors, the stop rule and
``SolverInfo`` are the reference's.
"""

from __future__ import annotations

import logging
import time
from typing import Optional, Tuple, Union

import torch

from .. import kernels as K
from .. import tensor_train
from ..tensor_train import TensorTrain, _merge_cores
from .amen import _c3, _Stats, _Sweeper, _take
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


class _PairSweeper(_Sweeper):
    """The AMEn sweeper's local steps on the supercore of sites (k, k+1).

    ``bonds`` holds the bond dimensions of the solve: mid-sweep the core
    right of the last split still carries its old left bond, so the cores
    alone do not give them.  ``center`` is the (site, block) pair left by the
    last split, the warm start's stand-in for that stale core
    (``two_site.py:130-153``)."""

    def __init__(self, A: TensorTrain, b: TensorTrain, x: TensorTrain,
                 settings: _SolverSettings, error_threshold: float, max_rank: Optional[int],
                 residual_damp: float):
        super().__init__(A, b, x, None, settings, 1, error_threshold, max_rank, residual_damp)
        self.bonds = list(x.bonds)
        self.center: Optional[Tuple[int, torch.Tensor]] = None
        self._A2 = {}
        self._b2 = {}

    def _pair_A(self, k: int) -> torch.Tensor:
        if k not in self._A2:
            self._A2[k] = _merge_cores([self.A.cores[k], self.A.cores[k + 1]])
        return self._A2[k]

    def _pair_b(self, k: int) -> torch.Tensor:
        if k not in self._b2:
            self._b2[k] = _c3(_merge_cores([self.b.cores[k], self.b.cores[k + 1]]))
        return self._b2[k]

    def op(self, k: int):
        return self.left["A"][k], self._pair_A(k), self.right["A"][k + 1]

    def rhs_parts(self, k: int):
        return self.left["b"][k], self._pair_b(k), self.right["b"][k + 1]

    def local_shape(self, k: int) -> Tuple[int, int, int]:
        x = self.x
        return self.bonds[k], x.row_modes[k] * x.row_modes[k + 1], self.bonds[k + 2]

    def warm_start(self, k: int, u: torch.Tensor) -> bool:
        """The current supercore, or False when the shared bond of the two
        blocks disagrees or the supercore has the wrong size."""
        left, right = _c3(self.x.cores[k]), _c3(self.x.cores[k + 1])
        if self.center is not None:
            site, block = self.center
            if site == k:
                left = block
            elif site == k + 1:
                right = block
        if left.shape[2] != right.shape[0]:
            return False
        rows = left.shape[0] * left.shape[1]
        cols = right.shape[1] * right.shape[2]
        if rows * cols != u.numel():
            return False
        K.gemm(left.reshape(rows, left.shape[2]), right.reshape(right.shape[0], cols),
               u.view(rows, cols))
        return True

    def solve_pair(self, k: int, stats: _Stats):
        """``_solve_local_two_site`` (``two_site.py:156-241``): solve, split
        the supercore (bond * mode_k, mode_{k+1} * bond) by SVD and choose
        the rank of the shared bond.  Returns (U, S, Vh, rank)."""
        u, b_loc = self.solve_local(k, stats)
        rows = self.bonds[k] * self.x.row_modes[k]
        U, S, Vh = K.svd(u.reshape(rows, -1))
        rank = self._choose_rank(k, u, b_loc, U, S, Vh, stats)
        return U, S, Vh, rank


def mals(A: TensorTrain, b: TensorTrain, x0: Optional[TensorTrain] = None, inplace: bool = False,
         max_rank: Optional[int] = None, max_sweeps: int = 2,
         residual_tol: Optional[float] = None, residual_damp: float = 2.0,
         stagnation_factor: Union[float, str, None] = "auto", error_threshold: float = 1e-7,
         local_solver: Union[str, LocalSolver] = "auto", direct_solve_size: int = 1000,
         local_rtol: Optional[float] = None, allow_dense_fallback: bool = False,
         symmetric: bool = False, return_info: bool = False,
         ) -> Union[TensorTrain, Tuple[TensorTrain, SolverInfo]]:
    """MALS for ``A x = b`` on the GPU: the reference ``mals``
    (``ttnumpy/solvers/mals.py:61-292``) with every contraction,
    factorisation and rank decision on the device."""
    if max_rank is not None and max_rank <= 0:
        raise ValueError(f"max_rank must be a positive integer, got {max_rank}")
    if residual_damp < 1.0:
        raise ValueError(f"residual_damp must be >= 1, got {residual_damp}")
    settings = _SolverSettings.resolve(
        max_sweeps=max_sweeps, residual_tol=residual_tol, stagnation_factor=stagnation_factor,
        local_solver=local_solver, symmetric=symmetric, direct_solve_size=direct_solve_size,
        return_info=return_info, local_rtol=local_rtol,
        allow_dense_fallback=allow_dense_fallback, truncation_steps=max(2 * len(A) - 3, 1))
    if x0 is None:
        x0 = tensor_train.ones(b.physical_dims(), ranks=b.bonds)
    _validate_solver_inputs(A, b, x0)
    x = x0 if inplace else x0.copy()
    if x.orth_center != 0:
        x.orthonormalize(canonical="right", inplace=True)

    sw = _PairSweeper(A, b, x, settings, error_threshold, max_rank, residual_damp)
    d = sw.d
    for i in range(d - 1, 0, -1):  # mals.py:196-198
        sw.build_right(i, _ENVS)

    info = SolverInfo()
    b_norm = b.tt_norm() if settings.track_residual else None
    stats = _Stats()
    started = time.perf_counter()
    bonds = sw.bonds
    for sweep in range(settings.max_sweeps):
        for k in range(d - 1):  # mals.py:216-249
            sw.build_left(k, _ENVS)
            if k == d - 2:
                continue
            U, S, Vh, nb = sw.solve_pair(k, stats)
            n0, n1 = x.row_modes[k], x.row_modes[k + 1]
            block = K.empty(nb, n1, bonds[k + 2])
            K.copy_(block.view(nb, -1), Vh[:nb], scale=S[:nb], scale_axis=0)
            sw.center = (k + 1, block)
            x.cores[k] = _take(U[:, :nb]).view(bonds[k], n0, 1, nb)
            bonds[k + 1] = nb
            x.orth_center = k + 1
        for k in range(d - 2, -1, -1):  # mals.py:252-283
            sw.build_right(k + 1, _ENVS)
            U, S, Vh, nb = sw.solve_pair(k, stats)
            n0, n1 = x.row_modes[k], x.row_modes[k + 1]
            block = K.empty(bonds[k], n0, nb)
            K.copy_(block.view(-1, nb), U[:, :nb], scale=S[:nb], scale_axis=1)
            sw.center = (k, block)
            x.cores[k + 1] = _take(Vh[:nb]).view(nb, n1, 1, bonds[k + 2])
            bonds[k + 1] = nb
            if k == 0:
                x.cores[0] = block.view(bonds[0], n0, 1, nb)
            x.orth_center = k
        sw.check_lu()
        info.num_sweeps_run = sweep + 1
        info.max_bonds.append(max(bonds))
        info.local_solves += stats.local_solves
        info.local_fallbacks += stats.local_fallbacks
        info.local_inexact += stats.local_inexact
        stats = _Stats()
        if not settings.track_residual:
            continue
        res = relative_residual(A, b, x, b_norm=b_norm)
        info.residuals.append(res)
        logger.debug("MALS sweep %d/%d: relative residual %.3e, max bond %d, %.3fs", sweep + 1,
                     settings.max_sweeps, res, max(bonds), time.perf_counter() - started)
        if settings.residual_tol is not None and res <= settings.residual_tol:
            info.stop_reason = StopReason.CONVERGED
            break
        if (settings.stagnation_factor is not None and len(info.residuals) >= 2
                and info.residuals[-1] > settings.stagnation_factor * info.residuals[-2]):
            info.stop_reason = StopReason.STAGNATED
            logger.warning("MALS stagnated at sweep %d: relative residual %.3e vs %.3e previous",
                           sweep + 1, info.residuals[-1], info.residuals[-2])
            break
    if return_info:
        return x, info
    return x
