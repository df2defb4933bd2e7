"""AMEn one-site sweep with residual enrichment, on the GPU.

Drop-in for the reference ``amen`` (``ttnumpy/solvers/amen.py:395-725``):
same signature, defaults, validation, stopping rules and ``SolverInfo``.
The control flow (sweeps, sites, rank decisions) runs on the host; every
numeric step runs on the device through libttb200:

* environments (``common.py:149-217``): ``ttb_env_update``, five per site,
  one grouped call;
* local right-hand side (``one_site.py:27-46``): ``ttb_project``;
* local solve (``common.py:729-809``): ``ttb_local_matrix`` +
  ``ttb_lu_solve`` for systems of at most ``direct_solve_size`` unknowns,
  else ``ttb_minres`` / ``ttb_gmres`` on the matrix-free operator with the
  reference's true-residual restarts;
* residual core z (``amen.py:109-159``): ``ttb_project`` +
  ``ttb_local_apply`` with a rectangular frame;
* truncation (``amen.py:227-322``, ``common.py:812-929``): ``ttb_svd``,
  then ``ttb_local_apply`` on the rank-one terms and
  ``ttb_rank_residual`` (or ``ttb_rank_threshold``);
* enrichment and centre shifts (``amen.py:325-392``,
  ``one_site.py:181-209``): ``ttb_copy``, ``ttb_gemm``, ``ttb_qr``.

Only the chosen rank (one int per site) and the Krylov stop flags come back
to the host inside a sweep; the relative residual comes back once per sweep.
"""

from __future__ import annotations

import contextlib
import logging
import math
import threading
import time
from typing import Optional, Tuple, Union

import numpy as np
import torch

from .. import kernels as K
from .. import tensor_train
from ..tensor_train import TensorTrain, _apply_left, _apply_right
from .common import (
    LocalSolver,
    SolverInfo,
    StopReason,
    TruncationMode,
    _MAX_LOCAL_RESTARTS,
    _RESTART_RTOL_SHRINK,
    _SolverSettings,
    _validate_solver_inputs,
    relative_residual,
)

logger = logging.getLogger("ttnumpy")


class _TimeLimit(threading.local):
    seconds: Optional[float] = None


_TIME_LIMIT = _TimeLimit()


@contextlib.contextmanager
def solve_time_limit(seconds: Optional[float]):
    """Within the block, an ``amen`` call on this thread stops after the
    first sweep that ends more than ``seconds`` after the call started (the
    per-solve time limit of the reference's benchmark runner,
    ``benchmarks/poisson.py:95-143``); its ``SolverInfo`` then reports
    ``max_sweeps`` with the sweeps run so far.  Outside such a block the
    sweep count alone bounds a solve, as in the reference."""
    prev = _TIME_LIMIT.seconds
    _TIME_LIMIT.seconds = seconds
    try:
        yield
    finally:
        _TIME_LIMIT.seconds = prev


def _c3(core: torch.Tensor) -> torch.Tensor:
    """(r, n, r') view of a TT core (r, n, 1, r')."""
    return core.reshape(core.shape[0], core.shape[1], core.shape[3])


def _ones(*shape) -> torch.Tensor:
    return K.fill_(K.empty(*shape), 1.0)


def _take(view: torch.Tensor) -> torch.Tensor:
    """Contiguous copy of a strided view, made by the copy kernel."""
    out = K.empty(*view.shape)
    K.copy_(out, view)
    return out


class _Stats:
    """Per-sweep tallies (``common.py:403-444``)."""

    def __init__(self):
        self.local_solves = 0
        self.local_fallbacks = 0
        self.local_inexact = 0
        self.rank_decisions = 0
        self.rank_capped = 0


class _Sweeper:
    """State of one AMEn solve on the device."""

    ENVS = ("A", "b", "zb", "zAx", "xz")

    def __init__(self, A: TensorTrain, b: TensorTrain, x: TensorTrain, z: TensorTrain,
                 settings: _SolverSettings, kickrank: int, error_threshold: float,
                 max_rank: Optional[int], residual_damp: float):
        self.A, self.b, self.x, self.z = A, b, x, z
        self.st = settings
        self.kick = kickrank
        self.eth = error_threshold
        self.max_rank = max_rank
        self.damp = residual_damp
        d = len(A)
        self.d = d
        self.left = {k: [None] * d for k in self.ENVS}
        self.right = {k: [None] * d for k in self.ENVS}
        self.rank_dev = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.lu_info = []

    # -- environments -------------------------------------------------------

    def _pairs(self):
        x, z, b, A = self.x, self.z, self.b, self.A
        return {"A": (x, x, A), "b": (x, b, None), "zb": (z, b, None), "zAx": (z, x, A),
                "xz": (x, z, None)}

    def build_left(self, k: int, names=ENVS) -> None:
        pairs = self._pairs()
        descs, outs = [], []
        for name in names:
            frame, target, op = pairs[name]
            if k == 0:
                self.left[name][0] = _ones(1, 1, 1) if op is not None else _ones(1, 1)
                continue
            env = self.left[name][k - 1]
            fc, tc = _c3(frame.cores[k - 1]), _c3(target.cores[k - 1])
            opc = op.cores[k - 1] if op is not None else None
            if op is not None:
                out = K.empty(tc.shape[2], opc.shape[3], fc.shape[2])
            else:
                out = K.empty(tc.shape[2], fc.shape[2])
            descs.append(K.env_desc(0, env, fc, tc, out, opc))
            outs.append((name, out))
        K.env_update(descs)
        for name, out in outs:
            self.left[name][k] = out

    def build_right(self, k: int, names=ENVS) -> None:
        pairs = self._pairs()
        descs, outs = [], []
        for name in names:
            frame, target, op = pairs[name]
            if k == self.d - 1:
                self.right[name][k] = _ones(1, 1, 1) if op is not None else _ones(1, 1)
                continue
            env = self.right[name][k + 1]
            fc, tc = _c3(frame.cores[k + 1]), _c3(target.cores[k + 1])
            opc = op.cores[k + 1] if op is not None else None
            if op is not None:
                out = K.empty(tc.shape[0], opc.shape[0], fc.shape[0])
            else:
                out = K.empty(tc.shape[0], fc.shape[0])
            descs.append(K.env_desc(1, env, fc, tc, out, opc))
            outs.append((name, out))
        K.env_update(descs)
        for name, out in outs:
            self.right[name][k] = out

    # -- local algebra ------------------------------------------------------

    # The local system at site k is described by four hooks, so that a
    # two-site sweep can reuse every local step with a merged supercore.

    def op(self, k: int):
        """(left environment, operator core, right environment) of the local
        operator at site k."""
        return self.left["A"][k], self.A.cores[k], self.right["A"][k]

    def rhs_parts(self, k: int):
        """(left environment, right-hand-side core, right environment) of
        the local right-hand side at site k."""
        return self.left["b"][k], _c3(self.b.cores[k]), self.right["b"][k]

    def local_shape(self, k: int) -> Tuple[int, int, int]:
        c = self.x.cores[k]
        return c.shape[0], c.shape[1], c.shape[3]

    def warm_start(self, k: int, u: torch.Tensor) -> bool:
        """Fill ``u`` with the Krylov initial guess; False starts from zero."""
        K.copy_(u, _c3(self.x.cores[k]))  # the current centre core
        return True

    def local_rhs(self, k: int) -> torch.Tensor:
        out = K.empty(*self.local_shape(k))
        left, core, right = self.rhs_parts(k)
        K.project([K.project_desc(left, core, right, out)])
        return out

    def apply_A(self, k: int, u: torch.Tensor, out: torch.Tensor, cols: int = 1, alpha=1.0,
                beta=0.0) -> torch.Tensor:
        left, core, right = self.op(k)
        K.local_apply([K.local_desc(left, core, right, u, out, cols, alpha, beta)])
        return out

    def solve_local(self, k: int, stats: _Stats) -> Tuple[torch.Tensor, torch.Tensor]:
        """``_solve_local_one_site`` + ``_solve_local_system``
        (``one_site.py:118-178``, ``common.py:729-809``)."""
        shape = self.local_shape(k)
        size = shape[0] * shape[1] * shape[2]
        b_loc = self.local_rhs(k)
        st = self.st
        if not st.use_iterative(size):
            return self._direct(k, b_loc), b_loc
        method = "minres" if st.iterative_solver is LocalSolver.MINRES else "gmres"
        u = K.empty(*shape)
        warm = self.warm_start(k, u)
        if not warm:
            K.fill_(u, 0.0)
        rtol = st.local_rtol
        nb = K.empty(2)
        K.norm_into(nb[0:1], b_loc)
        tmp = K.empty(*shape)
        left, core, right = self.op(k)
        for _ in range(_MAX_LOCAL_RESTARTS):
            K.krylov(method, left, core, right, b_loc, u, rtol, warm)
            warm = True
            self.apply_A(k, u, tmp)
            K.norm_into(nb[1:2], tmp, b_loc)
            bn, rn = nb.tolist()
            if rn <= st.local_rtol * bn:
                stats.local_solves += 1
                return u, b_loc
            rtol = max(rtol * _RESTART_RTOL_SHRINK, 1e-15)
        stats.local_solves += 1
        if not st.allow_dense_fallback:
            stats.local_inexact += 1
            return u, b_loc
        stats.local_fallbacks += 1
        return self._direct(k, b_loc), b_loc

    def _direct(self, k: int, b_loc: torch.Tensor) -> torch.Tensor:
        M = K.local_matrix(*self.op(k))
        u = _take(b_loc)
        info = torch.zeros(1, dtype=torch.int32, device="cuda")
        K.lu_solve_(M, u.reshape(-1), info)
        self.lu_info.append(info)
        return u

    def residual_core(self, k: int, x_core: torch.Tensor) -> torch.Tensor:
        """z's core at k: P_z(b) - P_z(A x) (``amen.py:109-159``)."""
        zl, zr = self.left["zb"][k].shape[1], self.right["zb"][k].shape[1]
        n = self.b.cores[k].shape[1]
        out = K.empty(zl, n, zr)
        K.project([K.project_desc(self.left["zb"][k], _c3(self.b.cores[k]), self.right["zb"][k],
                                  out)])
        K.local_apply([K.local_desc(self.left["zAx"][k], self.A.cores[k], self.right["zAx"][k],
                                    x_core, out, 1, -1.0, 1.0)])
        return out

    # -- truncation ---------------------------------------------------------

    def _choose_rank(self, k, u, b_loc, U, S, Vh, stats: _Stats) -> int:
        """``_choose_truncation_rank`` (``common.py:888-929``)."""
        p = S.numel()
        if self.st.truncation_mode is TruncationMode.RESIDUAL:
            limit = p if self.max_rank is None else min(p, self.max_rank)
            size = u.numel()
            exact = K.empty(1)
            tmp = K.empty(*u.shape)
            self.apply_A(k, u, tmp)
            K.norm_into(exact, tmp, b_loc)
            with K.arena().scope():
                ar = K.arena()
                terms = ar.take(limit * size)[: limit * size].view(limit, U.shape[0], Vh.shape[1])
                svh = ar.take(limit * Vh.shape[1])[: limit * Vh.shape[1]].view(limit, Vh.shape[1])
                K.copy_(svh, Vh[:limit], scale=S[:limit], scale_axis=0)
                # term c = U[:, c] (outer) S[c] Vh[c, :]
                K.gemm(U.t()[:limit].unsqueeze(2), svh.unsqueeze(1), terms)
                contrib = ar.take(limit * size)[: limit * size].view(limit, size)
                self.apply_A(k, terms, contrib, cols=limit)
                K.rank_residual(contrib, b_loc, exact, S, limit, self.damp, self.st.truncation_tol,
                                self.rank_dev)
                rank = int(self.rank_dev.item())
            capped = rank == limit and self.max_rank is not None and self.max_rank < p
        else:
            K.rank_threshold(S, 0, self.eth, self.max_rank, self.rank_dev)
            rank = int(self.rank_dev.item())
            capped = self.max_rank is not None and rank == self.max_rank and p > self.max_rank
        stats.rank_decisions += 1
        stats.rank_capped += int(capped)
        return rank

    def truncate_right(self, k, u, b_loc, stats):
        """``_truncate_core_right`` (``amen.py:227-275``): (core, carry)."""
        rl, n, rr = u.shape
        U, S, Vh = K.svd(u.reshape(rl * n, rr))
        rank = self._choose_rank(k, u, b_loc, U, S, Vh, stats)
        core = _take(U[:, :rank]).reshape(rl, n, rank)
        carry = K.empty(rank, rr)
        K.copy_(carry, Vh[:rank], scale=S[:rank], scale_axis=0)
        return core, carry

    def truncate_left(self, k, u, b_loc, stats):
        """``_truncate_core_left`` (``amen.py:278-322``): (core, carry)."""
        rl, n, rr = u.shape
        U, S, Vh = K.svd(u.reshape(rl, n * rr))
        rank = self._choose_rank(k, u, b_loc, U, S, Vh, stats)
        core = _take(Vh[:rank]).reshape(rank, n, rr)
        carry = K.empty(rl, rank)
        K.copy_(carry, U[:, :rank], scale=S[:rank], scale_axis=1)
        return core, carry

    # -- centre shifts and enrichment --------------------------------------

    @staticmethod
    def shift_right(t: TensorTrain, k: int, core: torch.Tensor) -> None:
        """``_shift_center_right`` (``one_site.py:181-193``)."""
        rl, n, rr = core.shape
        q, r = K.qr(core.reshape(rl * n, rr))
        t.cores[k] = q.reshape(rl, n, 1, q.shape[1])
        t.cores[k + 1] = _apply_left(r, t.cores[k + 1])
        t.orth_center = k + 1

    @staticmethod
    def shift_left(t: TensorTrain, k: int, core: torch.Tensor) -> None:
        """``_shift_center_left`` (``one_site.py:196-209``)."""
        rl, n, rr = core.shape
        p = min(rl, n * rr)
        qt = K.empty(p, n * rr)
        _, r = K.qr(core.reshape(rl, n * rr).t(), q_out=qt.t())
        t.cores[k] = qt.reshape(p, n, 1, rr)
        t.cores[k - 1] = _apply_right(t.cores[k - 1], r.t())
        t.orth_center = k - 1

    def enrich_right(self, k, core, carry, z_new, stats) -> None:
        """Block, zero-padded carry and QR shift (``amen.py:325-360, 626``)."""
        x = self.x
        rl, n, rank = core.shape
        zl, _, zr = z_new.shape
        enriched = K.empty(rl, n, rank + zr)
        # block (rl, n*zr) = lxz^T (rl, zl) @ z_new (zl, n*zr)
        K.copy_(enriched[:, :, :rank], core)
        block = K.empty(rl, n, zr)
        K.gemm(self.left["xz"][k].t(), z_new.reshape(zl, n * zr), block.view(rl, n * zr))
        K.copy_(enriched[:, :, rank:], block)
        nxt = x.cores[k + 1]
        padded = K.empty(rank + zr, *nxt.shape[1:])
        K.fill_(padded[rank:], 0.0)
        K.gemm(carry, nxt.reshape(nxt.shape[0], -1), padded[:rank].view(rank, -1))
        x.cores[k + 1] = padded
        self.shift_right(x, k, enriched)
        if self.max_rank is not None and x.cores[k].shape[3] > self.max_rank:
            x.cores[k] = _take(x.cores[k][:, :, :, : self.max_rank])
            x.cores[k + 1] = _take(x.cores[k + 1][: self.max_rank])

    def enrich_left(self, k, core, carry, z_new, stats) -> None:
        """Mirror for the backward sweep (``amen.py:363-392, 703``)."""
        x = self.x
        rank, n, rr = core.shape
        zl, _, zr = z_new.shape
        enriched = K.empty(rank + zl, n, rr)
        K.copy_(enriched[:rank], core)
        # block (zl, n, rr) = z_new (zl*n, zr) @ rxz (zr, rr)
        K.gemm(z_new.reshape(zl * n, zr), self.right["xz"][k],
               enriched[rank:].view(zl * n, rr))
        prv = x.cores[k - 1]
        rl = carry.shape[0]
        padded = K.empty(*prv.shape[:3], rank + zl)
        K.fill_(padded[..., rank:], 0.0)
        K.gemm(prv.reshape(-1, rl), carry, padded[..., :rank].view(-1, rank))
        x.cores[k - 1] = padded
        self.shift_left(x, k, enriched)
        if self.max_rank is not None and x.cores[k].shape[0] > self.max_rank:
            x.cores[k] = _take(x.cores[k][: self.max_rank])
            x.cores[k - 1] = _take(x.cores[k - 1][..., : self.max_rank])

    # -- residual train -----------------------------------------------------

    def fit_residual(self, sweeps: int = 1) -> None:
        """ALS fit of z to ``b - A x`` (``amen.py:162-224``)."""
        d = self.d
        names = ("zb", "zAx")
        for i in range(d - 1, -1, -1):
            self.build_right(i, names)
        for _ in range(sweeps):
            for k in range(d - 1):
                self.build_left(k, names)
                core = self.residual_core(k, _c3(self.x.cores[k]))
                self.shift_right(self.z, k, core)
            self.build_left(d - 1, names)
            for k in range(d - 1, -1, -1):
                self.build_right(k, names)
                core = self.residual_core(k, _c3(self.x.cores[k]))
                if k > 0:
                    self.shift_left(self.z, k, core)
                else:
                    self.z.cores[0] = core.reshape(1, core.shape[1], 1, core.shape[2])
                    self.z.orth_center = 0

    # -- one sweep ----------------------------------------------------------

    def sweep(self, stats: _Stats) -> None:
        d, x, z = self.d, self.x, self.z
        for k in range(d - 1):
            self.build_left(k)
            u, b_loc = self.solve_local(k, stats)
            z_new = self.residual_core(k, u)
            core, carry = self.truncate_right(k, u, b_loc, stats)
            self.enrich_right(k, core, carry, z_new, stats)
            self.shift_right(z, k, z_new)
        self.build_left(d - 1)
        for k in range(d - 1, -1, -1):
            self.build_right(k)
            u, b_loc = self.solve_local(k, stats)
            z_new = self.residual_core(k, u)
            if k == 0:
                x.cores[0] = u.reshape(1, u.shape[1], 1, u.shape[2])
                x.orth_center = 0
                z.cores[0] = z_new.reshape(1, z_new.shape[1], 1, z_new.shape[2])
                z.orth_center = 0
            else:
                core, carry = self.truncate_left(k, u, b_loc, stats)
                self.enrich_left(k, core, carry, z_new, stats)
                self.shift_left(z, k, z_new)

    def check_lu(self) -> None:
        if not self.lu_info:
            return
        infos = torch.cat(self.lu_info).cpu().tolist()
        self.lu_info = []
        bad = [i for i in infos if i != 0]
        if bad:
            raise np.linalg.LinAlgError(f"local system is singular (zero pivot {bad[0]})")


def amen(A: TensorTrain, b: TensorTrain, x0: Optional[TensorTrain] = None, inplace: bool = False,
         kickrank: int = 4, error_threshold: float = 1e-7, max_rank: Optional[int] = None,
         max_sweeps: int = 1, residual_tol: Optional[float] = None, residual_damp: float = 2.0,
         stagnation_factor: Union[float, str, None] = "auto",
         local_solver: Union[str, LocalSolver] = "auto", direct_solve_size: int = 1000,
         local_rtol: Optional[float] = None, allow_dense_fallback: bool = False,
         symmetric: bool = False, return_info: bool = False, seed: Optional[int] = None,
         ) -> Union[TensorTrain, Tuple[TensorTrain, SolverInfo]]:
    """Alternating Minimal Energy (AMEn) method for ``A x = b`` on the GPU.

    Arguments, defaults, errors and results are those of the reference
    ``amen`` (``ttnumpy/solvers/amen.py:395-514``); see the module
    docstring for where each step runs.
    """
    if kickrank <= 0:
        raise ValueError(f"kickrank must be a positive integer, got {kickrank}")
    if max_rank is not None and max_rank <= 0:
        raise ValueError(f"max_rank must be a positive integer, got {max_rank}")
    if residual_damp < 1.0:
        raise ValueError(f"residual_damp must be >= 1, got {residual_damp}")
    settings = _SolverSettings.resolve(
        max_sweeps=max_sweeps, residual_tol=residual_tol, stagnation_factor=stagnation_factor,
        local_solver=local_solver, symmetric=symmetric, direct_solve_size=direct_solve_size,
        return_info=return_info, local_rtol=local_rtol,
        allow_dense_fallback=allow_dense_fallback, truncation_steps=max(2 * (A.n_cores - 1), 1))
    if x0 is None:
        x0 = tensor_train.ones(b.physical_dims(), ranks=b.bonds)
    _validate_solver_inputs(A, b, x0)
    x = x0 if inplace else x0.copy()
    if x.orth_center != 0:
        x.orthonormalize(canonical="right", inplace=True)

    # z: random rank-kickrank start drawn on the host like the reference
    # (amen.py:80-106), right-orthonormalised on the device
    z = tensor_train.rand(b.physical_dims(), ranks=kickrank, seed=seed)
    z.orthonormalize(canonical="right", inplace=True)

    sw = _Sweeper(A, b, x, z, settings, kickrank, error_threshold, max_rank, residual_damp)
    sw.fit_residual(1)
    for i in range(sw.d - 1, -1, -1):
        sw.build_right(i)

    info = SolverInfo()
    b_norm = b.tt_norm() if settings.track_residual else None
    stats = _Stats()
    started = time.perf_counter()
    for sweep in range(settings.max_sweeps):
        sw.sweep(stats)
        sw.check_lu()
        info.num_sweeps_run = sweep + 1
        info.max_bonds.append(max(x.bonds))
        info.local_solves += stats.local_solves
        info.local_fallbacks += stats.local_fallbacks
        info.local_inexact += stats.local_inexact
        if stats.local_inexact:
            logger.debug("AMEn sweep %d: %d/%d iterative local solves missed local_rtol %.2e",
                         sweep + 1, stats.local_inexact, stats.local_solves, settings.local_rtol)
        stats = _Stats()
        if not settings.track_residual:
            continue
        res = relative_residual(A, b, x, b_norm=b_norm)
        info.residuals.append(res)
        logger.debug("AMEn sweep %d/%d: relative residual %.3e, max bond %d, %.3fs", sweep + 1,
                     settings.max_sweeps, res, max(x.bonds), time.perf_counter() - started)
        if settings.residual_tol is not None and res <= settings.residual_tol:
            info.stop_reason = StopReason.CONVERGED
            break
        if (settings.stagnation_factor is not None and len(info.residuals) >= 2
                and info.residuals[-1] > settings.stagnation_factor * info.residuals[-2]):
            info.stop_reason = StopReason.STAGNATED
            logger.warning("AMEn stagnated at sweep %d: relative residual %.3e vs %.3e previous",
                           sweep + 1, info.residuals[-1], info.residuals[-2])
            break
        limit = _TIME_LIMIT.seconds
        if limit is not None and time.perf_counter() - started > limit:
            logger.warning("AMEn stopped at sweep %d by the time limit of %.1fs", sweep + 1, limit)
            break

    # amen.py:710-720: bonds above the product of the modes to their left
    d = len(x)
    redundant = [k for k in range(1, d) if x.bonds[k] > math.prod(x.row_modes[:k])]
    if redundant:
        x.orthonormalize(canonical="left", center_position=redundant[-1], inplace=True)
        x.orthonormalize(canonical="right", center_position=0, inplace=True)
    if info.residuals:
        logger.info("AMEn stopped after %d sweep(s) (%s), relative residual %.3e",
                    info.num_sweeps_run, info.stop_reason, info.residuals[-1])
        if settings.residual_tol is not None and info.stop_reason is StopReason.MAX_SWEEPS:
            logger.warning("AMEn did not reach residual_tol %.2e after %d sweep(s) (final "
                           "relative residual %.3e)", settings.residual_tol,
                           info.num_sweeps_run, info.residuals[-1])
    if return_info:
        return x, info
    return x
