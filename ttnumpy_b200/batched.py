"""Batched AMEn: many independent solves advanced in lockstep on one GPU.

Each solve's AMEn program is the reference algorithm
(``ttnumpy/solvers/amen.py:395-725``, same steps as ``solvers/amen.py`` of
this package) written as a generator that yields one primitive device
operation at a time (an environment update, a QR, an SVD, a Krylov solve,
a rank decision ...).  :class:`BatchEngine` advances every active solve by
one operation per *tick* and executes each tick's operations grouped by
kind: one libttb200 call per kind, whatever the number of solves, so the
launch count per tick is independent of the batch size and small solves
fill the GPU together.  Rank decisions and residual norms of all solves
come back to the host with one synchronisation per tick.

Solves can be admitted at any tick (continuous batching); each finishes
independently with its own ``SolverInfo``.
"""

from __future__ import annotations

import math
import time
from typing import Callable, Dict, List, Optional

import torch

from . import kernels as K
from . import tensor_train
from .solvers.common import (
    LocalSolver,
    SolverInfo,
    StopReason,
    TruncationMode,
    _MAX_LOCAL_RESTARTS,
    _RESTART_RTOL_SHRINK,
    _SolverSettings,
    _validate_solver_inputs,
)
from .tensor_train import TensorTrain


def _c3(core):
    return core.reshape(core.shape[0], core.shape[1], core.shape[3])


# ---------------------------------------------------------------------------
# operations a program can yield
# ---------------------------------------------------------------------------


class Op:
    kind = ""
    __slots__ = ("args",)

    def __init__(self, *args):
        self.args = args


class Env(Op):
    kind = "env"          # args: list of env descs


class Proj(Op):
    kind = "proj"         # args: list of project descs


class Apply(Op):
    kind = "apply"        # args: list of local descs


class Copy(Op):
    kind = "copy"         # args: list of copy descs


class Gemm(Op):
    kind = "gemm"         # args: list of gemm descs


class Qr(Op):
    kind = "qr"           # args: (a, want_q, want_r, q_out, r_out) -> (q, r)


class Svd(Op):
    kind = "svd"          # args: (a,) -> (u, s, vh)


class Direct(Op):
    kind = "direct"       # args: (left, op, right, b_loc) -> u


class Krylov(Op):
    kind = "krylov"       # args: (method, left, op, right, b, x, rtol, warm)


class Norm(Op):
    kind = "norm"         # args: list of (out, x, y)


class Kron(Op):
    kind = "kron"         # args: list of (op, core) -> list of cores


class RankRes(Op):
    kind = "rankres"      # args: (contrib, b, exact, s, limit, damp, tol) -> int


class RankThr(Op):
    kind = "rankthr"      # args: (s, mode, value, max_rank) -> int


class Read(Op):
    kind = "read"         # args: list of 1-element float64 device tensors -> floats


ORDER = ["env", "proj", "kron", "apply", "copy", "gemm", "qr", "svd", "direct", "krylov",
         "norm", "rankres", "rankthr", "read"]


# ---------------------------------------------------------------------------
# program helpers (each a generator of operations)
# ---------------------------------------------------------------------------


def _shift_right(t: TensorTrain, k: int, core):
    rl, n, rr = core.shape
    q, r = yield Qr(core.reshape(rl * n, rr), True, True, None, None)
    t.cores[k] = q.reshape(rl, n, 1, q.shape[1])
    nxt = t.cores[k + 1]
    out = K.empty(r.shape[0], *nxt.shape[1:])
    yield Gemm([K.gemm_desc(r, nxt.reshape(nxt.shape[0], -1), out.view(r.shape[0], -1))])
    t.cores[k + 1] = out
    t.orth_center = k + 1


def _shift_left(t: TensorTrain, k: int, core):
    rl, n, rr = core.shape
    p = min(rl, n * rr)
    qt = K.empty(p, n * rr)
    _, r = yield Qr(core.reshape(rl, n * rr).t(), False, True, qt.t(), None)
    t.cores[k] = qt.reshape(p, n, 1, rr)
    prv = t.cores[k - 1]
    out = K.empty(*prv.shape[:3], p)
    yield Gemm([K.gemm_desc(prv.reshape(-1, rl), r.t(), out.view(-1, p))])
    t.cores[k - 1] = out
    t.orth_center = k - 1


def _orth_right(t: TensorTrain, start: int, end: int):
    """QR sweep right to left over ``start..end+1`` (``utils.py:115-136``)."""
    for i in range(start, end, -1):
        c = t.cores[i]
        yield from _shift_left(t, i, c.reshape(c.shape[0], c.shape[1], c.shape[3]))


def _orth_left(t: TensorTrain, start: int, end: int):
    for i in range(start, end):
        c = t.cores[i]
        yield from _shift_right(t, i, c.reshape(c.shape[0], c.shape[1], c.shape[3]))


def _tt_norm(cores: List[torch.Tensor]):
    """Right QR sweep keeping only R factors, then the norm of core 0
    (``tensor_train.py:509-540``); returns a 1-element device tensor."""
    carry = None
    for i in range(len(cores) - 1, 0, -1):
        c = cores[i]
        if carry is not None:
            m = K.empty(*c.shape[:-1], carry.shape[1])
            yield Gemm([K.gemm_desc(c.reshape(-1, c.shape[-1]), carry, m.view(-1, carry.shape[1]))])
        else:
            m = c
        mat = m.reshape(m.shape[0], -1)
        _, r = yield Qr(mat.t(), False, True, None, None)
        carry = r.t()
    c0 = cores[0]
    first = K.empty(*c0.shape[:-1], carry.shape[1])
    yield Gemm([K.gemm_desc(c0.reshape(-1, c0.shape[-1]), carry, first.view(-1, carry.shape[1]))])
    out = K.empty(1)
    yield Norm([(out, first, None)])
    return out


class SolveState:
    """One AMEn solve in the engine."""

    ENVS = ("A", "b", "zb", "zAx", "xz")

    def __init__(self, rid, A: TensorTrain, b: TensorTrain, x: TensorTrain, z: TensorTrain,
                 settings: _SolverSettings, kickrank, error_threshold, max_rank, residual_damp):
        self.rid = rid
        self.A, self.b, self.x, self.z = A, b, x, z
        self.st = settings
        self.kick = kickrank
        self.eth = error_threshold
        self.max_rank = max_rank
        self.damp = residual_damp
        self.d = len(A)
        self.left = {k: [None] * self.d for k in self.ENVS}
        self.right = {k: [None] * self.d for k in self.ENVS}
        self.info = SolverInfo()
        self.lu_info = []
        self.t_admit = None
        self.t_done = None
        self.error: Optional[BaseException] = None

    # -- environment descriptors (no device work; the engine runs them) ----

    def _pairs(self):
        x, z, b, A = self.x, self.z, self.b, self.A
        return {"A": (x, x, A), "b": (x, b, None), "zb": (z, b, None), "zAx": (z, x, A),
                "xz": (x, z, None)}

    def env_left(self, k, names=ENVS):
        pairs = self._pairs()
        descs = []
        for name in names:
            frame, target, op = pairs[name]
            if k == 0:
                self.left[name][0] = K.fill_(K.empty(1, 1, 1) if op is not None else K.empty(1, 1), 1.0)
                continue
            env = self.left[name][k - 1]
            fc, tc = _c3(frame.cores[k - 1]), _c3(target.cores[k - 1])
            opc = op.cores[k - 1] if op is not None else None
            out = (K.empty(tc.shape[2], opc.shape[3], fc.shape[2]) if op is not None
                   else K.empty(tc.shape[2], fc.shape[2]))
            descs.append(K.env_desc(0, env, fc, tc, out, opc))
            self.left[name][k] = out
        return Env(descs)

    def env_right(self, k, names=ENVS):
        pairs = self._pairs()
        descs = []
        for name in names:
            frame, target, op = pairs[name]
            if k == self.d - 1:
                self.right[name][k] = K.fill_(K.empty(1, 1, 1) if op is not None else K.empty(1, 1), 1.0)
                continue
            env = self.right[name][k + 1]
            fc, tc = _c3(frame.cores[k + 1]), _c3(target.cores[k + 1])
            opc = op.cores[k + 1] if op is not None else None
            out = (K.empty(tc.shape[0], opc.shape[0], fc.shape[0]) if op is not None
                   else K.empty(tc.shape[0], fc.shape[0]))
            descs.append(K.env_desc(1, env, fc, tc, out, opc))
            self.right[name][k] = out
        return Env(descs)

    def local_A(self, k):
        return self.left["A"][k], self.A.cores[k], self.right["A"][k]

    # -- staged local algebra ----------------------------------------------

    def residual_core(self, k, x_core):
        zl, zr = self.left["zb"][k].shape[1], self.right["zb"][k].shape[1]
        n = self.b.cores[k].shape[1]
        out = K.empty(zl, n, zr)
        yield Proj([K.project_desc(self.left["zb"][k], _c3(self.b.cores[k]), self.right["zb"][k],
                                   out)])
        yield Apply([K.local_desc(self.left["zAx"][k], self.A.cores[k], self.right["zAx"][k],
                                  x_core, out, 1, -1.0, 1.0)])
        return out

    def solve_local(self, k, stats):
        x, st = self.x, self.st
        rl, n, rr = x.cores[k].shape[0], x.cores[k].shape[1], x.cores[k].shape[3]
        b_loc = K.empty(rl, n, rr)
        yield Proj([K.project_desc(self.left["b"][k], _c3(self.b.cores[k]), self.right["b"][k],
                                   b_loc)])
        left, op, right = self.local_A(k)
        if not st.use_iterative(rl * n * rr):
            u = yield Direct(left, op, right, b_loc)
            return u, b_loc
        method = "minres" if st.iterative_solver is LocalSolver.MINRES else "gmres"
        u = K.empty(rl, n, rr)
        nb = K.empty(2)
        tmp = K.empty(rl, n, rr)
        yield Copy([K.copy_desc(_c3(x.cores[k]), u)])
        rtol = st.local_rtol
        for _ in range(_MAX_LOCAL_RESTARTS):
            yield Krylov(method, left, op, right, b_loc, u, rtol, True)
            yield Apply([K.local_desc(left, op, right, u, tmp)])
            yield Norm([(nb[0:1], b_loc, None), (nb[1:2], tmp, b_loc)])
            bn, rn = yield Read([nb[0:1], nb[1:2]])
            if rn <= st.local_rtol * bn:
                stats["local_solves"] += 1
                return u, b_loc
            rtol = max(rtol * _RESTART_RTOL_SHRINK, 1e-15)
        stats["local_solves"] += 1
        if not st.allow_dense_fallback:
            stats["local_inexact"] += 1
            return u, b_loc
        stats["local_fallbacks"] += 1
        u = yield Direct(left, op, right, b_loc)
        return u, b_loc

    def choose_rank(self, k, u, b_loc, U, S, Vh, stats):
        p = S.numel()
        if self.st.truncation_mode is TruncationMode.RESIDUAL:
            limit = p if self.max_rank is None else min(p, self.max_rank)
            size = u.numel()
            left, op, right = self.local_A(k)
            exact = K.empty(1)
            tmp = K.empty(*u.shape)
            yield Apply([K.local_desc(left, op, right, u, tmp)])
            yield Norm([(exact, tmp, b_loc)])
            svh = K.empty(limit, Vh.shape[1])
            yield Copy([K.copy_desc(Vh[:limit], svh, 1.0, S[:limit], 0)])
            terms = K.empty(limit, U.shape[0], Vh.shape[1])
            yield Gemm([K.gemm_desc(U.t()[:limit].unsqueeze(2), svh.unsqueeze(1), terms)])
            contrib = K.empty(limit, size)
            yield Apply([K.local_desc(left, op, right, terms, contrib, limit)])
            rank = yield RankRes(contrib, b_loc, exact, S, limit, self.damp, self.st.truncation_tol)
        else:
            rank = yield RankThr(S, 0, self.eth, self.max_rank)
        stats["rank_decisions"] += 1
        return rank

    def truncate(self, k, u, b_loc, forward, stats):
        rl, n, rr = u.shape
        mat = u.reshape(rl * n, rr) if forward else u.reshape(rl, n * rr)
        U, S, Vh = yield Svd(mat)
        rank = yield from self.choose_rank(k, u, b_loc, U, S, Vh, stats)
        if forward:
            core = K.empty(rl, n, rank)
            carry = K.empty(rank, rr)
            yield Copy([K.copy_desc(U[:, :rank], core.view(rl * n, rank)),
                        K.copy_desc(Vh[:rank], carry, 1.0, S[:rank], 0)])
        else:
            core = K.empty(rank, n, rr)
            carry = K.empty(rl, rank)
            yield Copy([K.copy_desc(Vh[:rank], core.view(rank, n * rr)),
                        K.copy_desc(U[:, :rank], carry, 1.0, S[:rank], 1)])
        return core, carry

    def enrich_right(self, k, core, carry, z_new):
        x = self.x
        rl, n, rank = core.shape
        zl, _, zr = z_new.shape
        enriched = K.empty(rl, n, rank + zr)
        nxt = x.cores[k + 1]
        padded = K.empty(rank + zr, *nxt.shape[1:])
        yield Copy([K.copy_desc(core, enriched[:, :, :rank]), K.copy_desc(None, padded[rank:], 0.0)])
        block = K.empty(rl, n, zr)
        yield Gemm([K.gemm_desc(self.left["xz"][k].t(), z_new.reshape(zl, n * zr),
                                block.view(rl, n * zr)),
                    K.gemm_desc(carry, nxt.reshape(nxt.shape[0], -1), padded[:rank].view(rank, -1))])
        yield Copy([K.copy_desc(block, enriched[:, :, rank:])])
        x.cores[k + 1] = padded
        yield from _shift_right(x, k, enriched)
        if self.max_rank is not None and x.cores[k].shape[3] > self.max_rank:
            mr = self.max_rank
            a, b2 = K.empty(*x.cores[k].shape[:3], mr), K.empty(mr, *x.cores[k + 1].shape[1:])
            yield Copy([K.copy_desc(x.cores[k][..., :mr], a), K.copy_desc(x.cores[k + 1][:mr], b2)])
            x.cores[k], x.cores[k + 1] = a, b2

    def enrich_left(self, k, core, carry, z_new):
        x = self.x
        rank, n, rr = core.shape
        zl, _, zr = z_new.shape
        enriched = K.empty(rank + zl, n, rr)
        prv = x.cores[k - 1]
        rl = carry.shape[0]
        padded = K.empty(*prv.shape[:3], rank + zl)
        yield Copy([K.copy_desc(core, enriched[:rank]), K.copy_desc(None, padded[..., rank:], 0.0)])
        yield Gemm([K.gemm_desc(z_new.reshape(zl * n, zr), self.right["xz"][k],
                                enriched[rank:].view(zl * n, rr)),
                    K.gemm_desc(prv.reshape(-1, rl), carry, padded[..., :rank].view(-1, rank))])
        x.cores[k - 1] = padded
        yield from _shift_left(x, k, enriched)
        if self.max_rank is not None and x.cores[k].shape[0] > self.max_rank:
            mr = self.max_rank
            a, b2 = K.empty(mr, *x.cores[k].shape[1:]), K.empty(*x.cores[k - 1].shape[:3], mr)
            yield Copy([K.copy_desc(x.cores[k][:mr], a), K.copy_desc(x.cores[k - 1][..., :mr], b2)])
            x.cores[k], x.cores[k - 1] = a, b2

    def relative_residual(self, b_norm):
        """``||A x - b|| / ||b||`` (``common.py:118-146``), staged."""
        A, b, x = self.A, self.b, self.x
        d = self.d
        prods = yield Kron([(A.cores[i], x.cores[i]) for i in range(d)])
        # residual train: block sum of A x and -b (b scaled at its centre)
        bc = list(b.cores)
        kb = b.orth_center if b.orth_center is not None else 0
        ra = [1] + [p.shape[0] for p in prods[1:]] + [1]
        rb = b.bonds
        ranks = [1] + [ra[i] + rb[i] for i in range(1, d)] + [1]
        cores, fills, copies = [], [], []
        for i in range(d):
            a_c, b_c = prods[i], bc[i]
            out = K.empty(ranks[i], a_c.shape[1], a_c.shape[2], ranks[i + 1])
            fills.append(K.copy_desc(None, out, 0.0))
            copies.append(K.copy_desc(a_c, out[: ra[i], :, :, : ra[i + 1]]))
            copies.append(K.copy_desc(b_c, out[ranks[i] - rb[i]:, :, :, ranks[i + 1] - rb[i + 1]:],
                                      -1.0 if i == kb else 1.0))
            cores.append(out)
        yield Copy(fills)
        yield Copy(copies)
        rn = yield from _tt_norm(cores)
        (res,) = yield Read([rn])
        return res if b_norm == 0.0 else res / b_norm


def program(s: SolveState):
    """The AMEn solve of ``s`` as a sequence of device operations
    (``ttnumpy/solvers/amen.py:529-725``)."""
    x, z, d, st = s.x, s.z, s.d, s.st
    stats = {"local_solves": 0, "local_fallbacks": 0, "local_inexact": 0, "rank_decisions": 0}
    if x.orth_center != 0:
        yield from _orth_right(x, d - 1, 0)
        x.orth_center = 0
    yield from _orth_right(z, d - 1, 0)
    z.orth_center = 0
    # fit z to b - A x (amen.py:162-224)
    for i in range(d - 1, -1, -1):
        yield s.env_right(i, ("zb", "zAx"))
    yield s.env_left(0, ("zb", "zAx"))
    for k in range(d - 1):
        if k > 0:
            yield s.env_left(k, ("zb", "zAx"))
        core = yield from s.residual_core(k, _c3(x.cores[k]))
        yield from _shift_right(z, k, core)
    yield s.env_left(d - 1, ("zb", "zAx"))
    for k in range(d - 1, -1, -1):
        yield s.env_right(k, ("zb", "zAx"))
        core = yield from s.residual_core(k, _c3(x.cores[k]))
        if k > 0:
            yield from _shift_left(z, k, core)
        else:
            z.cores[0] = core.reshape(1, core.shape[1], 1, core.shape[2])
            z.orth_center = 0
    for i in range(d - 1, -1, -1):
        yield s.env_right(i)
    b_norm = None
    if st.track_residual:
        if s.b.orth_center is not None:
            out = K.empty(1)
            yield Norm([(out, s.b.cores[s.b.orth_center], None)])
        else:
            out = yield from _tt_norm(s.b.cores)
        (b_norm,) = yield Read([out])
    info = s.info
    for sweep in range(st.max_sweeps):
        for k in range(d - 1):
            yield s.env_left(k)
            u, b_loc = yield from s.solve_local(k, stats)
            z_new = yield from s.residual_core(k, u)
            core, carry = yield from s.truncate(k, u, b_loc, True, stats)
            yield from s.enrich_right(k, core, carry, z_new)
            yield from _shift_right(z, k, z_new)
        yield s.env_left(d - 1)
        for k in range(d - 1, -1, -1):
            yield s.env_right(k)
            u, b_loc = yield from s.solve_local(k, stats)
            z_new = yield from s.residual_core(k, u)
            if k == 0:
                x.cores[0] = u.reshape(1, u.shape[1], 1, u.shape[2])
                x.orth_center = 0
                z.cores[0] = z_new.reshape(1, z_new.shape[1], 1, z_new.shape[2])
                z.orth_center = 0
            else:
                core, carry = yield from s.truncate(k, u, b_loc, False, stats)
                yield from s.enrich_left(k, core, carry, z_new)
                yield from _shift_left(z, k, z_new)
        info.num_sweeps_run = sweep + 1
        info.max_bonds.append(max(x.bonds))
        info.local_solves += stats["local_solves"]
        info.local_fallbacks += stats["local_fallbacks"]
        info.local_inexact += stats["local_inexact"]
        for key in ("local_solves", "local_fallbacks", "local_inexact"):
            stats[key] = 0
        if not st.track_residual:
            continue
        res = yield from s.relative_residual(b_norm)
        info.residuals.append(res)
        if st.residual_tol is not None and res <= st.residual_tol:
            info.stop_reason = StopReason.CONVERGED
            break
        if (st.stagnation_factor is not None and len(info.residuals) >= 2
                and info.residuals[-1] > st.stagnation_factor * info.residuals[-2]):
            info.stop_reason = StopReason.STAGNATED
            break
    redundant = [k for k in range(1, d) if x.bonds[k] > math.prod(x.row_modes[:k])]
    if redundant:
        yield from _orth_left(x, 0, redundant[-1])
        yield from _orth_right(x, redundant[-1], 0)
        x.orth_center = 0


class BatchEngine:
    """Runs many AMEn programs in lockstep (see the module docstring)."""

    def __init__(self):
        K.device_ok()
        self.active: List[tuple] = []  # (state, generator, pending op)
        self.finished: List[SolveState] = []
        self._next_id = 0
        self.ticks = 0

    def admit(self, A: TensorTrain, b: TensorTrain, x0: Optional[TensorTrain] = None,
              kickrank: int = 4, error_threshold: float = 1e-7, max_rank: Optional[int] = None,
              max_sweeps: int = 1, residual_tol: Optional[float] = None,
              residual_damp: float = 2.0, stagnation_factor="auto", local_solver="auto",
              direct_solve_size: int = 1000, local_rtol: Optional[float] = None,
              allow_dense_fallback: bool = False, symmetric: bool = False,
              return_info: bool = True, seed: Optional[int] = None, rid=None) -> SolveState:
        """Validate like ``amen`` and queue the solve; its first operation
        runs at the next tick."""
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
            allow_dense_fallback=allow_dense_fallback,
            truncation_steps=max(2 * (A.n_cores - 1), 1))
        if x0 is None:
            x0 = tensor_train.ones(b.physical_dims(), ranks=b.bonds)
        _validate_solver_inputs(A, b, x0)
        x = x0.copy()
        z = tensor_train.rand(b.physical_dims(), ranks=kickrank, seed=seed)
        if rid is None:
            rid = self._next_id
        self._next_id += 1
        s = SolveState(rid, A, b, x, z, settings, kickrank, error_threshold, max_rank,
                       residual_damp)
        s.t_admit = time.perf_counter()
        gen = program(s)
        self.active.append([s, gen, None, True])
        return s

    def tick(self) -> List[SolveState]:
        """Advance every active solve by one operation; returns the solves
        that finished during this tick."""
        groups: Dict[str, list] = {}
        done: List[SolveState] = []
        # resume generators whose previous op has a result (or that start)
        for entry in self.active:
            s, gen, op, fresh = entry
            if fresh:
                try:
                    entry[2] = next(gen)
                except StopIteration:
                    entry[2] = None
                entry[3] = False
        for entry in self.active:
            if entry[2] is not None:
                groups.setdefault(entry[2].kind, []).append(entry)
        results = {}
        host_ints, host_floats = [], []
        for kind in ORDER:
            items = groups.get(kind)
            if not items:
                continue
            ops = [e[2] for e in items]
            if kind == "env":
                K.env_update([d for o in ops for d in o.args[0]])
            elif kind == "proj":
                K.project([d for o in ops for d in o.args[0]])
            elif kind == "apply":
                K.local_apply([d for o in ops for d in o.args[0]])
            elif kind == "copy":
                K.copy_many([d for o in ops for d in o.args[0]])
            elif kind == "gemm":
                K.gemm_many([d for o in ops for d in o.args[0]])
            elif kind == "norm":
                K.norm_many([it for o in ops for it in o.args[0]])
            elif kind == "kron":
                outs = K.kron_many([it for o in ops for it in o.args[0]])
                pos = 0
                for e, o in zip(items, ops):
                    n = len(o.args[0])
                    results[id(e)] = outs[pos:pos + n]
                    pos += n
            elif kind == "qr":
                outs = K.qr_many([o.args for o in ops])
                for e, r in zip(items, outs):
                    results[id(e)] = r
            elif kind == "svd":
                outs = K.svd_many([o.args[0] for o in ops])
                for e, r in zip(items, outs):
                    results[id(e)] = r
            elif kind == "direct":
                info = torch.zeros(len(ops), dtype=torch.int32, device="cuda")
                outs = K.direct_many([o.args for o in ops], info)
                for j, (e, r) in enumerate(zip(items, outs)):
                    results[id(e)] = r
                    e[0].lu_info.append(info[j:j + 1])
            elif kind == "krylov":
                for method in ("minres", "gmres"):
                    sel = [o for o in ops if o.args[0] == method]
                    K.krylov_many(method, [o.args[1:] for o in sel])
            elif kind in ("rankres", "rankthr"):
                ranks = torch.zeros(len(ops), dtype=torch.int32, device="cuda")
                if kind == "rankres":
                    K.rank_residual_many([o.args + (ranks[j:j + 1],) for j, o in enumerate(ops)])
                else:
                    K.rank_threshold_many([o.args + (ranks[j:j + 1],) for j, o in enumerate(ops)])
                host_ints.append((items, ranks))
            elif kind == "read":
                host_floats.append(items)
        # one synchronisation for every host-bound value of the tick
        if host_ints or host_floats:
            tensors = [r.to(torch.float64) for _, r in host_ints]
            for items in host_floats:
                tensors.extend(t for e in items for t in e[2].args[0])
            vals = torch.cat([t.reshape(-1) for t in tensors]).tolist() if tensors else []
            pos = 0
            for items, r in host_ints:
                for e in items:
                    results[id(e)] = int(vals[pos])
                    pos += 1
            for items in host_floats:
                for e in items:
                    n = len(e[2].args[0])
                    results[id(e)] = vals[pos:pos + n]
                    pos += n
        # resume everyone with its result
        still = []
        for entry in self.active:
            s, gen, op, _ = entry
            if op is None:
                done.append(s)
                continue
            try:
                entry[2] = gen.send(results.get(id(entry)))
                still.append(entry)
            except StopIteration:
                done.append(s)
            except Exception as exc:  # noqa: BLE001 - reported per solve
                s.error = exc
                done.append(s)
        self.active = still
        self.ticks += 1
        now = time.perf_counter()
        for s in done:
            s.t_done = now
            if s.lu_info and s.error is None:
                infos = torch.cat(s.lu_info).cpu().tolist()
                if any(i != 0 for i in infos):
                    import numpy as np

                    s.error = np.linalg.LinAlgError("local system is singular")
            self.finished.append(s)
        return done

    def run(self) -> List[SolveState]:
        while self.active:
            self.tick()
        return self.finished


def amen_batch(problems, **kwargs) -> List[SolveState]:
    """Solve ``[(A, b, x0), ...]`` together; keyword arguments as ``amen``."""
    eng = BatchEngine()
    for A, b, x0 in problems:
        eng.admit(A, b, x0, **kwargs)
    return eng.run()
