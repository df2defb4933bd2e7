"""CPU oracle for the tensor-train solve path.

TEST INFRASTRUCTURE ONLY.  This module is a plain NumPy/SciPy restatement of
the reference algorithm (ttnumpy 0.3.0): the AMEn one-site sweep, the TT
rounding it depends on and the TTM-by-TT product, and beside them ALS, MALS,
randomized rounding (generic and HaTT-1 for element-wise products), TT-SVD
and the QTT conversions.  It exists so that the
parity tests, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` have something to check the CUDA path against and something to
time on the host cores.  Nothing in the product package imports it.

Parity of this oracle is pinned against the reference itself: the fixtures
under ``tests/golden/`` were produced by importing the reference package and
``tests/test_oracle.py`` checks this module against every one of them.

Every function names the reference file and lines it restates.  Paths are
relative to the reference project root.

Conventions (reference ``ttnumpy/tensor_train.py:150-244``): a train is a
list of 4-D float64 cores ``(r_k, row_mode_k, col_mode_k, r_{k+1})``; a TT
vector has ``col_mode == 1``.  ``Train.orth_center`` mirrors the reference
attribute of the same name.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import scipy.linalg as sla
import scipy.sparse.linalg as spla


class Train:
    """List of 4-D cores plus the orthogonality centre.

    Mirrors the state the reference keeps on ``TensorTrain``
    (``ttnumpy/tensor_train.py:232-239``).
    """

    def __init__(self, cores: List[np.ndarray], orth_center: Optional[int] = None):
        fixed = []
        for core in cores:
            core = np.asarray(core, dtype=np.float64)
            if core.ndim == 3:
                core = core.reshape(core.shape[0], core.shape[1], 1, core.shape[2])
            fixed.append(core)
        self.cores = fixed
        self.orth_center = orth_center

    def __len__(self) -> int:
        return len(self.cores)

    @property
    def bonds(self) -> List[int]:
        return [c.shape[0] for c in self.cores] + [1]

    @property
    def row_modes(self) -> List[int]:
        return [c.shape[1] for c in self.cores]

    @property
    def col_modes(self) -> List[int]:
        return [c.shape[2] for c in self.cores]

    def is_ttm(self) -> bool:
        return any(c.shape[2] != 1 for c in self.cores)

    def copy(self) -> "Train":
        return Train([c.copy() for c in self.cores], self.orth_center)

    def full(self) -> np.ndarray:
        """Dense vector (TT) or matrix (TTM) in the reference index order.

        Restates ``TensorTrain.matricize`` (``tensor_train.py:626-641``): rows
        are the row modes in core order, columns the column modes.
        """
        out = np.ones((1, 1, 1))
        for c in self.cores:
            rows, cols, r = out.shape[0], out.shape[1], out.shape[2]
            t = np.einsum("abr,rijs->aibjs", out, c)
            out = t.reshape(rows * c.shape[1], cols * c.shape[2], c.shape[3])
        out = out[:, :, 0]
        return out[:, 0] if not self.is_ttm() else out


# --------------------------------------------------------------------------
# constructors (tensor_train.py:1250-1387)
# --------------------------------------------------------------------------


def _expand_ranks(n_cores: int, ranks) -> List[int]:
    if isinstance(ranks, list):
        return ranks
    return [1] + [int(ranks)] * (n_cores - 1) + [1]


def rand(dims, ranks=1, seed=None) -> Train:
    """Uniform [0, 1) cores drawn core by core from one generator.

    Restates ``tensor_train.rand`` (``tensor_train.py:1350-1387``): one
    ``np.random.default_rng(seed)``, cores drawn in order with
    ``rng.random`` of shape ``(r, n, 1, r')``.
    """
    r = _expand_ranks(len(dims), ranks)
    rng = np.random.default_rng(seed)
    return Train([rng.random((r[i], dims[i], 1, r[i + 1])) for i in range(len(dims))])


def ones(dims, ranks=1) -> Train:
    """All-ones cores (``tensor_train.py:1250-1285``)."""
    r = _expand_ranks(len(dims), ranks)
    return Train([np.ones((r[i], dims[i], 1, r[i + 1])) for i in range(len(dims))])


# --------------------------------------------------------------------------
# arithmetic (tensor_train.py:254-540)
# --------------------------------------------------------------------------


def add(a: Train, b: Train) -> Train:
    """Block-diagonal sum of two trains (``tensor_train.py:254-322``)."""
    d = len(a)
    ra, rb = a.bonds, b.bonds
    ranks = [1] + [ra[i] + rb[i] for i in range(1, d)] + [1]
    cores = []
    for i in range(d):
        ca, cb = a.cores[i], b.cores[i]
        out = np.zeros((ranks[i], ca.shape[1], ca.shape[2], ranks[i + 1]))
        out[: ra[i], :, :, : ra[i + 1]] = ca
        out[ranks[i] - rb[i] :, :, :, ranks[i + 1] - rb[i + 1] :] = cb
        cores.append(out)
    return Train(cores)


def scale(a: Train, factor: float) -> Train:
    """Scalar multiple (``tensor_train.py:389-395``): the centre core (or
    core 0 without a centre) is scaled."""
    out = a.copy()
    k = out.orth_center if out.orth_center is not None else 0
    out.cores[k] = factor * out.cores[k]
    return out


def dot(A: Train, x: Train) -> Train:
    """TTM-by-TT (or TTM-by-TTM) product (``tensor_train.py:427-499``).

    Each output core is the Kronecker combination
    ``einsum('aijb,mjkn->amikbn')`` reshaped to
    ``(R r, n_row, m_col, R' r')`` (``tensor_train.py:483-495``).
    """
    cores = []
    for ca, cx in zip(A.cores, x.cores):
        t = np.einsum("aijb,mjkn->amikbn", ca, cx, optimize="optimal")
        cores.append(
            t.reshape(
                ca.shape[0] * cx.shape[0],
                ca.shape[1],
                cx.shape[2],
                ca.shape[3] * cx.shape[3],
            )
        )
    return Train(cores)


def _mul_left(matrix: np.ndarray, core: np.ndarray) -> np.ndarray:
    """``matrix @ core`` over the first core axis (``utils.py:72-76``)."""
    return (matrix @ core.reshape(core.shape[0], -1)).reshape(
        (matrix.shape[0],) + core.shape[1:]
    )


def _mul_right(core: np.ndarray, matrix: np.ndarray) -> np.ndarray:
    """``core @ matrix`` over the last core axis (``utils.py:79-83``)."""
    return (core.reshape(-1, core.shape[-1]) @ matrix).reshape(
        core.shape[:-1] + (matrix.shape[1],)
    )


def left_orth_sweep(cores: List[np.ndarray], start: int, end: int) -> None:
    """QR sweep left to right over ``start..end-1`` (``utils.py:86-112``)."""
    for i in range(start, end):
        s = cores[i].shape
        q, r = sla.qr(cores[i].reshape(s[0] * s[1] * s[2], s[3]), mode="economic")
        cores[i] = q.reshape(s[0], s[1], s[2], q.shape[1])
        cores[i + 1] = _mul_left(r, cores[i + 1])


def right_orth_sweep(cores: List[np.ndarray], start: int, end: int) -> None:
    """QR sweep right to left over ``start..end+1`` (``utils.py:115-136``)."""
    for i in range(start, end, -1):
        s = cores[i].shape
        q, r = sla.qr(cores[i].reshape(s[0], s[1] * s[2] * s[3]).T, mode="economic")
        cores[i] = q.T.reshape(q.shape[1], s[1], s[2], s[3])
        cores[i - 1] = _mul_right(cores[i - 1], r.T)


def orthonormalize(t: Train, canonical: str, center_position: Optional[int] = None) -> Train:
    """In-place QR canonicalisation, ``left`` or ``right`` only
    (``tensor_train.py:705-787``), including the rules for the resulting
    ``orth_center``."""
    d = len(t)
    had_center = t.orth_center is not None
    if canonical == "left":
        end = center_position if center_position is not None else d - 1
        start = 0
        if t.orth_center is not None:
            start = t.orth_center
            if start <= end:
                t.orth_center = end
        if start >= end:
            return t
        left_orth_sweep(t.cores, start, end)
    elif canonical == "right":
        end = center_position if center_position is not None else 0
        start = d - 1
        if t.orth_center is not None:
            start = t.orth_center
            if start >= end:
                t.orth_center = end
        if start <= end:
            return t
        right_orth_sweep(t.cores, start, end)
    else:
        raise ValueError(canonical)
    if had_center or end in (0, d - 1):
        t.orth_center = end
    else:
        t.orth_center = None
    return t


def truncated_bond(s: np.ndarray, delta: float, max_rank: Optional[int] = None) -> int:
    """Tail-norm rank rule with the eps * len * sigma_1 noise floor
    (``utils.py:22-69``)."""
    vals = np.asarray(s, dtype=np.float64).copy()
    if vals.size:
        floor = np.finfo(np.float64).eps * vals.size * vals[0]
        vals[vals <= floor] = 0.0
    tail = np.cumsum((vals**2)[::-1])[::-1]
    bond = max(1, int(np.count_nonzero(tail > delta * delta)))
    if max_rank is not None:
        bond = min(bond, max_rank)
    return bond


def _svd(matrix: np.ndarray):
    """Thin SVD, gesdd then gesvd (``utils.py:336-361``)."""
    try:
        return sla.svd(matrix, full_matrices=False, check_finite=False)
    except np.linalg.LinAlgError:
        if not np.isfinite(matrix).all():
            raise ValueError("core has NaN or infinite entries")
        return sla.svd(matrix, full_matrices=False, check_finite=False, lapack_driver="gesvd")


def left_svd_sweep(cores: List[np.ndarray], error: float, max_rank=None) -> None:
    """SVD truncation sweep left to right (``utils.py:364-411``)."""
    c0 = cores[0]
    norm = np.linalg.norm(c0.reshape(c0.shape[1] * c0.shape[2], c0.shape[3]))
    delta = error / math.sqrt(len(cores) - 1) * norm
    bond = 1
    for i in range(len(cores) - 1):
        s = cores[i].shape
        u, sv, vh = _svd(cores[i].reshape(bond * s[1] * s[2], s[3]))
        nb = truncated_bond(sv, delta, max_rank)
        cores[i] = u[:, :nb].reshape(bond, s[1], s[2], nb)
        cores[i + 1] = _mul_left(sv[:nb, None] * vh[:nb], cores[i + 1])
        bond = nb


def right_svd_sweep(cores: List[np.ndarray], error: float, max_rank=None) -> None:
    """SVD truncation sweep right to left (``utils.py:414-460``)."""
    cl = cores[-1]
    norm = np.linalg.norm(cl.reshape(cl.shape[0], cl.shape[1] * cl.shape[2]))
    delta = error / math.sqrt(len(cores) - 1) * norm
    bond = 1
    for i in range(len(cores) - 1, 0, -1):
        s = cores[i].shape
        u, sv, vh = _svd(cores[i].reshape(s[0], s[1] * s[2] * bond))
        nb = truncated_bond(sv, delta, max_rank)
        cores[i] = vh[:nb].reshape(nb, s[1], s[2], bond)
        cores[i - 1] = _mul_right(cores[i - 1], u[:, :nb] * sv[:nb])
        bond = nb


def compress_svd(t: Train, error: float = 0.0, max_rank=None, canonical="auto") -> Train:
    """In-place SVD compression (``tensor_train.py:789-850``)."""
    d = len(t)
    if canonical == "auto":
        canonical = "left" if (t.orth_center is None or t.orth_center <= (d - 1) / 2) else "right"
    if canonical == "right":
        right_svd_sweep(t.cores, error, max_rank)
        t.orth_center = 0
    elif canonical == "left":
        left_svd_sweep(t.cores, error, max_rank)
        t.orth_center = d - 1
    else:
        raise ValueError(canonical)
    return t


def sketch_rank(max_rank, options) -> int:
    """Bond of the random sketch (``tensor_train.py:122-140``)."""
    if max_rank is None:
        raise ValueError("method='randomized' needs max_rank")
    options = {} if options is None else options
    if set(options) - {"oversampling"}:
        raise ValueError("unknown options")
    over = options.get("oversampling", 10)
    if not isinstance(over, (int, np.integer)) or isinstance(over, bool) or over < 0:
        raise ValueError("oversampling must be a non-negative integer")
    return max_rank + over


def randomized_left_orth(cores: List[np.ndarray], rank: int, rng) -> List[np.ndarray]:
    """Randomize-then-orthogonalise, left to right
    (``left_randomized_orthonormalize``, ``utils.py:139-203``): sketches of
    the cores to the right of each bond against a Gaussian train (drawn
    right to left, each sketch scaled by its largest entry), then the QR of
    each unfolding times the next sketch."""
    if rank < 1:
        raise ValueError("rank must be positive")
    count = len(cores)
    sketches = [None] * count + [np.ones((1, 1))]
    for i in range(count - 1, 0, -1):
        contracted = _mul_right(cores[i], sketches[i + 1])
        contracted = contracted.reshape(contracted.shape[0], -1)
        bond = min(rank, *contracted.shape)
        sk = contracted @ rng.standard_normal((contracted.shape[1], bond))
        scale = np.abs(sk).max()
        if scale > 0:
            sk /= scale
        sketches[i] = sk
    for i in range(count - 1):
        shape = cores[i].shape
        matrix = cores[i].reshape(shape[0] * shape[1] * shape[2], shape[3])
        q, _ = sla.qr(matrix @ sketches[i + 1], mode="economic")
        cores[i] = q.reshape(shape[0], shape[1], shape[2], -1)
        cores[i + 1] = _mul_left(q.T @ matrix, cores[i + 1])
    return cores


def randomized_right_orth(cores: List[np.ndarray], rank: int, rng) -> List[np.ndarray]:
    """Mirror image of :func:`randomized_left_orth` (``utils.py:206-236``)."""
    mirrored = [c.transpose(3, 1, 2, 0) for c in reversed(cores)]
    mirrored = randomized_left_orth(mirrored, rank, rng)
    cores[:] = [np.ascontiguousarray(c.transpose(3, 1, 2, 0)) for c in reversed(mirrored)]
    return cores


def hadamard(a: Train, b: Train) -> Train:
    """Element-wise product of two trains (``tensor_train.py:380-395``):
    core k is the Kronecker product of the two cores over the bonds,
    indexed ((a, x), i, j, (b, y))."""
    cores = []
    for p, q in zip(a.cores, b.cores):
        c = np.einsum("aijb,xijy->axijby", p, q)
        cores.append(c.reshape(p.shape[0] * q.shape[0], p.shape[1], p.shape[2],
                               p.shape[3] * q.shape[3]))
    return Train(cores)


def randomized_hadamard(lhs: List[np.ndarray], rhs: List[np.ndarray], rank: int, rng) -> List[np.ndarray]:
    """HaTT-1 (``utils.py:262-333``): the randomised left orthonormalisation
    of the element-wise product train without forming its cores.  The
    sketch of the product right of each bond is built from one core of each
    factor at a time (``utils.py:225-240``), the Gaussian cores drawn in the
    order and shapes of the generic sketch, each sketch scaled by its
    largest entry; left to right, the carried projection times the two
    cores (``utils.py:243-259``) times the next sketch is factorised by QR."""
    if rank < 1:
        raise ValueError(f"rank must be positive, but got {rank}")
    count = len(lhs)
    sketches = [None] * count + [np.ones((1, 1, 1))]
    for i in range(count - 1, 0, -1):
        a, b = lhs[i], rhs[i]
        m = a.shape[1] * a.shape[2]
        contracted = np.einsum("apb,cpd,bdt->acpt", a.reshape(a.shape[0], m, a.shape[3]),
                               b.reshape(b.shape[0], m, b.shape[3]), sketches[i + 1],
                               optimize="optimal")
        contracted = contracted.reshape(a.shape[0] * b.shape[0], -1)
        bond = min(rank, *contracted.shape)
        sketch = contracted @ rng.standard_normal((contracted.shape[1], bond))
        top = np.abs(sketch).max()
        if top > 0:
            sketch /= top
        sketches[i] = sketch.reshape(a.shape[0], b.shape[0], bond)
    cores = []
    carry = np.ones((1, 1, 1))
    for i in range(count):
        a, b = lhs[i], rhs[i]
        m = a.shape[1] * a.shape[2]
        matrix = np.einsum("tac,apb,cpd->tpbd", carry, a.reshape(a.shape[0], m, a.shape[3]),
                           b.reshape(b.shape[0], m, b.shape[3]), optimize="optimal")
        matrix = matrix.reshape(carry.shape[0] * m, -1)
        shape = (carry.shape[0], a.shape[1], a.shape[2], -1)
        if i == count - 1:
            cores.append(matrix.reshape(shape))
            break
        q, _ = sla.qr(matrix @ sketches[i + 1].reshape(matrix.shape[1], -1), mode="economic")
        cores.append(q.reshape(shape))
        carry = (q.T @ matrix).reshape(q.shape[1], a.shape[3], b.shape[3])
    return cores


def multiply(a: Train, b: Train, truncate_: bool = False, error=None, max_rank=None,
             method: str = "direct", seed=None, options=None) -> Train:
    """``TensorTrain.multiply`` of two trains (``tensor_train.py:327-407``):
    the product train, rounded when ``truncate_``; the randomized rounding
    goes through HaTT-1 and the SVD sweep."""
    if truncate_ and method == "randomized":
        out = Train(randomized_hadamard(a.cores, b.cores, sketch_rank(max_rank, options),
                                        np.random.default_rng(seed)), orth_center=len(a) - 1)
        return compress_svd(out, 0.0 if error is None else error, max_rank)
    out = hadamard(a, b)
    if not truncate_:
        return out
    return truncate(out, 0.0 if error is None else error, max_rank, method=method, seed=seed,
                    options=options)


def truncate(t: Train, error: float = 0.0, max_rank=None, canonical="auto", method="direct",
             seed=None, options=None) -> Train:
    """TT rounding (``tensor_train.py:852-940``): QR (``method='direct'``)
    or sketched (``'randomized'``) canonicalisation towards one end, then
    the SVD sweep back."""
    if method == "randomized":
        rank = sketch_rank(max_rank, options)
    out = t.copy()
    orth_form = "left" if canonical == "right" else "right"
    if canonical == "auto":
        if out.orth_center is None or out.orth_center >= len(out) / 2:
            orth_form = "left"
        else:
            orth_form = "right"
    if method == "direct":
        orthonormalize(out, orth_form)
    else:
        rng = np.random.default_rng(seed)
        if orth_form == "left":
            randomized_left_orth(out.cores, rank, rng)
            out.orth_center = len(out) - 1
        else:
            randomized_right_orth(out.cores, rank, rng)
            out.orth_center = 0
    compress_svd(out, error, max_rank)
    return out


def tt_norm(t: Train) -> float:
    """Frobenius norm via a right QR sweep (``tensor_train.py:509-540``)."""
    if t.orth_center is not None:
        return float(np.linalg.norm(t.cores[t.orth_center].reshape(-1)))
    cores = [c.reshape(c.shape[0], c.shape[1] * c.shape[2], 1, c.shape[3]).copy() for c in t.cores]
    right_orth_sweep(cores, len(cores) - 1, 0)
    return float(np.linalg.norm(cores[0].reshape(-1)))


def inner(a, b) -> float:
    """Inner product <a, b> of two TT vectors given as core lists (or
    Trains) of equal mode sizes, by a left-to-right contraction of the
    cores: a fingerprint of a solution that does not depend on its gauge
    (QR/SVD signs), used to compare solutions without storing their cores."""
    ca = a.cores if hasattr(a, "cores") else a
    cb = b.cores if hasattr(b, "cores") else b
    env = np.ones((1, 1))
    for x, y in zip(ca, cb):
        x = np.asarray(x).reshape(x.shape[0], -1, x.shape[-1])
        y = np.asarray(y).reshape(y.shape[0], -1, y.shape[-1])
        env = np.einsum("ab,anc,bnd->cd", env, x, y)
    return float(env[0, 0])


def relative_residual(A: Train, b: Train, x: Train, b_norm: Optional[float] = None) -> float:
    """``||A x - b|| / ||b||`` in TT arithmetic (``solvers/common.py:118-146``)."""
    res = add(dot(A, x), scale(b, -1.0))
    if b_norm is None:
        b_norm = tt_norm(b)
    rn = tt_norm(res)
    return rn if b_norm == 0.0 else rn / b_norm


# --------------------------------------------------------------------------
# environments and one-site local algebra
# --------------------------------------------------------------------------


def env_left(env: list, ind: int, frame: Train, target: Train, A: Optional[Train] = None) -> None:
    """Left projection recursion (``solvers/common.py:149-188``).

    With ``A`` the result is indexed (target, operator, frame), else
    (target, frame).
    """
    if ind == 0:
        env[0] = np.ones((1, 1, 1)) if A is not None else np.ones((1, 1))
        return
    f = frame.cores[ind - 1][:, :, 0, :]
    g = target.cores[ind - 1][:, :, 0, :]
    if A is not None:
        s = np.tensordot(env[ind - 1], f, axes=([2], [0]))
        s = np.tensordot(s, A.cores[ind - 1], axes=([1, 2], [0, 1]))
        env[ind] = np.tensordot(s, g, axes=([0, 2], [0, 1])).transpose(2, 1, 0)
    else:
        s = np.tensordot(env[ind - 1], f, axes=([1], [0]))
        env[ind] = np.tensordot(s, g, axes=([0, 1], [0, 1])).T


def env_right(env: list, ind: int, frame: Train, target: Train, A: Optional[Train] = None) -> None:
    """Right projection recursion (``solvers/common.py:191-217``)."""
    if ind == len(frame) - 1:
        env[-1] = np.ones((1, 1, 1)) if A is not None else np.ones((1, 1))
        return
    f = frame.cores[ind + 1][:, :, 0, :]
    g = target.cores[ind + 1][:, :, 0, :]
    if A is not None:
        s = np.tensordot(g, env[ind + 1], axes=([2], [0]))
        s = np.tensordot(s, A.cores[ind + 1], axes=([1, 2], [2, 3]))
        env[ind] = np.tensordot(s, f, axes=([1, 3], [2, 1]))
    else:
        s = np.tensordot(g, env[ind + 1], axes=([2], [0]))
        env[ind] = np.tensordot(s, f, axes=([1, 2], [1, 2]))


def local_rhs(left_b: np.ndarray, b_core: np.ndarray, right_b: np.ndarray) -> np.ndarray:
    """One-site right-hand side ``einsum('ai,ajc,cl->ijl')``
    (``solvers/one_site.py:27-46``), flattened."""
    return np.einsum("ai,ajc,cl->ijl", left_b, b_core[:, :, 0, :], right_b,
                     optimize="optimal").reshape(-1)


def local_matrix(left_A: np.ndarray, A_core: np.ndarray, right_A: np.ndarray) -> np.ndarray:
    """Explicit one-site operator (``solvers/one_site.py:49-75``); rows
    (frame bond, row mode, frame bond), columns (target bond, col mode,
    target bond)."""
    t = np.einsum("iaj,aklb,mbn->ijklmn", left_A, A_core, right_A, optimize="optimal")
    rl, rr = left_A.shape[0], right_A.shape[0]
    rows = rl * A_core.shape[1] * rr
    cols = rl * A_core.shape[2] * rr
    return t.transpose(1, 2, 5, 0, 3, 4).reshape(rows, cols)


def local_operator(left_A: np.ndarray, A_core: np.ndarray, right_A: np.ndarray):
    """Matrix-free one-site operator (``solvers/one_site.py:78-115``)."""
    rl, rr = left_A.shape[0], right_A.shape[0]
    size = rl * A_core.shape[2] * rr
    shape = (rl, A_core.shape[2], rr)

    def matmat(block):
        y = np.asarray(block).reshape(shape + (-1,))
        t = np.tensordot(y, right_A, axes=(2, 0))
        t = np.tensordot(t, A_core, axes=((1, 3), (2, 3)))
        t = np.tensordot(t, left_A, axes=((0, 3), (0, 1)))
        return t.transpose(3, 2, 1, 0).reshape(size, -1)

    return spla.LinearOperator(
        (size, size), matvec=lambda v: matmat(v).ravel(), matmat=matmat, dtype=np.float64
    )


# --------------------------------------------------------------------------
# solver settings, local solves, truncation rules (solvers/common.py)
# --------------------------------------------------------------------------

LOCAL_TOL_FACTOR = 0.1  # common.py:224
DEFAULT_LOCAL_RTOL = 1e-8  # common.py:227
MAX_LOCAL_RESTARTS = 4  # common.py:230
RESTART_RTOL_SHRINK = 1e-2  # common.py:233
DEFAULT_STAGNATION = 0.9  # common.py:237


@dataclass
class Settings:
    """Resolved options (``solvers/common.py:244-400``)."""

    max_sweeps: int
    residual_tol: Optional[float]
    stagnation_factor: Optional[float]
    iterative: Optional[str]  # "minres" / "gmres" / None
    direct_solve_size: int
    track_residual: bool
    local_rtol: Optional[float]
    allow_dense_fallback: bool
    truncation_steps: int

    @property
    def residual_mode(self) -> bool:
        return self.residual_tol is not None

    @property
    def truncation_tol(self) -> Optional[float]:
        if self.residual_tol is None:
            return None
        return self.residual_tol / np.sqrt(self.truncation_steps)


def resolve_settings(max_sweeps, residual_tol, stagnation_factor, local_solver, symmetric,
                     direct_solve_size, return_info, local_rtol, allow_dense_fallback,
                     truncation_steps) -> Settings:
    """``_SolverSettings.resolve`` (``solvers/common.py:301-400``)."""
    if residual_tol is not None and residual_tol <= 0.0:
        raise ValueError("residual_tol must be positive")
    if isinstance(stagnation_factor, str):
        if stagnation_factor != "auto":
            raise ValueError("bad stagnation_factor")
        stagnation_factor = DEFAULT_STAGNATION if (residual_tol is not None or return_info) else None
    if stagnation_factor is not None and not 0.0 < stagnation_factor <= 1.0:
        raise ValueError("stagnation_factor must be in (0, 1]")
    track = return_info or residual_tol is not None or (stagnation_factor is not None and max_sweeps > 1)
    if local_rtol is not None and local_rtol <= 0.0:
        raise ValueError("local_rtol must be positive")
    local_solver = str(getattr(local_solver, "value", local_solver))
    if local_solver not in ("auto", "direct", "minres", "gmres"):
        raise ValueError("bad local_solver")
    if local_solver == "auto":
        iterative = "minres" if symmetric else "gmres"
    elif local_solver == "direct":
        iterative = None
    else:
        iterative = local_solver
    if iterative is None:
        lr = None
    elif local_rtol is not None:
        lr = local_rtol
    elif residual_tol is not None:
        lr = LOCAL_TOL_FACTOR * residual_tol
    else:
        lr = DEFAULT_LOCAL_RTOL
    return Settings(max_sweeps, residual_tol, stagnation_factor, iterative, direct_solve_size,
                    track, lr, allow_dense_fallback, truncation_steps)


@dataclass
class Info:
    """``SolverInfo`` fields (``solvers/common.py:85-115``)."""

    residuals: List[float] = field(default_factory=list)
    num_sweeps_run: int = 0
    stop_reason: str = "max_sweeps"
    max_bonds: List[int] = field(default_factory=list)
    local_solves: int = 0
    local_fallbacks: int = 0
    local_inexact: int = 0


def solve_local(operator, b_loc, settings: Settings, iterative: bool, warm, fallback, info: Info):
    """``_solve_local_system`` (``solvers/common.py:729-809``)."""
    bv = b_loc.ravel()
    if not iterative:
        return np.asarray(sla.solve(operator, bv, check_finite=False)).ravel(), operator
    target = settings.local_rtol * np.linalg.norm(bv)
    u = warm
    rtol = settings.local_rtol
    for _ in range(MAX_LOCAL_RESTARTS):
        if settings.iterative == "minres":
            u, _ = spla.minres(operator, bv, x0=u, rtol=rtol)
        else:
            u, _ = spla.gmres(operator, bv, x0=u, rtol=rtol, atol=0.0)
        if np.linalg.norm(operator @ u - bv) <= target:
            info.local_solves += 1
            return np.asarray(u).ravel(), operator
        rtol = max(rtol * RESTART_RTOL_SHRINK, 1e-15)
    info.local_solves += 1
    if fallback is None:
        info.local_inexact += 1
        return np.asarray(u).ravel(), operator
    info.local_fallbacks += 1
    operator = fallback()
    return np.asarray(sla.solve(operator, bv, check_finite=False)).ravel(), operator


def rank_by_residual(A_loc, b_loc, U, S, V, exact_residual, trunc_tol, damp, max_rank) -> int:
    """``_truncation_rank_by_residual`` (``solvers/common.py:812-866``)."""
    if S[0] == 0.0:
        return 1
    limit = len(S) if max_rank is None else min(len(S), max_rank)
    threshold = max(damp * exact_residual, 0.5 * trunc_tol * np.linalg.norm(b_loc))
    terms = np.einsum("ik,kj->kij", U[:, :limit] * S[:limit], V[:limit, :], optimize="optimal")
    contrib = A_loc @ terms.reshape(limit, -1).T
    partial = -b_loc.copy()
    for r in range(limit):
        partial += contrib[:, r]
        if np.linalg.norm(partial) <= threshold:
            return r + 1
    return limit


def rank_by_threshold(S, error_threshold, max_rank) -> int:
    """``_svd_truncation_rank`` (``solvers/common.py:872-885``)."""
    if S.size == 0 or S[0] == 0.0:
        return 1
    rank = max(int(np.count_nonzero(S / S[0] > error_threshold)), 1)
    if max_rank is not None and rank > max_rank:
        return max_rank
    return rank


def truncate_core(core, left: bool, settings: Settings, error_threshold, max_rank, operator, b_loc, damp):
    """``_truncate_core_right`` / ``_truncate_core_left``
    (``solvers/amen.py:227-322``).  ``left=False`` is the forward
    (right-bond) variant returning (U core, carry), ``left=True`` the backward
    variant returning (Vh core, carry)."""
    rl, n, rr = core.shape
    exact = float(np.linalg.norm(operator @ core.ravel() - b_loc)) if settings.residual_mode else 0.0
    mat = core.reshape(rl, n * rr) if left else core.reshape(rl * n, rr)
    U, S, Vh = sla.svd(mat, full_matrices=False, check_finite=False, lapack_driver="gesvd")
    if settings.residual_mode:
        rank = rank_by_residual(operator, b_loc, U, S, Vh, exact, settings.truncation_tol, damp, max_rank)
    else:
        rank = rank_by_threshold(S, error_threshold, max_rank)
    if left:
        return Vh[:rank].reshape(rank, n, rr), U[:, :rank] * S[:rank]
    return U[:, :rank].reshape(rl, n, rank), S[:rank, None] * Vh[:rank]


# --------------------------------------------------------------------------
# centre shifts, residual train, enrichment (one_site.py, amen.py)
# --------------------------------------------------------------------------


def shift_right(x: Train, k: int, core: np.ndarray) -> None:
    """``_shift_center_right`` (``solvers/one_site.py:181-193``)."""
    q, r = sla.qr(core.reshape(-1, core.shape[-1]), mode="economic")
    x.cores[k] = q.reshape(core.shape[0], core.shape[1], 1, q.shape[1])
    x.cores[k + 1] = _mul_left(r, x.cores[k + 1])
    x.orth_center = k + 1


def shift_left(x: Train, k: int, core: np.ndarray) -> None:
    """``_shift_center_left`` (``solvers/one_site.py:196-209``)."""
    q, r = sla.qr(core.reshape(core.shape[0], -1).T, mode="economic")
    x.cores[k] = q.T.reshape(q.shape[1], core.shape[1], 1, core.shape[2])
    x.cores[k - 1] = _mul_right(x.cores[k - 1], r.T)
    x.orth_center = k - 1


def residual_core(k, lzb, rzb, lzax, rzax, A: Train, b: Train, x: Train, x_core=None) -> np.ndarray:
    """Projection of ``b - A x`` onto z's frame at site ``k``
    (``solvers/amen.py:109-159``); three GEMMs for the ``A x`` part."""
    bp = local_rhs(lzb[k], b.cores[k], rzb[k]).reshape(lzb[k].shape[1], b.cores[k].shape[1], rzb[k].shape[1])
    if x_core is None:
        x_core = x.cores[k][:, :, 0, :]
    left, core, right = lzax[k], A.cores[k], rzax[k]
    xl, al, zl = left.shape
    _, rows, cols, ar = core.shape
    xr, _, zr = right.shape
    s = left.transpose(2, 1, 0).reshape(zl * al, xl) @ x_core.reshape(xl, cols * xr)
    s = s.reshape(zl, al, cols, xr).transpose(0, 3, 1, 2).reshape(zl * xr, al * cols)
    s = s @ core.transpose(0, 2, 1, 3).reshape(al * cols, rows * ar)
    s = s.reshape(zl, xr, rows, ar).transpose(0, 2, 1, 3).reshape(zl * rows, xr * ar)
    s = s @ right.reshape(xr * ar, zr)
    return bp - s.reshape(zl, rows, zr)


def fit_residual(A: Train, b: Train, x: Train, z: Train, sweeps: int = 1) -> Train:
    """ALS fit of z to ``b - A x`` (``solvers/amen.py:162-224``)."""
    d = len(z)
    rzb, rzax, lzb, lzax = [None] * d, [None] * d, [None] * d, [None] * d
    for i in range(d - 1, -1, -1):
        env_right(rzb, i, z, b)
        env_right(rzax, i, z, x, A)
    for _ in range(sweeps):
        for k in range(d - 1):
            env_left(lzb, k, z, b)
            env_left(lzax, k, z, x, A)
            shift_right(z, k, residual_core(k, lzb, rzb, lzax, rzax, A, b, x))
        env_left(lzb, d - 1, z, b)
        env_left(lzax, d - 1, z, x, A)
        for k in range(d - 1, -1, -1):
            env_right(rzb, k, z, b)
            env_right(rzax, k, z, x, A)
            core = residual_core(k, lzb, rzb, lzax, rzax, A, b, x)
            if k > 0:
                shift_left(z, k, core)
            else:
                z.cores[0] = core.reshape(1, core.shape[1], 1, core.shape[2])
                z.orth_center = 0
    return z


def enrich_right(x: Train, k, core, carry, block, max_rank=None) -> None:
    """``_enrich_right`` (``solvers/amen.py:325-360``)."""
    enriched = np.concatenate([core, block], axis=2)
    pad = np.zeros((block.shape[2], carry.shape[1]))
    x.cores[k + 1] = _mul_left(np.concatenate([carry, pad], axis=0), x.cores[k + 1])
    shift_right(x, k, enriched)
    if max_rank is not None and x.cores[k].shape[3] > max_rank:
        x.cores[k] = x.cores[k][:, :, :, :max_rank]
        x.cores[k + 1] = x.cores[k + 1][:max_rank]


def enrich_left(x: Train, k, core, carry, block, max_rank=None) -> None:
    """``_enrich_left`` (``solvers/amen.py:363-392``)."""
    enriched = np.concatenate([core, block], axis=0)
    pad = np.zeros((carry.shape[0], block.shape[0]))
    x.cores[k - 1] = _mul_right(x.cores[k - 1], np.concatenate([carry, pad], axis=1))
    shift_left(x, k, enriched)
    if max_rank is not None and x.cores[k].shape[0] > max_rank:
        x.cores[k] = x.cores[k][:max_rank]
        x.cores[k - 1] = x.cores[k - 1][:, :, :, :max_rank]


def _local_solve_one_site(k, x, A, b, lA, rA, lb, rb, settings: Settings, info: Info):
    """``_solve_local_one_site`` (``solvers/one_site.py:118-178``)."""
    size = x.bonds[k] * x.row_modes[k] * x.bonds[k + 1]
    b_loc = local_rhs(lb[k], b.cores[k], rb[k])
    iterative = settings.iterative is not None and size > settings.direct_solve_size
    if iterative:
        op = local_operator(lA[k], A.cores[k], rA[k])
        warm = x.cores[k][:, :, 0, :].reshape(-1)
        if warm.size != size:
            warm = None
        fb = (lambda: local_matrix(lA[k], A.cores[k], rA[k])) if settings.allow_dense_fallback else None
    else:
        op = local_matrix(lA[k], A.cores[k], rA[k])
        warm, fb = None, None
    u, op = solve_local(op, b_loc, settings, iterative, warm, fb, info)
    return u, op, b_loc


def amen(A: Train, b: Train, x0: Optional[Train] = None, kickrank=4, error_threshold=1e-7,
         max_rank=None, max_sweeps=1, residual_tol=None, residual_damp=2.0,
         stagnation_factor="auto", local_solver="auto", direct_solve_size=1000,
         local_rtol=None, allow_dense_fallback=False, symmetric=False, seed=None,
         return_info=True, time_limit=None):
    """AMEn one-site sweep with residual enrichment (``solvers/amen.py:395-725``).

    Returns ``(x, info)``.  The per-sweep monitor restates
    ``_SweepMonitor.record`` (``solvers/common.py:504-592``).  With
    ``time_limit`` (seconds, host clock) the solve stops after the first
    local step that ends past it, with stop reason "time_limit" (the
    per-solve limit of the reference's benchmark runner,
    ``benchmarks/poisson.py:95-143``); the solution is then not valid.
    """
    import time as _time

    t_start = _time.perf_counter()

    def over_time():
        return time_limit is not None and _time.perf_counter() - t_start > time_limit

    if kickrank <= 0:
        raise ValueError("kickrank must be a positive integer")
    if max_rank is not None and max_rank <= 0:
        raise ValueError("max_rank must be a positive integer")
    if residual_damp < 1.0:
        raise ValueError("residual_damp must be >= 1")
    d = len(A)
    st = resolve_settings(max_sweeps, residual_tol, stagnation_factor, local_solver, symmetric,
                          direct_solve_size, return_info, local_rtol, allow_dense_fallback,
                          max(2 * (d - 1), 1))
    if x0 is None:
        x0 = ones(b.row_modes, ranks=b.bonds)
    x = x0.copy()
    if x.orth_center != 0:
        orthonormalize(x, "right")
    z = rand(b.row_modes, ranks=kickrank, seed=seed)
    orthonormalize(z, "right")
    fit_residual(A, b, x, z, sweeps=1)

    envs = {name: [None] * d for name in ("lA", "rA", "lb", "rb", "lzb", "rzb", "lzax", "rzax", "lxz", "rxz")}
    E = envs

    def build_left(k):
        env_left(E["lA"], k, x, x, A)
        env_left(E["lb"], k, x, b)
        env_left(E["lzb"], k, z, b)
        env_left(E["lzax"], k, z, x, A)
        env_left(E["lxz"], k, x, z)

    def build_right(k):
        env_right(E["rA"], k, x, x, A)
        env_right(E["rb"], k, x, b)
        env_right(E["rzb"], k, z, b)
        env_right(E["rzax"], k, z, x, A)
        env_right(E["rxz"], k, x, z)

    for i in range(d - 1, -1, -1):
        build_right(i)

    info = Info()
    b_norm = tt_norm(b) if st.track_residual else None
    for sweep in range(st.max_sweeps):
        for k in range(d - 1):
            build_left(k)
            u, op, b_loc = _local_solve_one_site(k, x, A, b, E["lA"], E["rA"], E["lb"], E["rb"], st, info)
            core3 = u.reshape(x.bonds[k], x.row_modes[k], x.bonds[k + 1])
            z_new = residual_core(k, E["lzb"], E["rzb"], E["lzax"], E["rzax"], A, b, x, x_core=core3)
            core, carry = truncate_core(core3, False, st, error_threshold, max_rank, op, b_loc, residual_damp)
            block = np.einsum("ba,bin->ain", E["lxz"][k], z_new)
            enrich_right(x, k, core, carry, block, max_rank)
            shift_right(z, k, z_new)
            if over_time():
                info.stop_reason = "time_limit"
                return x, info
        build_left(d - 1)
        for k in range(d - 1, -1, -1):
            build_right(k)
            u, op, b_loc = _local_solve_one_site(k, x, A, b, E["lA"], E["rA"], E["lb"], E["rb"], st, info)
            core3 = u.reshape(x.bonds[k], x.row_modes[k], x.bonds[k + 1])
            z_new = residual_core(k, E["lzb"], E["rzb"], E["lzax"], E["rzax"], A, b, x, x_core=core3)
            if k == 0:
                x.cores[0] = core3.reshape(1, core3.shape[1], 1, core3.shape[2])
                x.orth_center = 0
                z.cores[0] = z_new.reshape(1, z_new.shape[1], 1, z_new.shape[2])
                z.orth_center = 0
            else:
                core, carry = truncate_core(core3, True, st, error_threshold, max_rank, op, b_loc, residual_damp)
                block = _mul_right(z_new, E["rxz"][k])
                enrich_left(x, k, core, carry, block, max_rank)
                shift_left(z, k, z_new)
            if over_time():
                info.stop_reason = "time_limit"
                return x, info
        info.num_sweeps_run = sweep + 1
        info.max_bonds.append(max(x.bonds))
        if st.track_residual:
            res = relative_residual(A, b, x, b_norm=b_norm)
            info.residuals.append(res)
            if st.residual_tol is not None and res <= st.residual_tol:
                info.stop_reason = "converged"
                break
            if (st.stagnation_factor is not None and len(info.residuals) >= 2
                    and info.residuals[-1] > st.stagnation_factor * info.residuals[-2]):
                info.stop_reason = "stagnated"
                break
    # amen.py:710-720: QR cleanup of bonds above the product of the modes
    redundant = [k for k in range(1, d) if x.bonds[k] > math.prod(x.row_modes[:k])]
    if redundant:
        orthonormalize(x, "left", center_position=redundant[-1])
        orthonormalize(x, "right", center_position=0)
    return x, info


def als(A: Train, b: Train, x0: Optional[Train] = None, max_sweeps=4, residual_tol=None,
        stagnation_factor="auto", local_solver="auto", direct_solve_size=1000, local_rtol=None,
        allow_dense_fallback=False, symmetric=False, return_info=True):
    """ALS one-site sweeps (``solvers/als.py:57-212``): AMEn's local solves
    and centre shifts without the residual train, enrichment or truncation,
    so the bonds of ``x0`` never change.  Returns ``(x, info)``; the
    per-sweep monitor is the one of ``amen`` (``solvers/common.py:504-592``).
    """
    d = len(A)
    st = resolve_settings(max_sweeps, residual_tol, stagnation_factor, local_solver, symmetric,
                          direct_solve_size, return_info, local_rtol, allow_dense_fallback, 1)
    if x0 is None:
        x0 = ones(b.row_modes, ranks=b.bonds)
    x = x0.copy()
    if x.orth_center != 0:
        orthonormalize(x, "right")
    E = {name: [None] * d for name in ("lA", "rA", "lb", "rb")}
    for i in range(d - 1, -1, -1):  # als.py:144-146
        env_right(E["rA"], i, x, x, A)
        env_right(E["rb"], i, x, b)
    info = Info()
    b_norm = tt_norm(b) if st.track_residual else None
    for sweep in range(st.max_sweeps):
        for k in range(d - 1):  # als.py:153-170
            env_left(E["lA"], k, x, x, A)
            env_left(E["lb"], k, x, b)
            u, _, _ = _local_solve_one_site(k, x, A, b, E["lA"], E["rA"], E["lb"], E["rb"], st, info)
            shift_right(x, k, u.reshape(x.bonds[k], x.row_modes[k], x.bonds[k + 1]))
        env_left(E["lA"], d - 1, x, x, A)  # als.py:172-175
        env_left(E["lb"], d - 1, x, b)
        for k in range(d - 1, -1, -1):  # als.py:177-201
            env_right(E["rA"], k, x, x, A)
            env_right(E["rb"], k, x, b)
            u, _, _ = _local_solve_one_site(k, x, A, b, E["lA"], E["rA"], E["lb"], E["rb"], st, info)
            core = u.reshape(x.bonds[k], x.row_modes[k], x.bonds[k + 1])
            if k == 0:
                x.cores[0] = core.reshape(core.shape[0], core.shape[1], 1, core.shape[2])
                x.orth_center = 0
            else:
                shift_left(x, k, core)
        info.num_sweeps_run = sweep + 1
        info.max_bonds.append(max(x.bonds))
        if st.track_residual:
            res = relative_residual(A, b, x, b_norm=b_norm)
            info.residuals.append(res)
            if st.residual_tol is not None and res <= st.residual_tol:
                info.stop_reason = "converged"
                break
            if (st.stagnation_factor is not None and len(info.residuals) >= 2
                    and info.residuals[-1] > st.stagnation_factor * info.residuals[-2]):
                info.stop_reason = "stagnated"
                break
    return x, info


def local_rhs_pair(left_b, b1, b2, right_b) -> np.ndarray:
    """Two-site right-hand side (``solvers/two_site.py:28-49``), indexed
    (frame bond, mode k, mode k+1, frame bond) and flattened."""
    t = np.tensordot(left_b, b1[:, :, 0, :], axes=(0, 0))        # (i, j, b)
    t = np.tensordot(t, b2[:, :, 0, :], axes=(2, 0))             # (i, j, k, c)
    return np.tensordot(t, right_b, axes=(3, 0)).reshape(-1)     # (i, j, k, l)


def local_matrix_pair(left_A, A1, A2, right_A) -> np.ndarray:
    """Explicit two-site operator (``solvers/two_site.py:52-79``): the
    one-site operator of the merged core ``A1 A2`` (row modes and column
    modes of the pair merged), which orders rows (frame bond, row k,
    row k+1, frame bond) and columns likewise on the target side."""
    return local_matrix(left_A, merge_cores([A1, A2]), right_A)


def local_operator_pair(left_A, A1, A2, right_A):
    """Matrix-free two-site operator (``solvers/two_site.py:82-127``): the
    matrix-free one-site operator of the merged core ``A1 A2``."""
    return local_operator(left_A, merge_cores([A1, A2]), right_A)


def _pair_warm_start(x: Train, k: int, center):
    """Current supercore of sites k, k+1 (``solvers/two_site.py:130-153``),
    with the block left by the last split in place of its stale core."""
    left, right = x.cores[k][:, :, 0, :], x.cores[k + 1][:, :, 0, :]
    if center is not None:
        if center[0] == k:
            left = center[1]
        elif center[0] == k + 1:
            right = center[1]
    if left.shape[-1] != right.shape[0]:
        return None
    return np.tensordot(left, right, axes=(2, 0)).reshape(-1)


def _local_solve_two_site(k, x, A, b, bonds, E, st: Settings, error_threshold, max_rank, damp,
                          center, info: Info):
    """``_solve_local_two_site`` (``solvers/two_site.py:156-241``): solve the
    projected system of the supercore, split it by SVD and pick the rank of
    the shared bond.  Returns (U, S, Vh, rank)."""
    rows, cols = bonds[k] * x.row_modes[k], x.row_modes[k + 1] * bonds[k + 2]
    size = rows * cols
    b_loc = local_rhs_pair(E["lb"][k], b.cores[k], b.cores[k + 1], E["rb"][k + 1])
    ops = (E["lA"][k], A.cores[k], A.cores[k + 1], E["rA"][k + 1])
    iterative = st.iterative is not None and size > st.direct_solve_size
    if iterative:
        operator = local_operator_pair(*ops)
        warm = _pair_warm_start(x, k, center)
        if warm is not None and warm.size != size:
            warm = None
        fallback = (lambda: local_matrix_pair(*ops)) if st.allow_dense_fallback else None
    else:
        operator, warm, fallback = local_matrix_pair(*ops), None, None
    u, operator = solve_local(operator, b_loc, st, iterative, warm, fallback, info)
    exact = float(np.linalg.norm(operator @ u - b_loc)) if st.residual_mode else 0.0
    U, S, Vh = sla.svd(u.reshape(rows, cols), full_matrices=False, check_finite=False,
                       lapack_driver="gesvd")
    if st.residual_mode:
        rank = rank_by_residual(operator, b_loc, U, S, Vh, exact, st.truncation_tol, damp, max_rank)
    else:
        rank = rank_by_threshold(S, error_threshold, max_rank)
    return U, S, Vh, rank


def mals(A: Train, b: Train, x0: Optional[Train] = None, max_rank=None, max_sweeps=2,
         residual_tol=None, residual_damp=2.0, stagnation_factor="auto", error_threshold=1e-7,
         local_solver="auto", direct_solve_size=1000, local_rtol=None, allow_dense_fallback=False,
         symmetric=False, return_info=True):
    """MALS two-site sweeps (``solvers/mals.py:61-292``).  Left to right
    the supercores of sites (k, k+1), k < d - 2, are solved and split, the
    left factor kept as core k and the right factor held as the warm-start
    block of site k+1; right to left every pair is solved again, the right
    factor kept as core k+1 (and the left factor times S as core 0 at the
    end).  The truncation budget is shared by 2d - 3 splits per sweep.
    Returns ``(x, info)``."""
    if max_rank is not None and max_rank <= 0:
        raise ValueError(f"max_rank must be a positive integer, got {max_rank}")
    if residual_damp < 1.0:
        raise ValueError(f"residual_damp must be >= 1, got {residual_damp}")
    d = len(A)
    st = resolve_settings(max_sweeps, residual_tol, stagnation_factor, local_solver, symmetric,
                          direct_solve_size, return_info, local_rtol, allow_dense_fallback,
                          max(2 * d - 3, 1))
    if x0 is None:
        x0 = ones(b.row_modes, ranks=b.bonds)
    x = x0.copy()
    if x.orth_center != 0:
        orthonormalize(x, "right")
    E = {name: [None] * d for name in ("lA", "rA", "lb", "rb")}
    for i in range(d - 1, 0, -1):  # mals.py:196-198
        env_right(E["rA"], i, x, x, A)
        env_right(E["rb"], i, x, b)
    bonds = list(x.bonds)
    info = Info()
    b_norm = tt_norm(b) if st.track_residual else None
    center = None
    args = (st, error_threshold, max_rank, residual_damp)
    for sweep in range(st.max_sweeps):
        for k in range(d - 1):  # mals.py:216-249
            env_left(E["lA"], k, x, x, A)
            env_left(E["lb"], k, x, b)
            if k == d - 2:
                continue
            U, S, Vh, nb = _local_solve_two_site(k, x, A, b, bonds, E, *args, center, info)
            center = (k + 1, (S[:nb, None] * Vh[:nb]).reshape(nb, x.row_modes[k + 1],
                                                                bonds[k + 2]))
            x.cores[k] = U[:, :nb].reshape(bonds[k], x.row_modes[k], 1, nb)
            bonds[k + 1] = nb
            x.orth_center = k + 1
        for k in range(d - 2, -1, -1):  # mals.py:252-283
            env_right(E["rA"], k + 1, x, x, A)
            env_right(E["rb"], k + 1, x, b)
            U, S, Vh, nb = _local_solve_two_site(k, x, A, b, bonds, E, *args, center, info)
            us = U[:, :nb] * S[:nb]
            center = (k, us.reshape(bonds[k], x.row_modes[k], nb))
            x.cores[k + 1] = Vh[:nb].reshape(nb, x.row_modes[k + 1], 1, bonds[k + 2])
            bonds[k + 1] = nb
            if k == 0:
                x.cores[0] = us.reshape(bonds[0], x.row_modes[0], 1, nb)
            x.orth_center = k
        info.num_sweeps_run = sweep + 1
        info.max_bonds.append(max(bonds))
        if st.track_residual:
            res = relative_residual(A, b, x, b_norm=b_norm)
            info.residuals.append(res)
            if st.residual_tol is not None and res <= st.residual_tol:
                info.stop_reason = "converged"
                break
            if (st.stagnation_factor is not None and len(info.residuals) >= 2
                    and info.residuals[-1] > st.stagnation_factor * info.residuals[-2]):
                info.stop_reason = "stagnated"
                break
    return x, info


def tt_svd(tensor: np.ndarray, error: float = 1e-12, max_rank=None, physical_indexes=None,
           ttm: bool = False) -> Train:
    """TT-SVD (``tensor_train.py:1138-1247``): left to right, the unfolding
    (bond * modes_i, rest) is split by an SVD (gesvd), truncated with
    ``truncated_bond`` at ``delta = error / sqrt(ndim - 1) * ||tensor||``
    and the remainder ``U^T @ matrix`` carried on."""
    t = np.array(tensor, dtype=np.float64, copy=True)
    if t.ndim == 1 and physical_indexes is None:
        raise ValueError("1-D tensor needs physical_indexes")
    if physical_indexes is not None:
        if ttm:
            d = len(physical_indexes)
            perm = tuple(np.arange(2 * d).reshape(2, d).T.flatten())
            t = np.transpose(t, perm).reshape([x for pair in physical_indexes for x in pair])
            phys = [tuple(p) for p in physical_indexes]
        else:
            t = t.reshape(physical_indexes)
            phys = [(x, 1) for x in physical_indexes]
    else:
        if ttm:
            raise ValueError("TTM needs physical_indexes")
        phys = [(x, 1) for x in t.shape]
    norm = float(np.linalg.norm(t))
    delta = error / np.sqrt(t.ndim - 1) * norm
    cores, bond = [], 1
    for i in range(len(phys) - 1):
        rest = int(np.prod([int(np.prod(p)) for p in phys[i + 1:]]))
        matrix = t.reshape(bond * int(np.prod(phys[i])), rest)
        u, s, _ = sla.svd(matrix, full_matrices=False, check_finite=False, lapack_driver="gesvd")
        nb = truncated_bond(s, delta, max_rank)
        ut = u[:, :nb]
        cores.append(ut.reshape((bond,) + tuple(phys[i]) + (nb,)))
        c = ut.T @ matrix
        if i == len(phys) - 2:
            cores.append(c.reshape((c.shape[0],) + tuple(phys[i + 1]) + (1,)))
        else:
            bond = c.shape[0]
            t = c
    return Train(cores, orth_center=len(cores) - 1)


def tt_to_qtt(t: Train, mode_size: int = 2, error: float = 1e-12, max_rank=None) -> Train:
    """Quantisation of every mode (``tensor_train.py:942-1066``): after a
    right QR sweep, each core of mode ``mode_size^q`` is split left to right
    into q cores by q - 1 truncated SVDs (row and column halves kept
    paired), and the remainder of each group is pushed into the next core
    by one more SVD; one error budget ``error / sqrt(#SVDs) * ||t||``."""
    if mode_size < 2:
        raise ValueError("mode_size must be at least 2")
    if max_rank is not None and max_rank <= 0:
        raise ValueError("max_rank must be a positive integer.")
    nums = []
    for i, m in enumerate(t.row_modes):
        q = 0
        while mode_size ** q < m:
            q += 1
        if mode_size ** q != m:
            raise ValueError(f"Row mode {m} not a power of {mode_size}")
        if t.is_ttm() and mode_size ** q != t.col_modes[i]:
            raise ValueError("Column mode size of TTM not a power of mode size")
        nums.append(q)
    rms = mode_size
    cms = mode_size if t.is_ttm() else 1
    count = max(1, sum(max(0, q - 1) for q in nums) + len(t) - 1)
    tt = orthonormalize(t.copy(), "right")
    delta = error / np.sqrt(count) * tt_norm(tt)
    out = []
    for i, q in enumerate(nums):
        core = tt.cores[i]
        lb, rb = core.shape[0], core.shape[-1]
        for j in range(q - 1, 0, -1):
            core = core.reshape(lb, rms, rms ** j, cms, cms ** j, rb).transpose(0, 1, 3, 2, 4, 5)
            matrix = core.reshape(lb * rms * cms, rms ** j * cms ** j * rb)
            u, s, _ = sla.svd(matrix, full_matrices=False, check_finite=False, lapack_driver="gesvd")
            nb = truncated_bond(s, delta, max_rank)
            out.append(u[:, :nb].reshape(lb, rms, cms, nb))
            core = u[:, :nb].T @ matrix
            lb = nb
        if i < len(t) - 1:
            matrix = core.reshape(lb * rms * cms, rb)
            u, s, _ = sla.svd(matrix, full_matrices=False, check_finite=False, lapack_driver="gesvd")
            nb = truncated_bond(s, delta, max_rank)
            out.append(u[:, :nb].reshape(lb, rms, cms, nb))
            tt.cores[i + 1] = np.tensordot(u[:, :nb].T @ matrix, tt.cores[i + 1], axes=(1, 0))
        else:
            out.append(core.reshape(lb, rms, cms, rb))
    return Train(out, orth_center=len(out) - 1)


def merge_cores(cores: List[np.ndarray]) -> np.ndarray:
    """Product of consecutive cores as one core (``tensor_train.py:57-92``,
    ``_contract_cores`` and ``_merge_cores``): contract the bonds left to
    right, then gather the row modes in front of the column modes."""
    lb, rb = cores[0].shape[0], cores[-1].shape[-1]
    rows = [c.shape[1] for c in cores]
    cols = [c.shape[2] for c in cores]
    m = cores[0].reshape(-1, cores[0].shape[-1])
    for c in cores[1:]:
        m = (m @ c.reshape(c.shape[0], -1)).reshape(-1, c.shape[-1])
    # axes of size 1 are left out of the transpose (a group of many such
    # cores would exceed NumPy's axis limit otherwise)
    axes = [(k % 2, x) for k, x in enumerate(v for pair in zip(rows, cols) for v in pair) if x > 1]
    inter = m.reshape([lb] + [x for _, x in axes] + [rb])
    perm = ([0] + [1 + k for k, (kind, _) in enumerate(axes) if kind == 0]
            + [1 + k for k, (kind, _) in enumerate(axes) if kind == 1] + [len(axes) + 1])
    return inter.transpose(perm).reshape(lb, int(np.prod(rows)), int(np.prod(cols)), rb)


def qtt_to_tt(t: Train, physical_indexes, error: float = 1e-12, max_rank=None) -> Train:
    """Inverse quantisation (``tensor_train.py:1072-1135``): consecutive
    cores are grouped so that each group's row (and, for a TTM, column)
    modes multiply to the requested index, each group is merged into one
    core, and the result is rounded by ``truncate``."""
    ttm = t.is_ttm()
    groups = []
    pos = 0
    for i, idx in enumerate(physical_indexes):
        rt, ct = (idx if ttm else (idx, 1))
        pr = pc = 1
        n = 0
        while n == 0 or pr != rt or pc != ct:
            if pos + n >= len(t):
                raise ValueError(f"Not enough QTT cores to match physical index for core {i}")
            pr *= t.row_modes[pos + n]
            pc *= t.col_modes[pos + n]
            n += 1
            if pr > rt or pc > ct:
                raise ValueError(f"QTT mode size exceeds the original mode size for core {i}")
        groups.append((pos, n))
        pos += n
    if pos != len(t):
        raise ValueError(f"Physical indexes cover only {pos} of {len(t)} QTT cores")
    merged = Train([merge_cores(t.cores[p:p + n]) for p, n in groups])
    return truncate(merged, error=error, max_rank=max_rank)
