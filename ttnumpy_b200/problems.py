"""Host-side input builders for the tensor-train solve workloads.

These build operators (TTM cores) and right-hand sides (TT cores) as NumPy
float64 arrays on the host; the solvers upload them.  Input preparation is
host work in the reference too (``ttnumpy/tensor_train.py:1138-1387``,
``benchmarks/poisson_problem.py:97-298``).

Workloads:

* ``laplacian_nd``: the d-dimensional Dirichlet Laplacian
  ``sum_j I x .. x L_j x .. x I`` with ``L = (1/h^2) tridiag(-1, 2, -1)``,
  ``h = 1/(n+1)``, TTM bond 2.
* ``qtt_poisson_2d``: the 2-D Dirichlet Laplacian on a ``2^N x 2^N`` grid in
  QTT form (``2N`` cores of mode 2, y digits first, most significant digit
  first) with the sampled right-hand side ``f(x, y)`` compressed by TT-SVD.
  The operator has the sign of the reference benchmark (diagonal ``-4/h^2``)
  and the right-hand side is ``-f``, as ``solve_poisson_tt`` passes it
  (``benchmarks/poisson_problem.py:343-365``).
* ``parametric_diffusion``: ``-div(a grad u) = 1`` on ``[0,1]^d`` with
  ``a(x) = 1 + c * sum_k theta_k sin(k pi x_k)``; TTM bond 4.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

import numpy as np


def _stiffness(n: int, h: float, coeff_mid: Optional[np.ndarray] = None) -> np.ndarray:
    """1-D Dirichlet stiffness ``-(c u')'`` on ``n`` interior nodes.

    ``coeff_mid`` holds the coefficient at the ``n + 1`` cell midpoints
    ``(i + 1/2) h``, ``i = 0..n``; None means the constant 1.
    """
    c = np.ones(n + 1) if coeff_mid is None else np.asarray(coeff_mid, dtype=np.float64)
    main = (c[:-1] + c[1:]) / h**2
    off = -c[1:-1] / h**2
    return np.diag(main) + np.diag(off, 1) + np.diag(off, -1)


def laplacian_nd(d: int, n: int) -> List[np.ndarray]:
    """TTM cores of ``sum_j I..L_j..I`` with ``L = (1/h^2) tridiag(-1,2,-1)``.

    Bond states: 1 = "the L factor is still to come", 0 = "already placed".
    """
    h = 1.0 / (n + 1)
    L = _stiffness(n, h)
    eye = np.eye(n)
    first = np.zeros((1, n, n, 2))
    first[0, :, :, 0] = L
    first[0, :, :, 1] = eye
    mid = np.zeros((2, n, n, 2))
    mid[0, :, :, 0] = eye
    mid[1, :, :, 0] = L
    mid[1, :, :, 1] = eye
    last = np.zeros((2, n, n, 1))
    last[0, :, :, 0] = eye
    last[1, :, :, 0] = L
    return [first] + [mid.copy() for _ in range(d - 2)] + [last]


def tt_svd_vector(tensor: np.ndarray, modes: Sequence[int], error: float) -> List[np.ndarray]:
    """TT-SVD of a dense vector into cores ``(r, n, 1, r')``.

    Sequential truncated SVDs with the per-split budget
    ``error * ||t|| / sqrt(d - 1)`` and the tail-norm rank rule with the
    ``eps * len * sigma_1`` noise floor, the published TT-SVD algorithm
    (Oseledets 2011, Alg. 1) as the reference applies it
    (``ttnumpy/tensor_train.py:1138-1247``, ``ttnumpy/utils.py:22-69``).
    """
    modes = list(modes)
    d = len(modes)
    t = np.asarray(tensor, dtype=np.float64).reshape(-1)
    delta = error / math.sqrt(d - 1) * np.linalg.norm(t)
    cores = []
    bond = 1
    rest = t
    for i in range(d - 1):
        mat = rest.reshape(bond * modes[i], -1)
        u, s, _ = np.linalg.svd(mat, full_matrices=False)
        vals = s.copy()
        vals[vals <= np.finfo(np.float64).eps * vals.size * vals[0]] = 0.0
        tail = np.cumsum((vals**2)[::-1])[::-1]
        nb = max(1, int(np.count_nonzero(tail > delta * delta)))
        u = u[:, :nb]
        cores.append(u.reshape(bond, modes[i], 1, nb))
        rest = u.T @ mat
        bond = nb
    cores.append(rest.reshape(bond, modes[-1], 1, 1))
    return cores


def _qtt_from_matrix(matrix: np.ndarray, levels: int) -> List[np.ndarray]:
    """Exact QTT cores ``(r, 2, 2, r')`` of a ``2^L x 2^L`` matrix by TT-SVD.

    The row and column index are split into binary digits, most
    significant first, and digit pairs ``(i_k, j_k)`` are merged into one
    core mode of size 4 for the decomposition.
    """
    t = matrix.reshape([2] * (2 * levels))
    perm = [v for k in range(levels) for v in (k, levels + k)]
    t = t.transpose(perm)
    cores = tt_svd_vector(t, [4] * levels, 0.0)
    return [c.reshape(c.shape[0], 2, 2, c.shape[3]) for c in cores]


def qtt_laplacian_2d(levels: int, h: float) -> List[np.ndarray]:
    """QTT cores of the 2-D Laplacian ``T_y (x) I + I (x) T_x`` with
    ``T = (1/h^2) tridiag(1, -2, 1)`` (negative definite, like the reference
    benchmark operator), y digits on the first ``levels`` cores."""
    size = 2**levels
    T = -_stiffness(size, h)
    t_cores = _qtt_from_matrix(T, levels)
    eye = np.eye(2).reshape(1, 2, 2, 1)
    y_term = t_cores + [eye.copy() for _ in range(levels)]
    x_term = [eye.copy() for _ in range(levels)] + t_cores
    cores = []
    d = 2 * levels
    for k in range(d):
        a, b = y_term[k], x_term[k]
        ra = [a.shape[0], a.shape[3]]
        rb = [b.shape[0], b.shape[3]]
        left = 1 if k == 0 else ra[0] + rb[0]
        right = 1 if k == d - 1 else ra[1] + rb[1]
        out = np.zeros((left, 2, 2, right))
        if k == 0:
            out[:, :, :, : ra[1]] = a
            out[:, :, :, ra[1]:] = b
        elif k == d - 1:
            out[: ra[0]] = a
            out[ra[0]:] = b
        else:
            out[: ra[0], :, :, : ra[1]] = a
            out[ra[0]:, :, :, ra[1]:] = b
        cores.append(out)
    return cores


@dataclass
class Problem:
    """One linear system ``A x = b`` in TT form plus how to solve it."""

    name: str
    A: List[np.ndarray]
    b: List[np.ndarray]
    x0: Optional[List[np.ndarray]] = None
    meta: Optional[dict] = None


def qtt_poisson_2d(levels: int = 10,
                   rhs: Callable[[np.ndarray, np.ndarray], np.ndarray] = None,
                   rhs_error: float = 1e-12) -> Problem:
    """2-D Poisson problem ``Lap u = -f`` on the unit square in QTT form.

    Interior nodes ``(i + 1) h`` with ``h = 1/(2^N + 1)``; ``f`` is sampled
    as ``f[y, x]`` and flattened y-major, as the reference benchmark does
    (``benchmarks/poisson_problem.py:215-298``).  The initial guess is the
    rank-3 all-ones train right-orthonormalised
    (``benchmarks/poisson_problem.py:343-347``), which the caller builds.
    """
    if rhs is None:
        rhs = lambda x, y: np.sin(np.pi * x) * np.sin(np.pi * y)  # noqa: E731
    K = 2**levels
    h = 1.0 / (K + 1)
    nodes = (np.arange(K) + 1) * h
    X, Y = np.meshgrid(nodes, nodes)  # X[y, x] = x_x, Y[y, x] = y_y
    f = rhs(X, Y)
    b = tt_svd_vector(-f.reshape(-1), [2] * (2 * levels), rhs_error)
    A = qtt_laplacian_2d(levels, h)
    return Problem(f"qtt_poisson_2d_N{levels}", A, b, meta={"levels": levels, "h": h})


def diffusion_operator(d: int, n: int, theta: np.ndarray, scale: float) -> List[np.ndarray]:
    """TTM cores of ``-div(a grad .)`` with ``a = 1 + sum_k f_k(x_k)``,
    ``f_k(x) = scale * theta_k * sin(k pi x)``, ``k = 1..d``.

    Axis ``j`` contributes ``(1 + sum_{k != j} f_k(x_k)) L_j + K_j[f_j]``,
    where ``L`` is the unit stiffness and ``K[f]`` the stiffness with
    coefficient ``f`` at the cell midpoints.  Summed over axes this is
    ``sum_j S_j + sum_{j != k} D_k L_j`` with ``S = L + K[f_j]`` and
    ``D_k = diag(f_k(x_k))``, a TTM of bond 4 with the states
    0 = nothing placed, 1 = a D placed (its L to come),
    2 = an L placed (its D to come), 3 = complete.
    """
    h = 1.0 / (n + 1)
    nodes = (np.arange(n) + 1) * h
    mids = (np.arange(n + 1) + 0.5) * h
    L = _stiffness(n, h)
    eye = np.eye(n)
    cores = []
    for m in range(d):
        freq = m + 1
        f_nodes = scale * theta[m] * np.sin(freq * np.pi * nodes)
        f_mids = scale * theta[m] * np.sin(freq * np.pi * mids)
        S = L + _stiffness(n, h, f_mids)
        D = np.diag(f_nodes)
        core = np.zeros((4, n, n, 4))
        core[0, :, :, 0] = eye
        core[0, :, :, 1] = D
        core[0, :, :, 2] = L
        core[0, :, :, 3] = S
        core[1, :, :, 1] = eye
        core[1, :, :, 3] = L
        core[2, :, :, 2] = eye
        core[2, :, :, 3] = D
        core[3, :, :, 3] = eye
        if m == 0:
            core = core[:1]
        if m == d - 1:
            core = core[:, :, :, 3:]
        cores.append(core)
    return cores


#: Coefficient amplitude of the parametric diffusion workload.  The
#: perturbation ``sum_k theta_k sin(k pi x_k)`` can reach ``d`` in absolute
#: value, so the amplitude is divided by ``d`` to keep ``a >= 0.5``.
def diffusion_scale(d: int) -> float:
    return 0.5 / d


def parametric_diffusion(d: int, n: int, theta: np.ndarray) -> Problem:
    A = diffusion_operator(d, n, theta, diffusion_scale(d))
    b = [np.ones((1, n, 1, 1)) for _ in range(d)]
    return Problem(f"diffusion_d{d}_n{n}", A, b, meta={"d": d, "n": n})


def diffusion_batch(count: int = 256, seed: int = 0,
                    d_range=(4, 12), modes=(16, 32, 64)) -> List[Problem]:
    """Batched parametric diffusion draws: ``d ~ U{4..12}``,
    ``n ~ U{16, 32, 64}``, ``theta_k ~ U(-1, 1)``, all from one generator."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        d = int(rng.integers(d_range[0], d_range[1] + 1))
        n = int(rng.choice(modes))
        theta = rng.uniform(-1.0, 1.0, size=d)
        out.append(parametric_diffusion(d, n, theta))
    return out


def random_tt(modes: Sequence[int], rank: int, seed: int) -> List[np.ndarray]:
    """Uniform [0, 1) cores drawn core by core from
    ``np.random.default_rng(seed)``, the distribution of the reference's
    ``tensor_train.rand`` (``ttnumpy/tensor_train.py:1350-1387``)."""
    rng = np.random.default_rng(seed)
    d = len(modes)
    ranks = [1] + [rank] * (d - 1) + [1]
    return [rng.random((ranks[i], modes[i], 1, ranks[i + 1])) for i in range(d)]


def large_diffusion(theta: np.ndarray, rhs_seed: int, n: int = 64, rank: int = 8) -> Problem:
    """The large request class: parametric diffusion in ``d = len(theta)``
    dimensions with mode size ``n`` and a random rank-``rank`` right-hand
    side (``random_tt`` with seed ``rhs_seed``)."""
    d = len(theta)
    A = diffusion_operator(d, n, theta, diffusion_scale(d))
    b = random_tt([n] * d, rank, seed=rhs_seed)
    return Problem(f"large_d{d}_n{n}", A, b, meta={"kind": "large", "d": d, "n": n})


#: Shares of the serving mix: large requests, then diffusion and QTT
#: Poisson in equal parts of the rest.
LARGE_SHARE = 0.1


def serving_request(rng: np.random.Generator, large_share: float = LARGE_SHARE,
                    large_d: int = 24, large_n: int = 64, large_rank: int = 8,
                    dims=(4, 12), modes=(16, 32, 64), levels=(3, 10)) -> Problem:
    """One request of the serving mix, drawn from ``rng``: with probability
    ``large_share`` a large diffusion solve (``d = large_d``, ``n =
    large_n``, random rank-``large_rank`` right-hand side); otherwise, with
    equal odds, a parametric diffusion draw (``d ~ U{dims}``, ``n ~
    U(modes)``, ``theta ~ U(-1, 1)``) or a 2-D QTT Poisson problem with
    ``2N`` cores, ``N ~ U{levels}``.  ``meta["kind"]`` names the class."""
    u = rng.random()
    if u < large_share:
        theta = rng.uniform(-1.0, 1.0, size=large_d)
        return large_diffusion(theta, int(rng.integers(1 << 31)), large_n, large_rank)
    if u < large_share + (1 - large_share) / 2:
        d = int(rng.integers(dims[0], dims[1] + 1))
        n = int(rng.choice(modes))
        p = parametric_diffusion(d, n, rng.uniform(-1.0, 1.0, size=d))
        p.meta["kind"] = "diffusion"
        return p
    N = int(rng.integers(levels[0], levels[1] + 1))
    base = _qtt_poisson_cached(N)
    return Problem(base.name, base.A, base.b, meta={"kind": "qtt", "levels": N})


_QTT_CACHE: dict = {}


def _qtt_poisson_cached(levels: int) -> Problem:
    """``qtt_poisson_2d(levels)`` built once per level (the TT-SVD of the
    right-hand side dominates building a request); requests share its
    read-only core arrays."""
    if levels not in _QTT_CACHE:
        _QTT_CACHE[levels] = qtt_poisson_2d(levels)
    return _QTT_CACHE[levels]


def serving_requests(count: int, seed: int = 0, **kw) -> List[Problem]:
    """``count`` requests of the serving mix from one generator seeded
    ``seed`` (see ``serving_request`` for the classes and keywords)."""
    rng = np.random.default_rng(seed)
    return [serving_request(rng, **kw) for _ in range(count)]


def serving_stream(count: int, rate: float, seed: int = 0, **kw):
    """Request stream: the requests of ``serving_requests(count, seed)``
    arriving as a Poisson process at ``rate`` per second (exponential gaps
    from a second generator seeded ``seed + 1``).  Returns
    ``[(arrival_time, Problem), ...]``."""
    reqs = serving_requests(count, seed, **kw)
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / rate, size=count)
    return list(zip(np.cumsum(gaps).tolist(), reqs))
