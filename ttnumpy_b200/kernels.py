"""Thin Python wrappers over the libttb200 C ABI.

Arguments are CUDA float64 ``torch.Tensor`` views; torch only supplies device
memory and the current stream.  Every function validates shapes, builds the
C problem structs and calls one entry point of ``include/ttb200.h``.  Scratch
memory comes from a per-device bump arena (:class:`Arena`) whose lifetime is
a ``with arena.scope():`` block; results never live in the arena.
"""

from __future__ import annotations

import contextlib
import ctypes as C
from typing import List, Optional, Sequence

import torch

from . import _lib
from ._lib import check

F64 = torch.float64


def device_ok() -> None:
    if not torch.cuda.is_available():
        raise RuntimeError("ttnumpy_b200 needs a CUDA device (B200, sm_100a); none is visible")


def lib():
    return _lib.load()


def stream() -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t: Optional[torch.Tensor]):
    return None if t is None else t.data_ptr()


def empty(*shape, device=None) -> torch.Tensor:
    return torch.empty(*shape, dtype=F64, device=device or "cuda")


class Arena:
    """Bump allocator for kernel scratch on the current stream.

    Memory handed out inside a ``scope()`` is reused after the scope ends;
    stream ordering makes that safe for work queued on one stream.
    """

    def __init__(self, doubles: int = 1 << 20):
        self.buf = None
        self.cap = doubles
        self.off = 0

    def take(self, n: int) -> torch.Tensor:
        n = max(32, (int(n) + 31) // 32 * 32)
        if self.buf is None or self.off + n > self.buf.numel():
            # a fresh block; views into the old one stay alive while used
            size = max(self.cap, 2 * (self.off + n))
            self.cap = size
            self.buf = torch.empty(size, dtype=F64, device="cuda")
            self.off = 0
        v = self.buf[self.off:self.off + n]
        self.off += n
        return v

    def take_int(self, n: int) -> torch.Tensor:
        return self.take((n + 1) // 2).view(torch.int32)[:n]

    @contextlib.contextmanager
    def scope(self):
        saved_buf, saved = self.buf, self.off
        try:
            yield self
        finally:
            if self.buf is saved_buf:
                self.off = saved


_arenas = {}


def arena() -> Arena:
    dev = torch.cuda.current_device()
    a = _arenas.get(dev)
    if a is None:
        a = _arenas[dev] = Arena()
    return a


def _strides(t: torch.Tensor):
    if t.dim() == 2:
        return 0, t.stride(0), t.stride(1), t.shape[0], t.shape[1], 1
    if t.dim() == 3:
        return t.stride(0), t.stride(1), t.stride(2), t.shape[1], t.shape[2], t.shape[0]
    raise ValueError("gemm operands must be 2-D or 3-D (batch first)")


# ---------------------------------------------------------------------------
# GEMM
# ---------------------------------------------------------------------------


def gemm_desc(a: torch.Tensor, b: torch.Tensor, c: torch.Tensor, alpha=1.0, beta=0.0):
    """C = alpha A B + beta C on 2-D or batch-first 3-D views (a batch of 1
    broadcasts with stride 0)."""
    a_bs, a_rs, a_cs, m, k, ab = _strides(a)
    b_bs, b_rs, b_cs, k2, n, bb = _strides(b)
    c_bs, c_rs, c_cs, m2, n2, cb = _strides(c)
    if k != k2 or m != m2 or n != n2:
        raise ValueError(f"gemm shape mismatch {tuple(a.shape)} {tuple(b.shape)} {tuple(c.shape)}")
    batch = cb
    if ab == 1:
        a_bs = 0
    if bb == 1:
        b_bs = 0
    if ab not in (1, batch) or bb not in (1, batch):
        raise ValueError("gemm batch mismatch")
    return _lib.Gemm(ptr(a), ptr(b), ptr(c), m, n, k, batch, a_rs, a_cs, a_bs, b_rs, b_cs, b_bs,
                     c_rs, c_cs, c_bs, float(alpha), float(beta))


def gemm_many(descs: Sequence) -> None:
    if not descs:
        return
    arr = (_lib.Gemm * len(descs))(*descs)
    check(lib().ttb_gemm(arr, len(descs), stream()), "ttb_gemm")


def gemm_3xtf32_many(descs: Sequence, status: Optional[torch.Tensor] = None) -> None:
    """The ttb_gemm problems on the tcgen05 tensor cores in 3xTF32
    (about 1e-6 relative accuracy); ``status`` (int32 device tensor) is set
    to 1 if a block gave up waiting on the tensor core."""
    if not descs:
        return
    arr = (_lib.Gemm * len(descs))(*descs)
    check(lib().ttb_gemm_3xtf32(arr, len(descs), ptr(status), stream()), "ttb_gemm_3xtf32")


def gemm(a, b, c, alpha=1.0, beta=0.0) -> torch.Tensor:
    gemm_many([gemm_desc(a, b, c, alpha, beta)])
    return c


def matmul(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    c = empty(a.shape[0], b.shape[1])
    return gemm(a, b, c)


# ---------------------------------------------------------------------------
# copies
# ---------------------------------------------------------------------------


def _pad4(shape, strides):
    shape = list(shape)
    strides = list(strides)
    while len(shape) < 4:
        shape.insert(0, 1)
        strides.insert(0, 0)
    return shape, strides


def copy_desc(src: Optional[torch.Tensor], dst: torch.Tensor, alpha=1.0,
              scale: Optional[torch.Tensor] = None, scale_axis: int = -1):
    """dst = alpha * (scale along ``scale_axis`` of dst) * src (src None: fill)."""
    if dst.dim() > 4:
        raise ValueError("copy supports up to 4 dimensions")
    shape, tstr = _pad4(dst.shape, dst.stride())
    if src is not None:
        if tuple(src.shape) != tuple(dst.shape):
            raise ValueError(f"copy shape mismatch {tuple(src.shape)} -> {tuple(dst.shape)}")
        _, sstr = _pad4(src.shape, src.stride())
    else:
        sstr = [0, 0, 0, 0]
    axis = -1
    if scale is not None:
        axis = scale_axis + (4 - dst.dim()) if scale_axis >= 0 else 4 + scale_axis
    return _lib.Copy(ptr(src), ptr(dst), ptr(scale), *shape, *sstr, *tstr, float(alpha), axis)


def copy_many(descs: Sequence) -> None:
    descs = [d for d in descs if d.d0 * d.d1 * d.d2 * d.d3 > 0]
    if not descs:
        return
    arr = (_lib.Copy * len(descs))(*descs)
    check(lib().ttb_copy(arr, len(descs), stream()), "ttb_copy")


def copy_(dst, src, alpha=1.0, scale=None, scale_axis=-1):
    copy_many([copy_desc(src, dst, alpha, scale, scale_axis)])
    return dst


def fill_(dst, value=0.0):
    copy_many([copy_desc(None, dst, value)])
    return dst


def zeros(*shape) -> torch.Tensor:
    return fill_(empty(*shape), 0.0)


# ---------------------------------------------------------------------------
# environments, local operator, projections
# ---------------------------------------------------------------------------


def env_desc(side: int, env, frame, target, out, op=None, work=None):
    """One projection step (side 0 = left, 1 = right); cores are 3-D
    ``(r, n, r')`` views of TT cores, op a 4-D TTM core."""
    if op is not None:
        t, R, f = env.shape
    else:
        (t, f), R = env.shape, 1
    if side == 0:
        f_, n, f2 = frame.shape
        t_, m, t2 = target.shape
        R2 = op.shape[3] if op is not None else 1
    else:
        f2, n, f_ = frame.shape
        t2, m, t_ = target.shape
        R2 = op.shape[0] if op is not None else 1
    if f_ != f or t_ != t:
        raise ValueError("environment/core bond mismatch")
    if op is None and n != m:
        raise ValueError("overlap environment needs equal modes")
    d = _lib.Env(ptr(env), ptr(frame), ptr(op), ptr(target), ptr(out), None, side, f, f2, t, t2,
                 R, R2, n, m)
    return d


def env_update(descs: List) -> None:
    """Run environment updates, taking scratch from the arena."""
    if not descs:
        return
    L = lib()
    ar = arena()
    with ar.scope():
        for d in descs:
            d.work = ar.take(L.ttb_env_work_doubles(C.byref(d))).data_ptr()
        arr = (_lib.Env * len(descs))(*descs)
        check(L.ttb_env_update(arr, len(descs), stream()), "ttb_env_update")


def local_desc(left, op, right, x, y, cols=1, alpha=1.0, beta=0.0):
    """y = alpha * B x + beta * y for the one-site operator B of
    (left, op, right); x holds ``cols`` vectors of (lt, m, rt)."""
    lt, R, lf = left.shape
    R_, n, m, R2 = op.shape
    rt, R2_, rf = right.shape
    if R_ != R or R2_ != R2:
        raise ValueError("operator bond mismatch")
    return _lib.Local(ptr(left), ptr(op), ptr(right), ptr(x), ptr(y), None, lt, lf, R, R2, n, m,
                      rt, rf, cols, float(alpha), float(beta))


def local_apply(descs: List) -> None:
    if not descs:
        return
    L = lib()
    ar = arena()
    with ar.scope():
        for d in descs:
            d.work = ar.take(L.ttb_local_work_doubles(C.byref(d))).data_ptr()
        arr = (_lib.Local * len(descs))(*descs)
        check(L.ttb_local_apply(arr, len(descs), stream()), "ttb_local_apply")


def local_matrix(left, op, right) -> torch.Tensor:
    """Explicit one-site matrix, column major: returns a (cols, rows) tensor
    whose row c is column c of the operator."""
    lt, R, lf = left.shape
    _, n, m, R2 = op.shape
    rt, _, rf = right.shape
    rows, cols = lf * n * rf, lt * m * rt
    out = empty(cols, rows)
    d = _lib.LocalMatrix(ptr(left), ptr(op), ptr(right), ptr(out), lt, lf, R, R2, n, m, rt, rf)
    arr = (_lib.LocalMatrix * 1)(d)
    check(lib().ttb_local_matrix(arr, 1, stream()), "ttb_local_matrix")
    return out


def project_desc(left, core, right, out, alpha=1.0, beta=0.0):
    """out (i, n, l) = alpha * sum Lb[a, i] core[a, n, c] Rb[c, l] + beta * out."""
    a, i = left.shape
    a_, n, c = core.shape
    c_, l = right.shape
    if a_ != a or c_ != c:
        raise ValueError("projection bond mismatch")
    return _lib.Project(ptr(left), ptr(core), ptr(right), ptr(out), None, a, i, n, c, l,
                        float(alpha), float(beta))


def project(descs: List) -> None:
    if not descs:
        return
    ar = arena()
    with ar.scope():
        for d in descs:
            d.work = ar.take(d.a * d.n * d.l).data_ptr()
        arr = (_lib.Project * len(descs))(*descs)
        check(lib().ttb_project(arr, len(descs), stream()), "ttb_project")


def hadamard(lhs: torch.Tensor, rhs: torch.Tensor) -> torch.Tensor:
    """Element-wise product core: out[(a,x), i, j, (b,y)] = lhs[a,i,j,b] rhs[x,i,j,y]."""
    ra, n, m, ra2 = lhs.shape
    rx, n_, m_, rx2 = rhs.shape
    if (n_, m_) != (n, m):
        raise ValueError("mode mismatch in element-wise product")
    if not (lhs.is_contiguous() and rhs.is_contiguous()):
        raise ValueError("element-wise product needs contiguous cores")
    out = empty(ra * rx, n, m, ra2 * rx2)
    d = _lib.Hadamard(ptr(lhs), ptr(rhs), ptr(out), ra, ra2, rx, rx2, n * m)
    arr = (_lib.Hadamard * 1)(d)
    check(lib().ttb_hadamard(arr, 1, stream()), "ttb_hadamard")
    return out


def kron(op: torch.Tensor, core: torch.Tensor) -> torch.Tensor:
    """TTM-by-TT core: out[(a,x), i, k, (b,y)] = sum_j op[a,i,j,b] core[x,j,k,y]."""
    ra, n, m, ra2 = op.shape
    rx, m_, kk, rx2 = core.shape
    if m_ != m:
        raise ValueError("mode mismatch in TTM product")
    out = empty(ra * rx, n, kk, ra2 * rx2)
    d = _lib.Kron(ptr(op), ptr(core), ptr(out), ra, ra2, n, m, rx, rx2, kk)
    arr = (_lib.Kron * 1)(d)
    check(lib().ttb_kron(arr, 1, stream()), "ttb_kron")
    return out


def norm_into(out: torch.Tensor, x: torch.Tensor, y: Optional[torch.Tensor] = None) -> torch.Tensor:
    """out[0] = ||x - y|| (or ||x||), computed on the device."""
    d = _lib.Norm(ptr(x), ptr(y), ptr(out), x.numel())
    arr = (_lib.Norm * 1)(d)
    check(lib().ttb_norm(arr, 1, stream()), "ttb_norm")
    return out


# ---------------------------------------------------------------------------
# factorisations
# ---------------------------------------------------------------------------


def qr(a: torch.Tensor, want_q=True, want_r=True, q_out=None, r_out=None):
    """Economic QR of a 2-D (strided) view: (Q (m, p), R (p, k))."""
    m, k = a.shape
    p = min(m, k)
    q = q_out if q_out is not None else (empty(m, p) if want_q else None)
    r = r_out if r_out is not None else (empty(p, k) if want_r else None)
    L = lib()
    ar = arena()
    with ar.scope():
        work = ar.take(L.ttb_qr_work_doubles(m, k))
        d = _lib.QR(ptr(a), a.stride(0), a.stride(1), ptr(q), q.stride(0) if q is not None else 0,
                    q.stride(1) if q is not None else 0, ptr(r),
                    r.stride(0) if r is not None else 0, r.stride(1) if r is not None else 0,
                    ptr(work), m, k)
        arr = (_lib.QR * 1)(d)
        check(L.ttb_qr(arr, 1, stream()), "ttb_qr")
    return q, r


def svd(a: torch.Tensor, status: Optional[torch.Tensor] = None):
    """Thin SVD of a 2-D (strided) view: (U (m, p), S (p,), Vh (p, k))."""
    m, k = a.shape
    p = min(m, k)
    u, s, vh = empty(m, p), empty(p), empty(p, k)
    L = lib()
    ar = arena()
    with ar.scope():
        work = ar.take(L.ttb_svd_work_doubles(m, k))
        d = _lib.SVD(ptr(a), a.stride(0), a.stride(1), ptr(u), u.stride(0), u.stride(1), ptr(s),
                     ptr(vh), vh.stride(0), vh.stride(1), ptr(work), ptr(status), m, k)
        arr = (_lib.SVD * 1)(d)
        check(L.ttb_svd(arr, 1, stream()), "ttb_svd")
    return u, s, vh


def lu_solve_(a_colmajor: torch.Tensor, b: torch.Tensor, info: Optional[torch.Tensor] = None):
    """Solve in place: ``a_colmajor`` is (n, n) whose row c is column c of the
    matrix (destroyed); b (n) becomes the solution."""
    n = b.numel()
    L = lib()
    ar = arena()
    with ar.scope():
        work = ar.take(L.ttb_lu_work_doubles(n)) if n > 1600 else None
        d = _lib.LU(ptr(a_colmajor), a_colmajor.stride(0), ptr(b), ptr(info), ptr(work), n)
        arr = (_lib.LU * 1)(d)
        check(L.ttb_lu_solve(arr, 1, stream()), "ttb_lu_solve")
    return b


# ---------------------------------------------------------------------------
# truncation ranks
# ---------------------------------------------------------------------------


def rank_residual(contrib, b, exact, s, limit, damp, tol, rank_out):
    n = b.numel()
    L = lib()
    ar = arena()
    with ar.scope():
        work = ar.take(L.ttb_rank_work_doubles(n, limit))
        d = _lib.Rank(ptr(contrib), ptr(b), ptr(exact), ptr(s), ptr(rank_out), ptr(work), n, limit,
                      s.numel(), float(damp), float(tol))
        arr = (_lib.Rank * 1)(d)
        check(L.ttb_rank_residual(arr, 1, stream()), "ttb_rank_residual")
    return rank_out


def rank_threshold(s, mode, value, max_rank, rank_out):
    d = _lib.RankRule(ptr(s), ptr(rank_out), s.numel(), int(mode),
                      int(max_rank) if max_rank else 0, float(value))
    arr = (_lib.RankRule * 1)(d)
    check(lib().ttb_rank_threshold(arr, 1, stream()), "ttb_rank_threshold")
    return rank_out


# ---------------------------------------------------------------------------
# Krylov solvers
# ---------------------------------------------------------------------------


def krylov(method: str, left, op, right, b, x, rtol, warm, maxiter=0, restart=20):
    """Run MINRES or GMRES on the one-site operator; returns (istop, iters)
    as a device int tensor of 2 entries."""
    opd = local_desc(left, op, right, x, b)
    res = torch.zeros(4, dtype=torch.int32, device="cuda")
    kd = _lib.Krylov(opd, ptr(b), ptr(x), None, res.data_ptr(), res.data_ptr() + 4, b.numel(),
                     float(rtol), int(maxiter), int(bool(warm)))
    L = lib()
    ar = arena()
    with ar.scope():
        if method == "minres":
            need = L.ttb_minres_work_doubles(C.byref(kd))
        else:
            need = L.ttb_gmres_work_doubles(C.byref(kd), restart)
        kd.work = ar.take(need).data_ptr()
        flags = ar.take_int(1)
        arr = (_lib.Krylov * 1)(kd)
        if method == "minres":
            check(L.ttb_minres(arr, 1, flags.data_ptr(), stream()), "ttb_minres")
        else:
            check(L.ttb_gmres(arr, 1, restart, flags.data_ptr(), stream()), "ttb_gmres")
    return res


def launch_count() -> int:
    return int(lib().ttb_launch_count())


# ---------------------------------------------------------------------------
# list forms: one grouped call for many independent problems
# ---------------------------------------------------------------------------


def qr_many(items) -> List:
    """items: (a, want_q, want_r, q_out, r_out); returns [(q, r)]."""
    if not items:
        return []
    L = lib()
    ar = arena()
    outs, descs = [], []
    with ar.scope():
        for a, want_q, want_r, q_out, r_out in items:
            m, k = a.shape
            p = min(m, k)
            q = q_out if q_out is not None else (empty(m, p) if want_q else None)
            r = r_out if r_out is not None else (empty(p, k) if want_r else None)
            work = ar.take(L.ttb_qr_work_doubles(m, k))
            descs.append(_lib.QR(ptr(a), a.stride(0), a.stride(1), ptr(q),
                                 q.stride(0) if q is not None else 0,
                                 q.stride(1) if q is not None else 0, ptr(r),
                                 r.stride(0) if r is not None else 0,
                                 r.stride(1) if r is not None else 0, ptr(work), m, k))
            outs.append((q, r))
        arr = (_lib.QR * len(descs))(*descs)
        check(L.ttb_qr(arr, len(descs), stream()), "ttb_qr")
    return outs


def svd_many(mats) -> List:
    if not mats:
        return []
    L = lib()
    ar = arena()
    outs, descs = [], []
    with ar.scope():
        for a in mats:
            m, k = a.shape
            p = min(m, k)
            u, s, vh = empty(m, p), empty(p), empty(p, k)
            work = ar.take(L.ttb_svd_work_doubles(m, k))
            descs.append(_lib.SVD(ptr(a), a.stride(0), a.stride(1), ptr(u), u.stride(0),
                                  u.stride(1), ptr(s), ptr(vh), vh.stride(0), vh.stride(1),
                                  ptr(work), None, m, k))
            outs.append((u, s, vh))
        arr = (_lib.SVD * len(descs))(*descs)
        check(L.ttb_svd(arr, len(descs), stream()), "ttb_svd")
    return outs


def direct_many(items, info: torch.Tensor) -> List:
    """items: (left, op, right, b_loc); explicit local matrices then GEPP
    solves, all grouped; ``info`` (int32, len(items)) receives the pivot
    status of each.  Returns the solutions (shaped like b_loc)."""
    if not items:
        return []
    L = lib()
    ar = arena()
    sols, lm, lu = [], [], []
    with ar.scope():
        for j, (left, op, right, b_loc) in enumerate(items):
            lt, R, lf = left.shape
            _, n, m, R2 = op.shape
            rt, _, rf = right.shape
            rows, cols = lf * n * rf, lt * m * rt
            M = ar.take(rows * cols)[: rows * cols].view(cols, rows)
            lm.append(_lib.LocalMatrix(ptr(left), ptr(op), ptr(right), ptr(M), lt, lf, R, R2, n,
                                       m, rt, rf))
            u = empty(*b_loc.shape)
            sols.append(u)
            work = ar.take(L.ttb_lu_work_doubles(rows)) if rows > 1600 else None
            lu.append(_lib.LU(ptr(M), rows, ptr(u), info.data_ptr() + 4 * j, ptr(work), rows))
        copy_many([copy_desc(b, u) for (_, _, _, b), u in zip(items, sols)])
        arr = (_lib.LocalMatrix * len(lm))(*lm)
        check(L.ttb_local_matrix(arr, len(lm), stream()), "ttb_local_matrix")
        arr = (_lib.LU * len(lu))(*lu)
        check(L.ttb_lu_solve(arr, len(lu), stream()), "ttb_lu_solve")
    return sols


def krylov_many(method: str, items, restart: int = 20) -> None:
    """items: (left, op, right, b, x, rtol, warm); x is updated in place."""
    if not items:
        return
    L = lib()
    ar = arena()
    with ar.scope():
        descs = []
        for left, op, right, b, x, rtol, warm in items:
            opd = local_desc(left, op, right, x, b)
            kd = _lib.Krylov(opd, ptr(b), ptr(x), None, None, None, b.numel(), float(rtol), 0,
                             int(bool(warm)))
            need = (L.ttb_minres_work_doubles(C.byref(kd)) if method == "minres"
                    else L.ttb_gmres_work_doubles(C.byref(kd), restart))
            kd.work = ar.take(need).data_ptr()
            descs.append(kd)
        flags = ar.take_int(len(descs))
        arr = (_lib.Krylov * len(descs))(*descs)
        if method == "minres":
            check(L.ttb_minres(arr, len(descs), flags.data_ptr(), stream()), "ttb_minres")
        else:
            check(L.ttb_gmres(arr, len(descs), restart, flags.data_ptr(), stream()), "ttb_gmres")


def norm_many(items) -> None:
    """items: (out, x, y or None)."""
    if not items:
        return
    descs = [_lib.Norm(ptr(x), ptr(y), ptr(out), x.numel()) for out, x, y in items]
    arr = (_lib.Norm * len(descs))(*descs)
    check(lib().ttb_norm(arr, len(descs), stream()), "ttb_norm")


def rank_residual_many(items) -> None:
    """items: (contrib, b, exact, s, limit, damp, tol, rank_out)."""
    if not items:
        return
    L = lib()
    ar = arena()
    with ar.scope():
        descs = []
        for contrib, b, exact, s, limit, damp, tol, rank_out in items:
            n = b.numel()
            work = ar.take(L.ttb_rank_work_doubles(n, limit))
            descs.append(_lib.Rank(ptr(contrib), ptr(b), ptr(exact), ptr(s), ptr(rank_out),
                                   ptr(work), n, limit, s.numel(), float(damp), float(tol)))
        arr = (_lib.Rank * len(descs))(*descs)
        check(L.ttb_rank_residual(arr, len(descs), stream()), "ttb_rank_residual")


def rank_threshold_many(items) -> None:
    """items: (s, mode, value, max_rank, rank_out)."""
    if not items:
        return
    descs = [_lib.RankRule(ptr(s), ptr(out), s.numel(), int(mode), int(mr) if mr else 0,
                           float(v)) for s, mode, v, mr, out in items]
    arr = (_lib.RankRule * len(descs))(*descs)
    check(lib().ttb_rank_threshold(arr, len(descs), stream()), "ttb_rank_threshold")


def kron_many(items) -> List:
    """items: (op, core); returns the Kronecker cores."""
    if not items:
        return []
    outs, descs = [], []
    for op, core in items:
        ra, n, m, ra2 = op.shape
        rx, m_, kk, rx2 = core.shape
        out = empty(ra * rx, n, kk, ra2 * rx2)
        outs.append(out)
        descs.append(_lib.Kron(ptr(op), ptr(core), ptr(out), ra, ra2, n, m, rx, rx2, kk))
    arr = (_lib.Kron * len(descs))(*descs)
    check(lib().ttb_kron(arr, len(descs), stream()), "ttb_kron")
    return outs
