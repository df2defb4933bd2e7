"""libttb200 kernels against NumPy/SciPy and the oracle, float64.

Tolerances: dense products and factorisations are compared at 1e-12
relative (rounding of float64 GEMMs of the sizes used); Krylov solves at the
solver tolerance.
"""

import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse.linalg as spla

from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def K():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ttnumpy_b200 import kernels

    kernels.lib()
    return kernels


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (64, 64, 64), (130, 67, 200),
                                   (1536, 96, 48), (48, 1536, 96), (5, 300, 1)])
def test_gemm_shapes(K, m, n, k):
    rng = np.random.default_rng(m * 1000 + n * 10 + k)
    a, b, c = rng.standard_normal((m, k)), rng.standard_normal((k, n)), rng.standard_normal((m, n))
    C = dev(c)
    K.gemm(dev(a), dev(b), C, alpha=0.5, beta=2.0)
    assert rel(host(C), 0.5 * a @ b + 2.0 * c) < 1e-13


def test_gemm_transposed_and_batched(K):
    rng = np.random.default_rng(1)
    a = rng.standard_normal((9, 40, 33))
    b = rng.standard_normal((33, 21))
    A = dev(a)
    C = torch.empty(9, 21, 40, dtype=torch.float64, device="cuda")
    # C[i]^T = A[i] @ b written through a transposed view
    K.gemm(A, dev(b).expand(9, 33, 21) if False else dev(b).unsqueeze(0), C.transpose(1, 2))
    want = np.einsum("bij,jk->bki", a, b)
    assert rel(host(C), want) < 1e-13
    # transposed A operand
    at = rng.standard_normal((50, 70))
    out = torch.empty(70, 30, dtype=torch.float64, device="cuda")
    bb = rng.standard_normal((50, 30))
    K.gemm(dev(at).t(), dev(bb), out)
    assert rel(host(out), at.T @ bb) < 1e-13


def test_copy_fill_scale(K):
    rng = np.random.default_rng(2)
    src = rng.standard_normal((3, 4, 5, 6))
    dst = torch.zeros(3, 4, 5, 10, dtype=torch.float64, device="cuda")
    K.copy_(dst[..., 2:8], dev(src), alpha=-2.0)
    want = np.zeros((3, 4, 5, 10))
    want[..., 2:8] = -2.0 * src
    assert np.array_equal(host(dst), want)
    s = rng.standard_normal(6)
    K.copy_(dst[..., :6], dev(src), scale=dev(s), scale_axis=3)
    want[..., :6] = src * s
    assert np.allclose(host(dst), want, rtol=0, atol=0)
    K.fill_(dst, 1.5)
    assert np.all(host(dst) == 1.5)


def _train(rng, modes, ranks, cols=None):
    cores = []
    for i, n in enumerate(modes):
        m = 1 if cols is None else cols[i]
        cores.append(rng.standard_normal((ranks[i], n, m, ranks[i + 1])))
    return cores


@pytest.mark.parametrize("with_op", [True, False])
@pytest.mark.parametrize("side", [0, 1])
def test_env_update_matches_oracle(K, side, with_op):
    rng = np.random.default_rng(3 + side + 2 * with_op)
    modes = [5, 6, 4]
    x = O.Train(_train(rng, modes, [1, 7, 9, 1]))
    y = O.Train(_train(rng, modes, [1, 3, 8, 1]))
    A = O.Train(_train(rng, modes, [1, 2, 3, 1], cols=modes)) if with_op else None
    env = [None] * 3
    if side == 0:
        O.env_left(env, 0, x, y, A)
        O.env_left(env, 1, x, y, A)
        O.env_left(env, 2, x, y, A)
        k, prev, src = 2, env[1], 1
    else:
        O.env_right(env, 2, x, y, A)
        O.env_right(env, 1, x, y, A)
        O.env_right(env, 0, x, y, A)
        k, prev, src = 0, env[1], 1
    fc = dev(x.cores[src][:, :, 0, :])
    tc = dev(y.cores[src][:, :, 0, :])
    opc = dev(A.cores[src]) if with_op else None
    out = torch.empty(env[k].shape, dtype=torch.float64, device="cuda")
    K.env_update([K.env_desc(side, dev(prev), fc, tc, out, opc)])
    assert rel(host(out), env[k]) < 1e-13


@pytest.mark.parametrize("rect", [False, True])
def test_local_apply_matches_oracle(K, rect):
    rng = np.random.default_rng(5)
    lt, R, lf, n, R2, rt, rf = 6, 3, (4 if rect else 6), 7, 2, 5, (3 if rect else 5)
    left = rng.standard_normal((lt, R, lf))
    op = rng.standard_normal((R, n, n, R2))
    right = rng.standard_normal((rt, R2, rf))
    cols = 4
    xs = rng.standard_normal((cols, lt, n, rt))
    y = torch.zeros(cols, lf, n, rf, dtype=torch.float64, device="cuda")
    K.local_apply([K.local_desc(dev(left), dev(op), dev(right), dev(xs), y, cols, 1.0, 0.0)])
    want = np.einsum("iaj,aklb,pbq,cilp->cjkq", left, op, right, xs)
    assert rel(host(y), want) < 1e-13
    if not rect:
        M = O.local_matrix(left, op, right)
        got = host(K.local_matrix(dev(left), dev(op), dev(right))).T
        assert rel(got, M) < 1e-13
        assert rel(M @ xs.reshape(cols, -1).T, want.reshape(cols, -1).T) < 1e-12


def test_project_matches_oracle(K):
    rng = np.random.default_rng(6)
    Lb, core, Rb = rng.standard_normal((3, 5)), rng.standard_normal((3, 4, 2)), rng.standard_normal((2, 6))
    out = torch.empty(5, 4, 6, dtype=torch.float64, device="cuda")
    K.project([K.project_desc(dev(Lb), dev(core), dev(Rb), out)])
    want = O.local_rhs(Lb, core.reshape(3, 4, 1, 2), Rb).reshape(5, 4, 6)
    assert rel(host(out), want) < 1e-13


def test_kron_and_norm(K):
    rng = np.random.default_rng(7)
    op = rng.standard_normal((2, 3, 4, 3))
    core = rng.standard_normal((5, 4, 1, 2))
    got = host(K.kron(dev(op), dev(core)))
    want = O.dot(O.Train([op]), O.Train([core])).cores[0]
    assert rel(got, want) < 1e-14
    v = rng.standard_normal(100001)
    w = rng.standard_normal(100001)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    K.norm_into(out, dev(v), dev(w))
    assert abs(out.item() - np.linalg.norm(v - w)) < 1e-12 * np.linalg.norm(v - w)


@pytest.mark.parametrize("m,k", [(1, 1), (5, 3), (3, 5), (64, 64), (256, 64), (1536, 48),
                                 (3000, 70), (70, 3000), (12, 1), (4640, 145), (1280, 44),
                                 (700, 700), (1000, 17), (300, 2000)])
def test_qr(K, m, k):
    rng = np.random.default_rng(m + 7 * k)
    a = rng.standard_normal((m, k))
    q, r = K.qr(dev(a))
    q, r = host(q), host(r)
    p = min(m, k)
    assert q.shape == (m, p) and r.shape == (p, k)
    assert rel(q @ r, a) < 1e-13
    assert np.abs(q.T @ q - np.eye(p)).max() < 1e-13
    assert np.allclose(np.tril(r, -1), 0)
    # LAPACK sign convention: the same R as scipy's geqrf
    _, r_ref = sla.qr(a, mode="economic")
    assert rel(r, r_ref) < 1e-11


def test_qr_rank_deficient(K):
    rng = np.random.default_rng(9)
    a = rng.standard_normal((40, 3)) @ rng.standard_normal((3, 10))
    q, r = K.qr(dev(a))
    assert rel(host(q) @ host(r), a) < 1e-13
    assert np.abs(host(q).T @ host(q) - np.eye(10)).max() < 1e-12


@pytest.mark.parametrize("m,k", [(1, 1), (6, 4), (4, 6), (64, 64), (256, 64), (64, 256),
                                 (1536, 48), (48, 1536), (300, 120), (7, 1), (1, 9),
                                 (3000, 90), (90, 3000), (2000, 33)])
def test_svd(K, m, k):
    rng = np.random.default_rng(11 * m + k)
    a = rng.standard_normal((m, k))
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    u, s, vh = K.svd(dev(a), status)
    u, s, vh = host(u), host(s), host(vh)
    p = min(m, k)
    s_ref = sla.svdvals(a)
    assert np.all(np.diff(s) <= 0)
    assert np.abs(s - s_ref).max() <= 1e-13 * s_ref[0]
    assert rel((u * s) @ vh, a) < 1e-13
    assert np.abs(u.T @ u - np.eye(p)).max() < 1e-12
    assert np.abs(vh @ vh.T - np.eye(p)).max() < 1e-12
    assert status.item() >= 0


def test_svd_graded(K):
    """Singular values spread over 14 decades keep relative accuracy."""
    rng = np.random.default_rng(12)
    u0, _ = np.linalg.qr(rng.standard_normal((80, 30)))
    v0, _ = np.linalg.qr(rng.standard_normal((30, 30)))
    s0 = np.logspace(0, -14, 30)
    a = (u0 * s0) @ v0.T
    _, s, _ = K.svd(dev(a))
    assert np.abs(host(s) - s0).max() < 1e-15 * 30


@pytest.mark.parametrize("n", [1, 7, 100, 161, 162, 400, 777, 1000, 1700])
def test_lu_solve(K, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + n * 0.1 * np.eye(n)
    b = rng.standard_normal(n)
    A = dev(a.T)  # row c of A is column c of the matrix
    x = dev(b)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    K.lu_solve_(A, x, info)
    assert info.item() == 0
    assert rel(host(x), np.linalg.solve(a, b)) < 1e-11


def test_lu_singular_reports_info(K):
    a = np.array([[1.0, 2.0], [2.0, 4.0]])
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    K.lu_solve_(dev(a.T), dev(np.ones(2)), info)
    assert info.item() == 2


def test_rank_rules(K):
    rng = np.random.default_rng(13)
    s = np.sort(np.abs(rng.standard_normal(40)) * np.logspace(0, -12, 40))[::-1].copy()
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    for delta in (0.0, 1e-10, 1e-6, 1e-2, 10.0):
        for mr in (None, 5):
            K.rank_threshold(dev(s), 1, delta, mr, out)
            assert out.item() == O.truncated_bond(s, delta, mr)
    for eth in (1e-14, 1e-7, 1e-3, 0.5):
        for mr in (None, 3):
            K.rank_threshold(dev(s), 0, eth, mr, out)
            assert out.item() == O.rank_by_threshold(s, eth, mr)


def test_rank_residual_matches_oracle(K):
    rng = np.random.default_rng(14)
    rl, n, rr, R = 5, 6, 7, 2
    left = rng.standard_normal((rl, R, rl))
    left = left + left.transpose(2, 1, 0)
    op = rng.standard_normal((R, n, n, R))
    op = op + op.transpose(0, 2, 1, 3)
    right = rng.standard_normal((rr, R, rr))
    right = right + right.transpose(2, 1, 0)
    A_loc = O.local_matrix(left, op, right) + 50 * np.eye(rl * n * rr)
    b = rng.standard_normal(rl * n * rr)
    u = np.linalg.solve(A_loc, b) + 1e-6 * rng.standard_normal(b.size)
    U, S, Vh = sla.svd(u.reshape(rl * n, rr), full_matrices=False)
    exact = np.linalg.norm(A_loc @ u - b)
    for tol in (1e-2, 1e-4, 1e-6):
        want = O.rank_by_residual(A_loc, b, U, S, Vh, exact, tol, 2.0, None)
        terms = np.einsum("ik,kj->kij", U * S, Vh).reshape(len(S), -1)
        contrib = (A_loc @ terms.T).T
        out = torch.zeros(1, dtype=torch.int32, device="cuda")
        K.rank_residual(dev(contrib), dev(b), dev(np.array([exact])), dev(S), len(S), 2.0, tol, out)
        assert out.item() == want


def _spd_local(rng, rl, n, rr, R):
    left = rng.standard_normal((rl, R, rl))
    left = left + left.transpose(2, 1, 0)
    op = rng.standard_normal((R, n, n, R)) * 0.2
    op = op + op.transpose(0, 2, 1, 3)
    op[0, :, :, 0] += 3 * np.eye(n) * (n + R)
    right = rng.standard_normal((rr, R, rr))
    right = right + right.transpose(2, 1, 0)
    right[:, 0, :] += 3 * np.eye(rr) * (rr + R)
    left[:, 0, :] += 3 * np.eye(rl) * (rl + R)
    return left, op, right


@pytest.mark.parametrize("method", ["minres", "gmres"])
@pytest.mark.parametrize("warm", [False, True])
def test_krylov_matches_scipy(K, method, warm):
    rng = np.random.default_rng(15 + warm)
    rl, n, rr, R = 6, 9, 5, 2
    left, op, right = _spd_local(rng, rl, n, rr, R)
    A_loc = O.local_matrix(left, op, right)
    assert np.allclose(A_loc, A_loc.T)
    b = rng.standard_normal(rl * n * rr)
    x0 = rng.standard_normal(b.size) if warm else None
    for rtol in (1e-6, 1e-10):
        if method == "minres":
            ref, _ = spla.minres(A_loc, b, x0=x0, rtol=rtol)
        else:
            ref, _ = spla.gmres(A_loc, b, x0=x0, rtol=rtol, atol=0.0)
        x = dev(x0 if warm else np.zeros(b.size))
        res = K.krylov(method, dev(left), dev(op), dev(right), dev(b), x, rtol, warm)
        got = host(x)
        r_got = np.linalg.norm(A_loc @ got - b)
        r_ref = np.linalg.norm(A_loc @ ref - b)
        # same algorithm and stopping rule: residuals of the same size
        assert r_got <= 10 * max(r_ref, 1e-14 * np.linalg.norm(b)), (r_got, r_ref)
        assert rel(got, ref) < 1e3 * rtol + 1e-12


def test_minres_large_system(K):
    """A local system of the size of the 8-D Laplacian solve (N ~ 40k)."""
    rng = np.random.default_rng(16)
    rl, n, rr, R = 32, 32, 40, 2
    left, op, right = _spd_local(rng, rl, n, rr, R)
    b = rng.standard_normal(rl * n * rr)
    x = torch.zeros(b.size, dtype=torch.float64, device="cuda")
    K.krylov("minres", dev(left), dev(op), dev(right), dev(b), x, 1e-10, False)
    y = torch.empty_like(x)
    K.local_apply([K.local_desc(dev(left), dev(op), dev(right), x, y)])
    r = np.linalg.norm(host(y) - b) / np.linalg.norm(b)
    assert r < 1e-8
