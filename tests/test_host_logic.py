"""Host-side logic of the persistent engine, run without a GPU: request
validation, the launch order, and the library's host-only sizing functions
(the work-area bounds the kernels are launched with)."""

import ctypes as C

import numpy as np
import pytest

from ttnumpy_b200 import _lib
from ttnumpy_b200 import persistent as pers
from ttnumpy_b200 import problems as P
from ttnumpy_b200 import tensor_train

KW = dict(residual_tol=1e-8, symmetric=True, max_sweeps=10)


@pytest.fixture(scope="module")
def lib():
    return _lib.load()


def _prep(prob, **kw):
    return pers.prepare([(prob.A, prob.b, None, dict(KW, **kw))])[0]


def test_prepare_validates_like_amen():
    p = P.parametric_diffusion(4, 16, np.zeros(4))
    with pytest.raises(ValueError):
        _prep(p, kickrank=0)
    with pytest.raises(ValueError):
        _prep(p, max_rank=0)
    with pytest.raises(ValueError):
        _prep(p, residual_damp=0.5)
    with pytest.raises(ValueError):
        _prep(p, residual_tol=-1.0)
    with pytest.raises(TypeError):
        _prep(p, not_an_argument=1)
    q = P.parametric_diffusion(4, 8, np.zeros(4))
    with pytest.raises(tensor_train.DimensionMismatch):
        pers.prepare([(p.A, q.b, None, KW)])


def test_launch_order_longest_first():
    """Blocks start in order of estimated cost: the larger mode and operator
    bond, and the longer train, go first."""
    small = _prep(P.qtt_poisson_2d(4))
    mid = _prep(P.parametric_diffusion(4, 16, np.zeros(4)))
    big = _prep(P.parametric_diffusion(5, 32, np.zeros(5)))
    costs = [pers._cost(x) for x in (small, mid, big)]
    assert costs[0] < costs[1] < costs[2]


def test_slab_bound_grows_with_capacity_and_rejects_long_trains(lib):
    p = _prep(P.parametric_diffusion(5, 32, np.zeros(5)))
    sizes = [pers.slab_doubles(p, r) for r in (16, 32, 64, 128)]
    assert all(a < b for a, b in zip(sizes, sizes[1:]))
    assert all(s % 64 == 0 for s in sizes)
    # the solution-core slots alone: d cores of rmax x n x rmax
    assert sizes[2] >= 5 * 64 * 32 * 64
    dims = (C.c_int * 3)(2, 2, 2)
    assert lib.ttb_amen_slab_doubles(1, dims, 4, 16, 1000) == -1
    long_dims = (C.c_int * (5 * 65 + 2))(*([2] * (5 * 65 + 2)))
    assert lib.ttb_amen_slab_doubles(65, long_dims, 4, 16, 1000) == -1


def test_work_area_bounds(lib):
    """The factorisation work areas are non-negative and monotone in the
    problem size (the host sizes every arena from them)."""
    qr = [lib.ttb_qr_work_doubles(m, 40) for m in (40, 400, 4000)]
    svd = [lib.ttb_svd_work_doubles(m, 40) for m in (40, 400, 4000)]
    assert all(v >= 0 for v in qr + svd)
    assert qr == sorted(qr) and svd == sorted(svd)
    assert lib.ttb_lu_work_doubles(2000) >= 2000


def test_serving_mix_generator():
    """The serving stream's requests: one seeded generator, the same
    requests for the same seed, about 10 % large, the rest split between
    diffusion and QTT Poisson, with the stated dimension and mode ranges."""
    from ttnumpy_b200 import problems as P

    a = P.serving_requests(400, 3)
    b = P.serving_requests(400, 3)
    assert [p.name for p in a] == [p.name for p in b]
    assert all(np.array_equal(x, y) for p, q in zip(a, b) for x, y in zip(p.A, q.A))
    kinds = [p.meta["kind"] for p in a]
    assert 20 <= kinds.count("large") <= 60
    assert 140 <= kinds.count("diffusion") <= 220 and 140 <= kinds.count("qtt") <= 220
    for p in a:
        if p.meta["kind"] == "diffusion":
            assert 4 <= len(p.A) <= 12 and p.A[0].shape[1] in (16, 32, 64)
        elif p.meta["kind"] == "qtt":
            assert len(p.A) % 2 == 0 and 6 <= len(p.A) <= 20
        else:
            assert len(p.A) == 24 and p.A[0].shape[1] == 64 and max(c.shape[0] for c in p.b) == 8
    arrivals = [t for t, _ in P.serving_stream(50, rate=10.0, seed=3)]
    assert all(t1 > t0 for t0, t1 in zip(arrivals, arrivals[1:]))


def test_split_index_division_formula():
    """The multiply-shift division the kernels use for split-index outputs
    (FastDiv in csrc/ttb_device.cuh: m = floor(2^32 (2^l - d) / d) + 1 with
    l = ceil(log2 d), n / d = (mulhi(m, n) + n) >> l for 0 <= n < 2^31),
    restated here and checked against integer division."""
    rng = np.random.default_rng(3)
    divisors = list(range(1, 600)) + [int(v) for v in rng.integers(600, 1 << 30, 400)]
    for d in divisors:
        l = (d - 1).bit_length()
        m = ((1 << 32) * ((1 << l) - d)) // d + 1
        assert 0 < m < (1 << 32)
        ns = [0, 1, d - 1, d, d + 1, 3 * d - 1, (1 << 31) - 1]
        ns += [int(v) for v in rng.integers(0, 1 << 31, 50)]
        for n in ns:
            if n < 0 or n >= (1 << 31):
                continue
            t = ((m * n) >> 32) + n
            assert t < (1 << 32)
            assert t >> l == n // d, (n, d)
