"""Mixed-precision GEMM on the tcgen05 tensor cores (3xTF32, FP32
accumulation) against the float64 GEMM of the same problems.

The split of each float64 operand into two TF32 parts keeps about 22
significant bits, and the products accumulate in FP32, so the error bound
used here is 1e-5 of |A| |B| (entry-wise, with |A| |B| the product of the
absolute values), well above the ~1e-6 observed and far below the O(1)
error of a wrong layout or descriptor.
"""

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SHAPES = [(1, 1, 1), (128, 64, 32), (57, 228, 1824), (1824, 57, 228), (130, 70, 33),
          (300, 129, 1000), (7, 300, 5), (64, 64, 0)]
TOL = 1e-5


@pytest.fixture(scope="module")
def K():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ttnumpy_b200 import kernels

    return kernels


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_3xtf32_matches_fp64(K, m, n, k):
    g = torch.Generator(device="cpu").manual_seed(m * 1000 + n + k)
    a = torch.randn(m, k, generator=g, dtype=torch.float64).cuda()
    b = torch.randn(k, n, generator=g, dtype=torch.float64).cuda()
    c0 = torch.randn(m, n, generator=g, dtype=torch.float64).cuda()
    ref, got = c0.clone(), c0.clone()
    K.gemm_many([K.gemm_desc(a, b, ref, 0.75, -0.5)])
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    K.gemm_3xtf32_many([K.gemm_desc(a, b, got, 0.75, -0.5)], status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    bound = 0.75 * (a.abs() @ b.abs()) if k > 0 else torch.zeros_like(ref)
    err = (got - ref).abs()
    assert bool((err <= TOL * bound + 1e-12 * ref.abs()).all()), float((err / (bound + 1e-300)).max())


def test_3xtf32_strided_and_batched(K):
    g = torch.Generator(device="cpu").manual_seed(5)
    a = torch.randn(3, 200, 90, generator=g, dtype=torch.float64).cuda().transpose(1, 2)  # 3 x 90 x 200
    b = torch.randn(200, 150, generator=g, dtype=torch.float64).cuda()
    ref = torch.zeros(3, 90, 150, dtype=torch.float64, device="cuda")
    got = torch.zeros_like(ref)
    K.gemm_many([K.gemm_desc(a, b, ref)])
    K.gemm_3xtf32_many([K.gemm_desc(a, b, got)])
    torch.cuda.synchronize()
    bound = a.abs() @ b.abs()
    assert bool(((got - ref).abs() <= TOL * bound).all())
