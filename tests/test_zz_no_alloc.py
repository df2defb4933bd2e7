"""ttb_qr_static, the QR entry point that takes its work areas from a fixed
array inside the library, against ttb_qr with caller-provided work areas.

Called through the C ABI with ctypes.  The problems mix shapes that fit in
shared memory with tall and wide ones that use the blocked factorisation
(and so the fixed array); two calls in a row must both agree with ttb_qr.
This file sorts last so that it also runs after every other GPU test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SHAPES = [(50, 10), (1000, 40), (40, 1000), (700, 64), (3000, 24)]
TOL = 1e-12


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ttnumpy_b200 import _lib

    return _lib


def _desc(L, a, q, r, work):
    m, k = a.shape
    return L.QR(a.data_ptr(), a.stride(0), a.stride(1), q.data_ptr(), q.stride(0), q.stride(1),
                r.data_ptr(), r.stride(0), r.stride(1), work.data_ptr() if work is not None else 0,
                m, k)


def _outputs(shapes):
    dev = torch.device("cuda:0")
    return [(torch.empty(m, min(m, k), dtype=torch.float64, device=dev),
             torch.empty(min(m, k), k, dtype=torch.float64, device=dev)) for m, k in shapes]


def _run(lib, fn, mats, outs, with_work):
    L = lib
    h = L.load()
    works = []
    descs = []
    for a, (q, r) in zip(mats, outs):
        w = None
        if with_work:
            w = torch.empty(h.ttb_qr_work_doubles(*a.shape), dtype=torch.float64, device=a.device)
            works.append(w)
        descs.append(_desc(L, a, q, r, w))
    arr = (L.QR * len(descs))(*descs)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    code = getattr(h, fn)(arr, len(descs), stream)
    torch.cuda.synchronize()
    return code


def test_static_matches_work_entry_point(lib):
    g = torch.Generator(device="cpu").manual_seed(7)
    mats = [torch.randn(m, k, generator=g, dtype=torch.float64).cuda() for m, k in SHAPES]
    ref = _outputs(SHAPES)
    assert _run(lib, "ttb_qr", mats, ref, True) == 0
    for call in range(2):
        got = _outputs(SHAPES)
        assert _run(lib, "ttb_qr_static", mats, got, False) == 0, call
        for (m, k), a, (q0, r0), (q1, r1) in zip(SHAPES, mats, ref, got):
            scale_q = q0.abs().max().item()
            scale_r = r0.abs().max().item()
            assert (q1 - q0).abs().max().item() <= TOL * scale_q, (call, m, k)
            assert (r1 - r0).abs().max().item() <= TOL * scale_r, (call, m, k)
            # and it is a QR factorisation of a
            err = (q1 @ r1 - a).abs().max().item() / a.abs().max().item()
            assert err < 1e-12, (call, m, k, err)


def test_static_rejects_oversize_call(lib):
    dev = torch.device("cuda:0")
    h = lib.load()
    # one blocked problem needing more than the fixed array
    m, k = 4096, 600
    assert m * k + k > 2097152
    a = torch.zeros(m, k, dtype=torch.float64, device=dev)
    q = torch.empty(m, k, dtype=torch.float64, device=dev)
    r = torch.empty(k, k, dtype=torch.float64, device=dev)
    arr = (lib.QR * 1)(_desc(lib, a, q, r, None))
    before = h.ttb_launch_count()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert h.ttb_qr_static(arr, 1, stream) == -2
    assert h.ttb_launch_count() == before
    # and the array is still usable afterwards
    small = [torch.randn(900, 30, dtype=torch.float64, device=dev)]
    out = _outputs([(900, 30)])
    assert _run(lib, "ttb_qr_static", small, out, False) == 0
    qq, rr = out[0]
    assert (qq @ rr - small[0]).abs().max().item() < 1e-12 * small[0].abs().max().item() * 10
