"""ctypes binding of libttb200 (the C ABI declared in ``include/ttb200.h``).

The shared library is built in-tree by :func:`ttnumpy_b200.build.build` and
loaded on first use.  There is no fallback: without the library or without
a CUDA device every entry point of the package raises.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libttb200.so")

P = C.c_void_p
I = C.c_int
L = C.c_longlong
D = C.c_double


class Gemm(C.Structure):
    _fields_ = [("a", P), ("b", P), ("c", P), ("m", I), ("n", I), ("k", I), ("batch", I),
                ("a_rs", L), ("a_cs", L), ("a_bs", L), ("b_rs", L), ("b_cs", L), ("b_bs", L),
                ("c_rs", L), ("c_cs", L), ("c_bs", L), ("alpha", D), ("beta", D)]


class Env(C.Structure):
    _fields_ = [("env", P), ("frame", P), ("op", P), ("target", P), ("out", P), ("work", P),
                ("side", I), ("f", I), ("f2", I), ("t", I), ("t2", I), ("R", I), ("R2", I),
                ("n", I), ("m", I)]


class Local(C.Structure):
    _fields_ = [("left", P), ("op", P), ("right", P), ("x", P), ("y", P), ("work", P),
                ("lt", I), ("lf", I), ("R", I), ("R2", I), ("n", I), ("m", I), ("rt", I),
                ("rf", I), ("cols", I), ("alpha", D), ("beta", D)]


class LocalMatrix(C.Structure):
    _fields_ = [("left", P), ("op", P), ("right", P), ("out", P), ("lt", I), ("lf", I),
                ("R", I), ("R2", I), ("n", I), ("m", I), ("rt", I), ("rf", I)]


class Project(C.Structure):
    _fields_ = [("left", P), ("core", P), ("right", P), ("out", P), ("work", P), ("a", I),
                ("i", I), ("n", I), ("c", I), ("l", I), ("alpha", D), ("beta", D)]


class QR(C.Structure):
    _fields_ = [("a", P), ("a_rs", L), ("a_cs", L), ("q", P), ("q_rs", L), ("q_cs", L),
                ("r", P), ("r_rs", L), ("r_cs", L), ("work", P), ("m", I), ("k", I)]


class SVD(C.Structure):
    _fields_ = [("a", P), ("a_rs", L), ("a_cs", L), ("u", P), ("u_rs", L), ("u_cs", L),
                ("s", P), ("vh", P), ("vh_rs", L), ("vh_cs", L), ("work", P), ("status", P),
                ("m", I), ("k", I)]


class LU(C.Structure):
    _fields_ = [("a", P), ("lda", L), ("b", P), ("info", P), ("work", P), ("n", I)]


class Copy(C.Structure):
    _fields_ = [("src", P), ("dst", P), ("scale", P), ("d0", I), ("d1", I), ("d2", I),
                ("d3", I), ("s0", L), ("s1", L), ("s2", L), ("s3", L), ("t0", L), ("t1", L),
                ("t2", L), ("t3", L), ("alpha", D), ("scale_axis", I)]


class Kron(C.Structure):
    _fields_ = [("op", P), ("core", P), ("out", P), ("ra", I), ("ra2", I), ("n", I), ("m", I),
                ("rx", I), ("rx2", I), ("kk", I)]


class Hadamard(C.Structure):
    _fields_ = [("lhs", P), ("rhs", P), ("out", P), ("ra", I), ("ra2", I), ("rx", I), ("rx2", I),
                ("modes", I)]


class Norm(C.Structure):
    _fields_ = [("x", P), ("y", P), ("out", P), ("n", L)]


class Rank(C.Structure):
    _fields_ = [("contrib", P), ("b", P), ("exact", P), ("s", P), ("rank", P), ("work", P),
                ("n", L), ("limit", I), ("p", I), ("damp", D), ("tol", D)]


class RankRule(C.Structure):
    _fields_ = [("s", P), ("rank", P), ("p", I), ("mode", I), ("max_rank", I), ("value", D)]


class Krylov(C.Structure):
    _fields_ = [("op", Local), ("b", P), ("x", P), ("work", P), ("istop", P), ("iters", P),
                ("n", L), ("rtol", D), ("maxiter", I), ("warm", I)]


class Round(C.Structure):
    _fields_ = [("p", P), ("q", P), ("p_off", P), ("q_off", P), ("p_bonds", P),
                ("q_bonds", P), ("modes", P), ("p_stride", L), ("q_stride", L), ("out", P),
                ("out_stride", L), ("out_off", P), ("bonds", P), ("work", P),
                ("work_stride", L), ("status", P), ("pairs", I), ("d", I), ("error", D),
                ("max_rank", I)]


class AmenTask(C.Structure):
    _fields_ = [("A", P), ("A_off", P), ("b", P), ("b_off", P), ("x0", P), ("x0_off", P),
                ("z0", P), ("z0_off", P), ("dims", P), ("slab", P), ("slab_doubles", L),
                ("residuals", P), ("result", P), ("x_offsets", P),
                ("d", I), ("kickrank", I), ("max_rank", I), ("max_sweeps", I),
                ("direct_solve_size", I), ("track_residual", I), ("residual_mode", I),
                ("stagnation_on", I), ("x0_orth_center", I), ("b_orth_center", I),
                ("residual_tol", D), ("error_threshold", D), ("residual_damp", D),
                ("stagnation_factor", D), ("local_rtol", D), ("truncation_tol", D),
                ("debug", I), ("time_limit_ns", L), ("precision", I),
                ("local_gmres", I)]


_SIGNATURES = {
    "ttb_version": ([], I),
    "ttb_launch_count": ([], L),
    "ttb_profile_enable": ([I], None),
    "ttb_profile_read": ([I, C.POINTER(D), C.POINTER(L), C.POINTER(D), C.POINTER(D)], I),
    "ttb_profile_reset": ([], None),
    "ttb_fma_peak": ([P, I, I, P], I),
    "ttb_gemm": ([C.POINTER(Gemm), I, P], I),
    "ttb_env_work_doubles": ([C.POINTER(Env)], L),
    "ttb_env_update": ([C.POINTER(Env), I, P], I),
    "ttb_local_work_doubles": ([C.POINTER(Local)], L),
    "ttb_local_apply": ([C.POINTER(Local), I, P], I),
    "ttb_local_matrix": ([C.POINTER(LocalMatrix), I, P], I),
    "ttb_project": ([C.POINTER(Project), I, P], I),
    "ttb_gemm_3xtf32": ([C.POINTER(Gemm), I, P, P], I),
    "ttb_qr_work_doubles": ([I, I], L),
    "ttb_qr": ([C.POINTER(QR), I, P], I),
    "ttb_qr_static": ([C.POINTER(QR), I, P], I),
    "ttb_svd_work_doubles": ([I, I], L),
    "ttb_svd": ([C.POINTER(SVD), I, P], I),
    "ttb_lu_work_doubles": ([I], L),
    "ttb_lu_solve": ([C.POINTER(LU), I, P], I),
    "ttb_copy": ([C.POINTER(Copy), I, P], I),
    "ttb_kron": ([C.POINTER(Kron), I, P], I),
    "ttb_hadamard": ([C.POINTER(Hadamard), I, P], I),
    "ttb_norm": ([C.POINTER(Norm), I, P], I),
    "ttb_rank_work_doubles": ([L, I], L),
    "ttb_rank_residual": ([C.POINTER(Rank), I, P], I),
    "ttb_rank_threshold": ([C.POINTER(RankRule), I, P], I),
    "ttb_minres_work_doubles": ([C.POINTER(Krylov)], L),
    "ttb_minres": ([C.POINTER(Krylov), I, P, P], I),
    "ttb_gmres_work_doubles": ([C.POINTER(Krylov), I], L),
    "ttb_gmres": ([C.POINTER(Krylov), I, I, P, P], I),
    "ttb_round_work_doubles": ([I, I, I], L),
    "ttb_round_batch": ([C.POINTER(Round), P], I),
    "ttb_amen_slab_doubles": ([I, C.POINTER(C.c_int), I, I, I], L),
    "ttb_amen_persistent": ([P, I, I, P], I),
    "ttb_amen_persistent_cluster": ([P, I, I, I, P], I),
}

_lib = None
_lock = threading.Lock()


def exported_symbols():
    """Names the header declares, in declaration order."""
    return list(_SIGNATURES)


def load(path: str = LIB_PATH):
    """Load (once) and return the library handle with typed entry points."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(
                f"libttb200 is not built ({path} missing); run "
                "`python -c 'import __graft_entry__ as g; g.build()'` or "
                "`python -m ttnumpy_b200.build`")
        lib = C.CDLL(path)
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


class CudaError(RuntimeError):
    """A libttb200 entry point returned a CUDA error code."""


def check(code: int, what: str) -> None:
    if code != 0:
        raise CudaError(f"{what} failed with CUDA error {code}")


def array(struct_type, items):
    """ctypes array of ``struct_type`` from a list of field dicts / structs."""
    arr = (struct_type * len(items))()
    for i, it in enumerate(items):
        if isinstance(it, dict):
            for k, v in it.items():
                setattr(arr[i], k, v)
        else:
            arr[i] = it
    return arr
