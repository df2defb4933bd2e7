"""The C-ABI library: builds, loads without a GPU, exports every symbol
``include/ttb200.h`` declares, and the ctypes mirror matches the header."""

import ctypes
import os
import re

from conftest import ROOT


def header_functions():
    text = open(os.path.join(ROOT, "include", "ttb200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"^\s*(?:long long|int|void)\s+(ttb_\w+)\s*\(", text, flags=re.M)


def test_library_exports_header_symbols():
    from ttnumpy_b200 import build, _lib

    path = build.build()
    lib = ctypes.CDLL(path)
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    # the Python mirror binds exactly the declared functions
    assert sorted(names) == sorted(_lib.exported_symbols())
    assert _lib.load(path).ttb_version() >= 1


def test_struct_sizes_match_c():
    """ctypes struct sizes against sizeof() compiled from the header."""
    import subprocess
    import tempfile

    from ttnumpy_b200 import _lib

    pairs = {"ttb_gemm_t": _lib.Gemm, "ttb_env_t": _lib.Env, "ttb_local_t": _lib.Local,
             "ttb_local_matrix_t": _lib.LocalMatrix, "ttb_project_t": _lib.Project,
             "ttb_qr_t": _lib.QR, "ttb_svd_t": _lib.SVD, "ttb_lu_t": _lib.LU,
             "ttb_copy_t": _lib.Copy, "ttb_kron_t": _lib.Kron, "ttb_norm_t": _lib.Norm,
             "ttb_hadamard_t": _lib.Hadamard,
             "ttb_rank_t": _lib.Rank, "ttb_rank_rule_t": _lib.RankRule,
             "ttb_krylov_t": _lib.Krylov, "ttb_round_t": _lib.Round,
             "ttb_amen_task_t": _lib.AmenTask}
    src = '#include <stdio.h>\n#include "ttb200.h"\nint main(void){\n'
    for name in pairs:
        src += f'printf("%zu\\n", sizeof({name}));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as tmp:
        c = os.path.join(tmp, "s.c")
        exe = os.path.join(tmp, "s")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        sizes = [int(v) for v in subprocess.run([exe], capture_output=True, text=True,
                                                check=True).stdout.split()]
    for (name, st), size in zip(pairs.items(), sizes):
        assert ctypes.sizeof(st) == size, name
