"""B200-native tensor-train solve path: AMEn, TT rounding, TTM-by-TT.

Drop-in replacements for the reference entry points ``amen``, ``als``,
``mals``, ``TensorTrain.truncate`` and ``TensorTrain.dot`` (ttnumpy 0.3.0), computed
by hand-written sm_100a kernels in ``libttb200.so`` (C ABI in
``include/ttb200.h``).  There is no CPU path: the entry points raise when
the library or a CUDA device is missing.
"""

__version__ = "0.1.0"

from .solvers.common import (  # noqa: F401
    LocalSolver,
    SolverInfo,
    StopReason,
    TruncationMode,
    relative_residual,
)
from .solvers.als import als  # noqa: F401
from .solvers.amen import amen  # noqa: F401
from .solvers.mals import mals  # noqa: F401
from .tensor_train import (  # noqa: F401
    AmbiguousFormat,
    DimensionMismatch,
    TensorTrain,
    TensorTrainType,
    WrongTTFormat,
    WrongTTType,
    canonical_tt,
    eye,
    ones,
    rand,
    tt_svd,
    zeros,
)

__all__ = [
    "TensorTrain", "TensorTrainType", "ones", "zeros", "eye", "rand", "amen", "als", "mals",
    "SolverInfo", "StopReason", "LocalSolver", "TruncationMode", "relative_residual",
    "DimensionMismatch", "WrongTTFormat", "WrongTTType", "AmbiguousFormat", "tt_svd", "canonical_tt",
]
