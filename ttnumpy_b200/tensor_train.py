"""Device-resident tensor train with the reference container's interface.

``TensorTrain`` keeps its cores as CUDA float64 tensors of shape
``(r_k, row_mode_k, col_mode_k, r_{k+1})`` (the reference layout,
``ttnumpy/tensor_train.py:150-244``).  Rounding (``truncate``,
``orthonormalize``, ``compress_svd``), the TTM-by-TT product (``dot``), sums
and norms run on the GPU through libttb200; only rank decisions and norms
come back to the host.  Constructors take host NumPy arrays (input
preparation is host work in the reference too) and upload them.
"""

from __future__ import annotations

import logging
import math
import numbers
from enum import Enum
from typing import List, Optional, Tuple, Union

import numpy as np
import torch

from . import kernels as K

logger = logging.getLogger("ttnumpy")


class AmbiguousFormat(Exception):
    """Not enough information to define a train (``tensor_train.py:45-50``)."""

    def __init__(self, msg="Not enough information to define object"):
        self.msg = msg
        super().__init__(self.msg)


class DimensionMismatch(Exception):
    """Exception for dimension errors (``tensor_train.py:21-26``)."""

    def __init__(self, msg="Dimension mismatch"):
        self.msg = msg
        super().__init__(self.msg)


class WrongTTFormat(Exception):
    """Exception for an invalid train structure (``tensor_train.py:29-34``)."""

    def __init__(self, msg="Wrong tensor train format"):
        self.msg = msg
        super().__init__(self.msg)


class WrongTTType(Exception):
    """Exception for a TT where a TTM is needed or vice versa
    (``tensor_train.py:37-42``)."""

    def __init__(self, msg="Wrong tensor train type"):
        self.msg = msg
        super().__init__(self.msg)


class TensorTrainType(Enum):
    TT = "Tensor Train"
    TTM = "Tensor Train Matrix"


def _to_device(core) -> torch.Tensor:
    if isinstance(core, torch.Tensor):
        t = core.to(device="cuda", dtype=torch.float64)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(core, dtype=np.float64))).to("cuda")
    return t.contiguous()


def _mat(core: torch.Tensor, rows: int) -> torch.Tensor:
    return core.reshape(rows, -1)


class TensorTrain:
    """Tensor train (TT) or tensor train matrix (TTM) on the GPU.

    Validation and attributes follow the reference constructor
    (``tensor_train.py:169-244``).
    """

    __array_ufunc__ = None

    def __init__(self, cores: List, orth_center: Optional[int] = None):
        K.device_ok()
        if len(cores) < 2:
            raise WrongTTFormat("Tensor train must has at least 2 sites")
        ndims = {len(c.shape) for c in cores}
        if ndims == {3}:
            cores = [_to_device(c).reshape(c.shape[0], c.shape[1], 1, c.shape[2]) for c in cores]
        elif ndims == {4}:
            cores = [_to_device(c) for c in cores]
        else:
            raise WrongTTFormat("All cores must be 3 or 4 rank tensors")
        tt_type = (TensorTrainType.TT if all(c.shape[2] == 1 for c in cores)
                   else TensorTrainType.TTM)
        bonds = [1]
        for i, core in enumerate(cores):
            if i == 0 and core.shape[0] != 1:
                raise WrongTTFormat("Only open boundary conditions is supported, first core "
                                    "must has first index equal to 1")
            if i == len(cores) - 1 and core.shape[-1] != 1:
                raise WrongTTFormat("Only open boundary conditions is supported, last core "
                                    "must has last index equal to 1")
            if core.shape[0] != bonds[i]:
                raise DimensionMismatch(
                    f"Connected sites bonds are mismatching: {core.shape[0]} != {bonds[i]}")
            bonds.append(core.shape[-1])
        self.cores = cores
        self.tt_type = tt_type
        self.orth_center = orth_center

    # -- attributes ---------------------------------------------------------

    @property
    def n_cores(self) -> int:
        return len(self.cores)

    @property
    def bonds(self) -> List[int]:
        return [int(c.shape[0]) for c in self.cores] + [1]

    @property
    def row_modes(self) -> List[int]:
        return [int(c.shape[1]) for c in self.cores]

    @property
    def col_modes(self) -> List[int]:
        if self.tt_type is TensorTrainType.TT:
            return [1] * len(self.cores)
        return [int(c.shape[2]) for c in self.cores]

    @property
    def max_rank(self) -> int:
        return max(self.bonds)

    def __len__(self) -> int:
        return len(self.cores)

    def __getitem__(self, idx):
        return self.cores[idx]

    def is_ttm(self) -> bool:
        return self.tt_type is TensorTrainType.TTM

    def physical_dims(self) -> List:
        if self.tt_type is TensorTrainType.TT:
            return self.row_modes
        return list(zip(self.row_modes, self.col_modes))

    def copy(self) -> "TensorTrain":
        out = TensorTrain.__new__(TensorTrain)
        out.cores = [c.clone() for c in self.cores]
        out.tt_type = self.tt_type
        out.orth_center = self.orth_center
        return out

    @classmethod
    def _wrap(cls, cores: List[torch.Tensor], orth_center=None) -> "TensorTrain":
        out = cls.__new__(cls)
        out.cores = cores
        out.tt_type = (TensorTrainType.TT if all(c.shape[2] == 1 for c in cores)
                       else TensorTrainType.TTM)
        out.orth_center = orth_center
        return out

    # -- host transfer ------------------------------------------------------

    def to_numpy(self) -> List[np.ndarray]:
        return [c.detach().cpu().numpy() for c in self.cores]

    def get_full_tensor(self) -> np.ndarray:
        """Dense tensor on the host (a convenience for small trains; the
        contraction order of ``tensor_train.py:599-624``)."""
        cores = self.to_numpy()
        t = cores[0].reshape(-1, cores[0].shape[-1])
        for c in cores[1:]:
            t = (t @ c.reshape(c.shape[0], -1)).reshape(-1, c.shape[-1])
        t = t.reshape(-1)
        if self.is_ttm():
            shape = [x for p in zip(self.row_modes, self.col_modes) for x in p]
            t = t.reshape(shape)
            d = len(self.cores)
            perm = list(range(0, 2 * d, 2)) + list(range(1, 2 * d, 2))
            return t.transpose(perm)
        shape = self.row_modes
        if shape == [1] * len(shape):
            return t.item()
        return t.reshape(shape)

    def get_element(self, element_index) -> float:
        """One entry (``tensor_train.py:556-596``): the product of each
        core's (bond x bond) slice at the given index, by device GEMMs on the
        strided slices.  A TT takes plain indices, a TTM (row, column)
        pairs."""
        if len(element_index) != len(self):
            raise DimensionMismatch(
                "Number of indexes not equal to number of tensor train cores: "
                f"{len(element_index)} != {len(self)}")
        idx = list(element_index)
        if self.tt_type is TensorTrainType.TT and isinstance(idx[0], (int, np.integer)):
            idx = [(int(i), 0) for i in idx]
        acc = self.cores[0][:, idx[0][0], idx[0][1], :]
        for core, (i, j) in zip(self.cores[1:], idx[1:]):
            acc = K.matmul(acc, core[:, i, j, :])
        return acc.reshape(-1)[0].item()

    def matricize(self):
        """The train as a vector (TT) or a (rows x columns) matrix (TTM) on
        the host (``tensor_train.py:626-638``), the cores merged on the
        device first."""
        merged = _merge_cores([c.contiguous() for c in self.cores]).cpu().numpy()
        if not self.is_ttm():
            return merged.reshape(-1)
        return merged.reshape(math.prod(self.row_modes), math.prod(self.col_modes))

    def transpose(self, cores_ind: Optional[List[int]] = None, conjugate: bool = False,
                  inplace: bool = False) -> "TensorTrain":
        """Swap the row and column modes of the given cores (all by default)
        by one permuted copy each (``tensor_train.py:647-689``).  The cores
        are real, so ``conjugate`` changes nothing."""
        t = self if inplace else self.copy()
        for i in (range(len(t)) if cores_ind is None else cores_ind):
            c = t.cores[i]
            out = K.empty(c.shape[0], c.shape[2], c.shape[1], c.shape[3])
            K.copy_(out, c.permute(0, 2, 1, 3))
            t.cores[i] = out
        t.tt_type = (TensorTrainType.TT if all(c.shape[2] == 1 for c in t.cores)
                     else TensorTrainType.TTM)
        return t

    def conj(self, inplace: bool = False) -> "TensorTrain":
        """Complex conjugate (``tensor_train.py:691-703``): the cores are
        real float64, so the train itself (or a copy)."""
        return self if inplace else self.copy()

    # -- arithmetic ---------------------------------------------------------

    def add(self, other: "TensorTrain", truncate: bool = False, error=None, max_rank=None,
            method: str = "direct", seed=None, options=None) -> "TensorTrain":
        """Block-diagonal sum (``tensor_train.py:254-322``)."""
        if not isinstance(other, TensorTrain):
            raise TypeError(
                f"unsupported operand type(s) for +: 'TensorTrain' and '{type(other)}'")
        if self.physical_dims() != other.physical_dims():
            raise DimensionMismatch("Tensor trains must have the same dimensions")
        d = len(self)
        ra, rb = self.bonds, other.bonds
        ranks = [1] + [ra[i] + rb[i] for i in range(1, d)] + [1]
        cores, descs = [], []
        for i in range(d):
            a, b = self.cores[i], other.cores[i]
            out = torch.empty(ranks[i], a.shape[1], a.shape[2], ranks[i + 1], dtype=torch.float64,
                              device="cuda")
            descs.append(K.copy_desc(None, out, 0.0))
            cores.append(out)
        K.copy_many(descs)
        descs = []
        for i in range(d):
            a, b, out = self.cores[i], other.cores[i], cores[i]
            descs.append(K.copy_desc(a, out[: ra[i], :, :, : ra[i + 1]]))
            descs.append(K.copy_desc(b, out[ranks[i] - rb[i]:, :, :, ranks[i + 1] - rb[i + 1]:]))
        K.copy_many(descs)
        res = TensorTrain._wrap(cores)
        return _round_result(res, truncate, error, max_rank, method, seed, options)

    def __add__(self, other):
        return self.add(other)

    def multiply(self, other, truncate: bool = False, error=None, max_rank=None,
                 method: str = "direct", seed=None, options=None) -> "TensorTrain":
        """Element-wise product with a train or a scalar
        (``tensor_train.py:327-407``).  Two trains: the product cores
        (Kronecker over the bonds) come from ``ttb_hadamard``; with
        ``truncate=True, method="randomized"`` they are never formed: HaTT-1
        (:func:`randomized_hadamard`) gives the left-orthonormal cores of the
        product, which the SVD sweep then truncates."""
        if isinstance(other, TensorTrain):
            if self.physical_dims() != other.physical_dims():
                raise DimensionMismatch("Tensor trains must have the same dimensions")
            if truncate and method == "randomized":
                cores = randomized_hadamard(self.cores, other.cores,
                                            _sketch_rank(max_rank, options),
                                            np.random.default_rng(seed))
                res = TensorTrain._wrap(cores, orth_center=len(cores) - 1)
                return res.compress_svd(0.0 if error is None else error, max_rank, inplace=True)
            cores = [K.hadamard(a.contiguous(), b.contiguous())
                     for a, b in zip(self.cores, other.cores)]
            return _round_result(TensorTrain._wrap(cores), truncate, error, max_rank, method,
                                 seed, options)
        if isinstance(other, numbers.Number) and not isinstance(other, bool):
            res = self.copy()
            k = res.orth_center if res.orth_center is not None else 0
            K.copy_(res.cores[k], self.cores[k], float(other))
            return _round_result(res, truncate, error, max_rank, method, seed, options)
        raise TypeError(f"unsupported operand type(s) for *: 'TensorTrain' and '{type(other)}'")

    def __mul__(self, other):
        return self.multiply(other)

    def __rmul__(self, other):
        return self.multiply(other)

    def __neg__(self):
        return self.multiply(-1)

    def __sub__(self, other):
        return self.add(-other)

    def dot(self, other: "TensorTrain", truncate: bool = False, error=None, max_rank=None,
            method: str = "direct", seed=None, options=None) -> "TensorTrain":
        """TTM-by-TT (or TTM-by-TTM) product, Kronecker cores built on the
        device (``tensor_train.py:427-499``)."""
        if not isinstance(other, TensorTrain):
            raise TypeError(
                f"unsupported operand type(s) for @: 'TensorTrain' and '{type(other)}'")
        if self.col_modes != other.row_modes:
            raise DimensionMismatch("Tensor trains must have the same last and first physical "
                                    "dimensions respectively")
        cores = [K.kron(a, x) for a, x in zip(self.cores, other.cores)]
        return _round_result(TensorTrain._wrap(cores), truncate, error, max_rank, method, seed,
                             options)

    def __matmul__(self, other):
        return self.dot(other)

    # -- norms and canonical forms ------------------------------------------

    def tt_norm(self) -> float:
        """Frobenius norm; the centre core's norm when ``orth_center`` is
        set, else a right QR sweep that keeps only the R factors
        (``tensor_train.py:509-540``)."""
        out = K.empty(1)
        if self.orth_center is not None:
            K.norm_into(out, self.cores[self.orth_center])
            return float(out.item())
        carry = None
        for i in range(len(self) - 1, 0, -1):
            c = self.cores[i]
            m = c if carry is None else _apply_right(c, carry)
            mat = _mat(m, m.shape[0])
            _, r = K.qr(mat.t(), want_q=False)
            carry = r.t()  # (r_i, p) : previous core @ carry
        first = _apply_right(self.cores[0], carry)
        K.norm_into(out, first)
        return float(out.item())

    def orthonormalize(self, canonical: str = "left", center_position: Optional[int] = None,
                       inplace: bool = False) -> "TensorTrain":
        """QR canonicalisation (``tensor_train.py:705-787``)."""
        d = len(self)
        if center_position is not None and not 0 <= center_position < d:
            raise ValueError(f"center_position must be in [0, {d - 1}], but got {center_position}")
        t = self if inplace else self.copy()
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
        elif canonical == "mix":
            if center_position is None:
                center_position = d // 2
            end = center_position
            left_orth_sweep(t.cores, 0, center_position)
            right_orth_sweep(t.cores, d - 1, center_position)
        else:
            raise ValueError(
                f"Canonical form must be 'left', 'right' or 'mix', but got {canonical}")
        if had_center or canonical == "mix" or end in (0, d - 1):
            t.orth_center = end
        else:
            t.orth_center = None
        return t

    def compress_svd(self, error: float = 0.0, max_rank: Optional[int] = None,
                     canonical: str = "auto", inplace: bool = False) -> "TensorTrain":
        """SVD truncation sweep (``tensor_train.py:789-850``)."""
        t = self if inplace else self.copy()
        d = len(t)
        if canonical == "auto":
            canonical = ("left" if (t.orth_center is None or t.orth_center <= (d - 1) / 2)
                         else "right")
        if canonical == "right":
            right_svd_sweep(t.cores, error, max_rank)
            t.orth_center = 0
        elif canonical == "left":
            left_svd_sweep(t.cores, error, max_rank)
            t.orth_center = d - 1
        else:
            raise ValueError(
                f"Canonical form must be 'left', 'right' or 'auto', but got {canonical}")
        return t

    def truncate(self, error: float = 0.0, max_rank: Optional[int] = None,
                 canonical: str = "auto", inplace: bool = False, method: str = "direct",
                 seed=None, options=None) -> "TensorTrain":
        """Round to minimal ranks: QR canonicalisation then the SVD sweep
        (``tensor_train.py:852-940``, ``method="direct"``)."""
        if canonical not in ("auto", "left", "right"):
            raise ValueError(
                f"Canonical form must be 'left', 'right' or 'auto', but got {canonical}")
        if method not in ("direct", "randomized"):
            raise ValueError(f"Method must be 'direct' or 'randomized', but got {method!r}")
        if method == "randomized":
            rank = _sketch_rank(max_rank, options)
        t = self if inplace else self.copy()
        orth_form = "left" if canonical == "right" else "right"
        if canonical == "auto":
            if t.orth_center is None or t.orth_center >= len(t) / 2:
                orth_form = "left"
            else:
                orth_form = "right"
        if method == "direct":
            t.orthonormalize(canonical=orth_form, inplace=True)
        else:
            rng = np.random.default_rng(seed)
            if orth_form == "left":
                randomized_left_orth(t.cores, rank, rng)
                t.orth_center = len(t) - 1
            else:
                randomized_right_orth(t.cores, rank, rng)
                t.orth_center = 0
        t.compress_svd(error, max_rank, inplace=True)
        return t

    def tt_to_qtt(self, mode_size: int = 2, error: float = 1e-12,
                  max_rank: Optional[int] = None) -> "TensorTrain":
        """Quantise every mode into cores of mode ``mode_size``, as the
        reference's ``tt_to_qtt`` (``tensor_train.py:942-1066``).

        After a right QR sweep, a core of mode ``mode_size^q`` is split left
        to right by q - 1 device SVDs of its (bond * mode_size, rest)
        unfolding (a TTM's row and column halves kept paired by one strided
        copy per split), and the remainder of each group is pushed into the
        next core by one more SVD.  Every split truncates at
        ``delta = error / sqrt(#SVDs) * ||t||``.  The result is
        left-orthonormal with its centre on the last core.
        """
        if mode_size < 2:
            raise ValueError(f"mode_size must be at least 2, but got {mode_size}")
        if max_rank is not None and max_rank <= 0:
            raise ValueError("max_rank must be a positive integer.")
        ttm = self.is_ttm()
        nums = []
        for i, m in enumerate(self.row_modes):
            q = 0
            while mode_size ** q < m:
                q += 1
            if mode_size ** q != m:
                raise DimensionMismatch(f"Row mode {m} not a power of {mode_size}")
            if ttm and mode_size ** q != self.col_modes[i]:
                raise DimensionMismatch("Column mode size of TTM not a power of mode size")
            if q == 0:
                raise ValueError("a core of mode 1 cannot be split into cores of mode "
                                 f"{mode_size}")
            nums.append(q)
        rms, cms = mode_size, (mode_size if ttm else 1)
        count = max(1, sum(q - 1 for q in nums) + len(self) - 1)
        t = self.orthonormalize(canonical="right")
        delta = error / math.sqrt(count) * t.tt_norm()
        cores = t.cores
        out: List[torch.Tensor] = []

        def split(matrix: torch.Tensor, lb: int):
            u, sv, _ = K.svd(matrix)
            nb = _svd_rank(sv, delta, max_rank)
            piece = K.empty(matrix.shape[0], nb)
            K.copy_(piece, u[:, :nb])
            out.append(piece.view(lb, rms, cms, nb))
            return K.matmul(piece.t(), matrix), nb

        for i, q in enumerate(nums):
            core = cores[i].reshape(-1)  # laid out (lb, rms, rms^j, cms, cms^j, rb)
            lb, rb = cores[i].shape[0], cores[i].shape[-1]
            for j in range(q - 1, 0, -1):
                tail = cms ** j * rb
                if cms > 1:  # bring the first column factor next to the first row factor
                    matrix = K.empty(lb * rms * cms, rms ** j * tail)
                    K.copy_(matrix.view(lb * rms, cms, rms ** j, tail),
                            core.as_strided((lb * rms, cms, rms ** j, tail),
                                            (rms ** j * cms * tail, tail, cms * tail, 1)))
                else:
                    matrix = core.view(lb * rms, -1)
                core, lb = split(matrix, lb)
                core = core.reshape(-1)
            if i < len(nums) - 1:
                carry, _ = split(core.view(lb * rms * cms, rb), lb)
                cores[i + 1] = _apply_left(carry, cores[i + 1])
            else:
                out.append(core.view(lb, rms, cms, rb))
        return TensorTrain._wrap(out, orth_center=len(out) - 1)

    def qtt_to_tt(self, physical_indexes, error: float = 1e-12,
                  max_rank: Optional[int] = None) -> "TensorTrain":
        """Merge groups of consecutive quantised cores back into one core
        each and round the result, as the reference's ``qtt_to_tt``
        (``tensor_train.py:1072-1135``): a group takes cores until its row
        (and, for a TTM, column) modes multiply to the requested index.
        Merging is one device GEMM per core plus, for a TTM, one strided
        copy that moves the new row factor in front of the column factors.
        """
        ttm = self.is_ttm()
        groups = []
        pos = 0
        for i, idx in enumerate(physical_indexes):
            rt, ct = (idx if ttm else (idx, 1))
            pr = pc = 1
            n = 0
            while n == 0 or pr != rt or pc != ct:
                if pos + n >= len(self):
                    raise DimensionMismatch(
                        f"Not enough QTT cores to match physical index for core {i}")
                pr *= self.row_modes[pos + n]
                pc *= self.col_modes[pos + n]
                n += 1
                if pr > rt:
                    raise DimensionMismatch(
                        f"Row mode size of QTT exceeds original row mode size for core {i}")
                if pc > ct:
                    raise DimensionMismatch(
                        f"Column mode size of QTT exceeds original column mode size for core {i}")
            groups.append((pos, n))
            pos += n
        if pos != len(self):
            raise DimensionMismatch(f"Physical indexes cover only {pos} of {len(self)} QTT cores")
        merged = [_merge_cores(self.cores[p:p + n]) for p, n in groups]
        return TensorTrain._wrap(merged).truncate(error=error, max_rank=max_rank)

    def __str__(self):
        return (f"{self.tt_type.value} with following properties:\n\t Number of cores: "
                f"{len(self)}\n\t Bonds: {self.bonds}\n\t Physical indexes: "
                f"{self.physical_dims()}")


def _round_result(res, truncate, error, max_rank, method, seed=None, options=None):
    """``_round_result`` (``tensor_train.py:94-119``)."""
    if not truncate:
        if method != "direct" or error is not None or max_rank is not None:
            raise ValueError("error, max_rank and method need truncate=True")
        return res
    return res.truncate(error=0.0 if error is None else error, max_rank=max_rank, inplace=True,
                        method=method, seed=seed, options=options)


# ---------------------------------------------------------------------------
# sweeps on lists of device cores (utils.py:86-136, 364-460)
# ---------------------------------------------------------------------------


def _apply_left(matrix: torch.Tensor, core: torch.Tensor) -> torch.Tensor:
    """``matrix @ core`` over the first core axis (``utils.py:72-76``)."""
    out = torch.empty((matrix.shape[0],) + tuple(core.shape[1:]), dtype=torch.float64,
                      device="cuda")
    K.gemm(matrix, core.reshape(core.shape[0], -1), out.view(matrix.shape[0], -1))
    return out


def _merge_cores(cores: List[torch.Tensor]) -> torch.Tensor:
    """Product of consecutive cores as one core (``tensor_train.py:57-92``):
    each step multiplies the (left * rows * cols, bond) unfolding of the
    running product by the next core's (bond, rest) unfolding, then moves
    the new row factor in front of the running column factor."""
    acc = cores[0]
    for c in cores[1:]:
        lb, R, C, b = acc.shape
        _, r, s, rb = c.shape
        prod = K.matmul(acc.reshape(-1, b), c.reshape(b, -1))
        if C > 1 and r > 1:
            out = K.empty(lb * R * r * C * s * rb)
            tail = s * rb
            K.copy_(out.view(lb * R, r, C, tail),
                    prod.view(-1).as_strided((lb * R, r, C, tail),
                                             (C * r * tail, tail, r * tail, 1)))
            prod = out
        acc = prod.view(lb, R * r, C * s, rb)
    return acc


def _apply_right(core: torch.Tensor, matrix: torch.Tensor) -> torch.Tensor:
    """``core @ matrix`` over the last core axis (``utils.py:79-83``)."""
    out = torch.empty(tuple(core.shape[:-1]) + (matrix.shape[1],), dtype=torch.float64,
                      device="cuda")
    K.gemm(core.reshape(-1, core.shape[-1]), matrix, out.view(-1, matrix.shape[1]))
    return out


def _sketch_rank(max_rank: Optional[int], options: Optional[dict]) -> int:
    """Bond of the random sketch of ``method="randomized"``
    (``tensor_train.py:122-140``)."""
    if max_rank is None:
        raise ValueError("method='randomized' needs max_rank")
    options = {} if options is None else options
    unknown = set(options) - {"oversampling"}
    if unknown:
        raise ValueError(f"Unknown options for method='randomized': {sorted(unknown)}")
    over = options.get("oversampling", 10)
    if not isinstance(over, numbers.Integral) or isinstance(over, bool) or over < 0:
        raise ValueError(f"oversampling must be a non-negative integer, but got {over!r}")
    return max_rank + over


def randomized_left_orth(cores: List[torch.Tensor], rank: int, rng) -> List[torch.Tensor]:
    """Randomize-then-orthogonalise (``left_randomized_orthonormalize``,
    ``utils.py:139-203``) on the device: the cores right of each bond are
    contracted with a Gaussian train (its cores drawn on the host from
    ``rng`` in the reference's order and shapes), then every unfolding
    times the next sketch is factorised by QR and the remainder moved right.
    Each sketch is scaled to unit norm (the reference scales by its largest
    entry; a positive scale leaves the Q factors unchanged, it only keeps
    long trains from overflowing)."""
    if rank < 1:
        raise ValueError(f"rank must be positive, but got {rank}")
    count = len(cores)
    sketches: List[Optional[torch.Tensor]] = [None] * count + [K.fill_(K.empty(1, 1), 1.0)]
    nrm = K.empty(1)
    for i in range(count - 1, 0, -1):
        c = cores[i]
        contracted = K.matmul(c.reshape(-1, c.shape[3]), sketches[i + 1])
        cols = contracted.numel() // c.shape[0]
        contracted = contracted.view(c.shape[0], cols)
        bond = min(rank, c.shape[0], cols)
        gauss = torch.from_numpy(rng.standard_normal((cols, bond))).to("cuda")
        sk = K.matmul(contracted, gauss)
        K.norm_into(nrm, sk)
        scale = float(nrm.item())
        if scale > 0:
            K.copy_(sk, sk, alpha=1.0 / scale)
        sketches[i] = sk
    for i in range(count - 1):
        s = cores[i].shape
        matrix = cores[i].reshape(s[0] * s[1] * s[2], s[3])
        q, _ = K.qr(K.matmul(matrix, sketches[i + 1]), want_r=False)
        cores[i] = q.reshape(s[0], s[1], s[2], q.shape[1])
        cores[i + 1] = _apply_left(K.matmul(q.t(), matrix), cores[i + 1])
    return cores


def randomized_right_orth(cores: List[torch.Tensor], rank: int, rng) -> List[torch.Tensor]:
    """Mirror image of :func:`randomized_left_orth`
    (``right_randomized_orthonormalize``, ``utils.py:206-236``)."""
    def mirror(c):
        out = K.empty(c.shape[3], c.shape[1], c.shape[2], c.shape[0])
        return K.copy_(out, c.permute(3, 1, 2, 0))

    mirrored = [mirror(c) for c in reversed(cores)]
    randomized_left_orth(mirrored, rank, rng)
    cores[:] = [mirror(c) for c in reversed(mirrored)]
    return cores


def _hadamard_times_sketch(lhs: torch.Tensor, rhs: torch.Tensor,
                           sketch: torch.Tensor) -> torch.Tensor:
    """The product core of ``lhs`` (r, m, n, r') and ``rhs`` (s, m, n, s')
    times ``sketch`` (r', s', l) over its right bond, as a (r * s, m n l)
    matrix, without the product core (``utils.py:225-240``): one GEMM with
    ``lhs``, one permuted copy, one GEMM per mode with ``rhs`` and a final
    permuted copy into (r, s, modes, l) order."""
    r, rr = lhs.shape[0], lhs.shape[3]
    s, sr = rhs.shape[0], rhs.shape[3]
    modes = lhs.shape[1] * lhs.shape[2]
    ell = sketch.shape[2]
    half = K.matmul(lhs.reshape(r * modes, rr), sketch.reshape(rr, sr * ell))
    half = half.view(r, modes, sr, ell)
    ht = K.empty(modes, sr, r, ell)  # (p, d, a, t)
    K.copy_(ht, half.permute(1, 2, 0, 3))
    full = K.empty(modes, s, r * ell)  # (p, c, (a, t))
    K.gemm(rhs.reshape(s, modes, sr).permute(1, 0, 2), ht.view(modes, sr, r * ell), full)
    out = K.empty(r, s, modes, ell)
    K.copy_(out, full.view(modes, s, r, ell).permute(2, 1, 0, 3))
    return out.view(r * s, modes * ell)


def _carry_times_hadamard(carry: torch.Tensor, lhs: torch.Tensor,
                          rhs: torch.Tensor) -> torch.Tensor:
    """``carry`` (l, r, s) times the product core of ``lhs`` (r, m, n, r')
    and ``rhs`` (s, m, n, s') over its left bond, as a (l m n, r' s')
    matrix, without the product core (``utils.py:243-259``): one GEMM per
    carry row with ``lhs``, one permuted copy, one GEMM per mode with
    ``rhs`` and a final permuted copy into (l, modes, r', s') order."""
    ell, r, s = carry.shape
    rr, sr = lhs.shape[3], rhs.shape[3]
    modes = lhs.shape[1] * lhs.shape[2]
    half = K.empty(ell, s, modes * rr)  # (t, c, (p, b))
    K.gemm(carry.permute(0, 2, 1), lhs.reshape(1, r, modes * rr), half)
    ht = K.empty(modes, ell, rr, s)  # (p, t, b, c)
    K.copy_(ht, half.view(ell, s, modes, rr).permute(2, 0, 3, 1))
    full = K.empty(modes, ell * rr, sr)  # (p, (t, b), d)
    K.gemm(ht.view(modes, ell * rr, s), rhs.reshape(s, modes, sr).permute(1, 0, 2), full)
    out = K.empty(ell, modes, rr, sr)
    K.copy_(out, full.view(modes, ell, rr, sr).permute(1, 0, 2, 3))
    return out.view(ell * modes, rr * sr)


def randomized_hadamard(lhs: List[torch.Tensor], rhs: List[torch.Tensor], rank: int,
                        rng) -> List[torch.Tensor]:
    """HaTT-1 (``randomized_hadamard``, ``utils.py:262-333``) on the device:
    the randomized left orthonormalisation of the element-wise product of
    two trains, never forming a product core.  Right to left, the product
    right of each bond is contracted with a Gaussian train drawn on the host
    from ``rng`` in the reference's order and shapes; left to right, the
    carried projection times the two cores times the next sketch is
    factorised by QR.  Sketches are scaled to unit norm (the reference
    scales by the largest entry; the Q factors do not change)."""
    if rank < 1:
        raise ValueError(f"rank must be positive, but got {rank}")
    count = len(lhs)
    lhs = [c.contiguous() for c in lhs]
    rhs = [c.contiguous() for c in rhs]
    sketches: List[Optional[torch.Tensor]] = [None] * count + [K.fill_(K.empty(1, 1, 1), 1.0)]
    nrm = K.empty(1)
    for i in range(count - 1, 0, -1):
        contracted = _hadamard_times_sketch(lhs[i], rhs[i], sketches[i + 1])
        bond = min(rank, *contracted.shape)
        gauss = torch.from_numpy(rng.standard_normal((contracted.shape[1], bond))).to("cuda")
        sk = K.matmul(contracted, gauss)
        K.norm_into(nrm, sk)
        scale = float(nrm.item())
        if scale > 0:
            K.copy_(sk, sk, alpha=1.0 / scale)
        sketches[i] = sk.view(lhs[i].shape[0], rhs[i].shape[0], bond)
    cores: List[torch.Tensor] = []
    carry = K.fill_(K.empty(1, 1, 1), 1.0)
    for i in range(count):
        matrix = _carry_times_hadamard(carry, lhs[i], rhs[i])
        n, m = lhs[i].shape[1], lhs[i].shape[2]
        if i == count - 1:
            cores.append(matrix.view(carry.shape[0], n, m, -1))
            break
        q, _ = K.qr(K.matmul(matrix, sketches[i + 1].reshape(matrix.shape[1], -1)),
                    want_r=False)
        cores.append(q.reshape(carry.shape[0], n, m, q.shape[1]))
        carry = K.matmul(q.t(), matrix).view(q.shape[1], lhs[i].shape[3], rhs[i].shape[3])
    return cores


def left_orth_sweep(cores: List[torch.Tensor], start: int, end: int) -> None:
    for i in range(start, end):
        s = cores[i].shape
        q, r = K.qr(cores[i].reshape(s[0] * s[1] * s[2], s[3]))
        cores[i] = q.reshape(s[0], s[1], s[2], q.shape[1])
        cores[i + 1] = _apply_left(r, cores[i + 1])


def right_orth_sweep(cores: List[torch.Tensor], start: int, end: int) -> None:
    for i in range(start, end, -1):
        s = cores[i].shape
        rest = s[1] * s[2] * s[3]
        p = min(rest, s[0])
        qt = K.empty(p, rest)  # Q^T, written through a transposed view
        _, r = K.qr(cores[i].reshape(s[0], rest).t(), q_out=qt.t())
        cores[i] = qt.reshape(p, s[1], s[2], s[3])
        cores[i - 1] = _apply_right(cores[i - 1], r.t())


def _svd_rank(s: torch.Tensor, delta: float, max_rank) -> int:
    rk = torch.empty(1, dtype=torch.int32, device="cuda")
    K.rank_threshold(s, 1, delta, max_rank, rk)
    return int(rk.item())


def left_svd_sweep(cores: List[torch.Tensor], error: float, max_rank=None) -> None:
    if max_rank is not None and max_rank <= 0:
        raise ValueError("max_rank must be a positive integer.")
    nrm = K.empty(1)
    K.norm_into(nrm, cores[0])
    delta = error / math.sqrt(len(cores) - 1) * float(nrm.item())
    for i in range(len(cores) - 1):
        s = cores[i].shape
        u, sv, vh = K.svd(cores[i].reshape(s[0] * s[1] * s[2], s[3]))
        nb = _svd_rank(sv, delta, max_rank)
        core = K.empty(s[0], s[1], s[2], nb)
        K.copy_(core.view(-1, nb), u[:, :nb])
        carry = K.empty(nb, s[3])
        K.copy_(carry, vh[:nb], scale=sv, scale_axis=0)
        cores[i] = core
        cores[i + 1] = _apply_left(carry, cores[i + 1])


def right_svd_sweep(cores: List[torch.Tensor], error: float, max_rank=None) -> None:
    if max_rank is not None and max_rank <= 0:
        raise ValueError("max_rank must be a positive integer.")
    nrm = K.empty(1)
    K.norm_into(nrm, cores[-1])
    delta = error / math.sqrt(len(cores) - 1) * float(nrm.item())
    for i in range(len(cores) - 1, 0, -1):
        s = cores[i].shape
        u, sv, vh = K.svd(cores[i].reshape(s[0], s[1] * s[2] * s[3]))
        nb = _svd_rank(sv, delta, max_rank)
        core = K.empty(nb, s[1], s[2], s[3])
        K.copy_(core.view(nb, -1), vh[:nb])
        carry = K.empty(s[0], nb)
        K.copy_(carry, u[:, :nb], scale=sv, scale_axis=1)
        cores[i] = core
        cores[i - 1] = _apply_right(cores[i - 1], carry)


# ---------------------------------------------------------------------------
# TT-SVD (tensor_train.py:1138-1247) on the device
# ---------------------------------------------------------------------------


def tt_svd(tensor, error: float = 1e-12, max_rank: Optional[int] = None,
           physical_indexes=None, ttm: bool = False) -> TensorTrain:
    """Dense tensor (numpy array or CUDA tensor) to a train by TT-SVD, as
    the reference's ``tt_svd`` (``tensor_train.py:1138-1247``): each
    unfolding (bond * modes_i, rest) is split by a device SVD, truncated by
    the tail-norm rule at ``delta = error / sqrt(ndim - 1) * ||tensor||``
    and ``U^T @ matrix`` carried to the next split.  A tensor already on the
    GPU stays there (a TTM's index pairs are interleaved by one transposing
    copy).  The result is left-orthonormal with its centre on the last core.
    """
    if isinstance(tensor, torch.Tensor):
        t = tensor.to(device="cuda", dtype=torch.float64)
    else:
        t = torch.from_numpy(np.ascontiguousarray(tensor, dtype=np.float64)).to("cuda")
    if t.dim() == 1 and physical_indexes is None:
        raise AmbiguousFormat("For 1 dimensional tensor physical indexes need to be provided")
    if max_rank is not None and max_rank <= 0:
        raise ValueError("max_rank must be a positive integer.")
    if physical_indexes is not None:
        if ttm:
            d = len(physical_indexes)
            perm = tuple(int(v) for v in np.arange(2 * d).reshape(2, d).T.flatten())
            t = t.permute(*perm).contiguous()
            phys = [tuple(int(x) for x in pair) for pair in physical_indexes]
            t = t.reshape([x for pair in phys for x in pair])
        else:
            phys = [(int(x), 1) for x in physical_indexes]
            t = t.reshape([p[0] for p in phys])
    else:
        if ttm:
            raise AmbiguousFormat("For Tensor Train Matrix type physical indexes is needed")
        phys = [(int(x), 1) for x in t.shape]
    t = t.contiguous()
    nrm = K.empty(1)
    K.norm_into(nrm, t.reshape(-1))
    delta = error / math.sqrt(t.dim() - 1) * float(nrm.item()) if t.dim() > 1 else 0.0
    if len(phys) == 1:
        return TensorTrain._wrap([t.reshape((1,) + phys[0] + (1,))], orth_center=0)
    cores: List[torch.Tensor] = []
    bond, cur = 1, t.reshape(-1)
    for i in range(len(phys) - 1):
        rows = bond * phys[i][0] * phys[i][1]
        matrix = cur.view(rows, -1)
        u, sv, _ = K.svd(matrix)
        nb = _svd_rank(sv, delta, max_rank)
        core = K.empty(rows, nb)
        K.copy_(core, u[:, :nb])
        cores.append(core.view((bond,) + phys[i] + (nb,)))
        c = K.matmul(core.t(), matrix)
        if i == len(phys) - 2:
            cores.append(c.view((nb,) + phys[i + 1] + (1,)))
        else:
            bond, cur = nb, c.reshape(-1)
    return TensorTrain._wrap(cores, orth_center=len(cores) - 1)


# ---------------------------------------------------------------------------
# constructors (tensor_train.py:1250-1387), host-generated and uploaded
# ---------------------------------------------------------------------------


def _ranks(n: int, ranks) -> List[int]:
    if isinstance(ranks, list):
        return ranks
    return [1] + [int(ranks)] * (n - 1) + [1]


def _mode_pairs(physical_indexes):
    if isinstance(physical_indexes[0], (int, np.integer)):
        return [(int(p), 1) for p in physical_indexes]
    return [(int(a), int(b)) for a, b in physical_indexes]


def ones(physical_indexes, ranks=1) -> TensorTrain:
    if len(physical_indexes) < 2:
        raise WrongTTFormat("Tensor train must have at least two cores.")
    r = _ranks(len(physical_indexes), ranks)
    modes = _mode_pairs(physical_indexes)
    return TensorTrain([np.ones((r[i], modes[i][0], modes[i][1], r[i + 1]))
                        for i in range(len(modes))])


def zeros(physical_indexes, ranks=1) -> TensorTrain:
    if len(physical_indexes) < 2:
        raise WrongTTFormat("Tensor train must have at least two cores.")
    r = _ranks(len(physical_indexes), ranks)
    modes = _mode_pairs(physical_indexes)
    return TensorTrain([np.zeros((r[i], modes[i][0], modes[i][1], r[i + 1]))
                        for i in range(len(modes))])


def eye(physical_indexes) -> TensorTrain:
    if len(physical_indexes) < 2:
        raise WrongTTFormat("Tensor train must have at least two cores.")
    return TensorTrain([np.eye(p).reshape(1, p, p, 1) for p in physical_indexes])


def canonical_cores(physical_indexes, max_rank: int) -> Tuple[List[np.ndarray], int]:
    """Host cores of ``canonical_tt`` and its orthogonality centre
    (``tensor_train.py:1390-1446``): products of canonical basis vectors,
    bond k = min(max_rank, states left of the cut, states right of it); the
    first half of the cores is left-orthogonal (the identity on the
    (bond, mode) -> bond unfolding), the rest right-orthogonal, and for an
    odd number of cores the middle one is left-orthogonal."""
    dims = [int(p) for p in physical_indexes]
    d = len(dims)
    if d < 2:
        raise WrongTTFormat("Tensor train must have at least two cores.")
    bonds = [1] * (d + 1)
    for k in range(1, d):
        bonds[k] = min(max_rank, math.prod(dims[:k]), math.prod(dims[k:]))
    half = d // 2
    cores = []
    for i, n in enumerate(dims):
        if i < half + d % 2:  # left-orthogonal, the middle core of an odd train included
            m = np.eye(bonds[i] * n, bonds[i + 1])
        else:
            m = np.eye(bonds[i], n * bonds[i + 1])
        cores.append(m.reshape(bonds[i], n, 1, bonds[i + 1]))
    return cores, (half if d % 2 else half - 1)


def canonical_tt(physical_indexes, max_rank: int) -> TensorTrain:
    """Full-rank train of canonical basis products, built on the host and
    uploaded (``tensor_train.py:1390-1446``)."""
    cores, center = canonical_cores(physical_indexes, max_rank)
    return TensorTrain(cores, orth_center=center)


def rand(physical_indexes, ranks=1, seed=None) -> TensorTrain:
    """Uniform [0, 1) cores from ``np.random.default_rng(seed)``, drawn core
    by core exactly as the reference does, then uploaded."""
    if len(physical_indexes) < 2:
        raise WrongTTFormat("Tensor train must have at least two cores.")
    rng = np.random.default_rng(seed)
    r = _ranks(len(physical_indexes), ranks)
    modes = _mode_pairs(physical_indexes)
    return TensorTrain([rng.random((r[i], modes[i][0], modes[i][1], r[i + 1]))
                        for i in range(len(modes))])
