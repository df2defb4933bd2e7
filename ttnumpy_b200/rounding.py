"""Batched TT rounding of sums of pairs of trains on the GPU.

``round_sum_batch`` rounds ``p_i + q_i`` for many pairs in one launch of the
fused ``ttb_round_batch`` kernel (one thread block per pair: left QR sweep of
the block-diagonal sum, then the right SVD sweep with the tail-norm rule),
which is ``(p + q).truncate(error, max_rank)`` of the reference
(``ttnumpy/tensor_train.py:254-322, 852-940``) for every pair.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from . import kernels as K
from ._lib import check
from .tensor_train import TensorTrain

SLOT = 16384  # TTB_ROUND_SLOT


@dataclass
class PackedTrains:
    """Many trains with the same modes and bonds, packed core by core:
    train i's core k starts at ``data[i, offsets[k]]``."""

    data: torch.Tensor  # (count, stride) float64
    offsets: List[int]
    bonds: List[int]
    modes: List[int]

    @property
    def count(self) -> int:
        return self.data.shape[0]

    @classmethod
    def from_numpy(cls, trains: Sequence[Sequence[np.ndarray]]) -> "PackedTrains":
        first = trains[0]
        sizes = [int(np.prod(c.shape)) for c in first]
        offsets = list(np.cumsum([0] + sizes[:-1]))
        host = np.empty((len(trains), sum(sizes)), dtype=np.float64)
        for i, t in enumerate(trains):
            host[i] = np.concatenate([np.asarray(c, dtype=np.float64).reshape(-1) for c in t])
        bonds = [c.shape[0] for c in first] + [1]
        modes = [c.shape[1] for c in first]
        return cls(torch.from_numpy(host).to("cuda"), [int(o) for o in offsets], bonds, modes)


@dataclass
class RoundResult:
    out: torch.Tensor      # (pairs, d * SLOT)
    bonds: torch.Tensor    # (pairs, d + 1) int32
    status: torch.Tensor   # (pairs,) int32
    modes: List[int]

    def train(self, i: int) -> TensorTrain:
        bonds = self.bonds[i].tolist()
        cores = []
        for k, n in enumerate(self.modes):
            size = bonds[k] * n * bonds[k + 1]
            cores.append(self.out[i, k * SLOT:k * SLOT + size].reshape(bonds[k], n, 1,
                                                                        bonds[k + 1]).clone())
        return TensorTrain._wrap(cores, orth_center=0)


class RoundPlan:
    """Device buffers for repeated batched rounding of one shape."""

    def __init__(self, pairs: int, d: int, modes: Sequence[int], p_bonds, q_bonds, p_offsets,
                 q_offsets):
        K.device_ok()
        self.pairs, self.d = pairs, d
        self.modes = list(modes)
        for k in range(d):
            rin = 1 if k == 0 else p_bonds[k] + q_bonds[k]
            rout = 1 if k == d - 1 else p_bonds[k + 1] + q_bonds[k + 1]
            if max(rin, rout) > 64 or modes[k] * max(rin, rout) > 256:
                raise ValueError("batched rounding needs bonds <= 64 and mode * bond <= 256")
        lib = K.lib()
        self.work_stride = int(lib.ttb_round_work_doubles(d, max(modes), 64))
        dev = "cuda"
        self.p_off = torch.tensor(p_offsets, dtype=torch.int64, device=dev)
        self.q_off = torch.tensor(q_offsets, dtype=torch.int64, device=dev)
        self.p_bonds = torch.tensor(p_bonds, dtype=torch.int32, device=dev)
        self.q_bonds = torch.tensor(q_bonds, dtype=torch.int32, device=dev)
        self.modes_d = torch.tensor(self.modes, dtype=torch.int32, device=dev)
        self.out = torch.empty(pairs, d * SLOT, dtype=torch.float64, device=dev)
        self.out_off = torch.empty(pairs * d, dtype=torch.int64, device=dev)
        self.bonds = torch.empty(pairs, d + 1, dtype=torch.int32, device=dev)
        self.status = torch.empty(pairs, dtype=torch.int32, device=dev)
        self.work = torch.empty(pairs * self.work_stride, dtype=torch.float64, device=dev)

    def run(self, p: torch.Tensor, q: torch.Tensor, error: float, max_rank: Optional[int]):
        desc = _lib.Round(p.data_ptr(), q.data_ptr(), self.p_off.data_ptr(),
                          self.q_off.data_ptr(), self.p_bonds.data_ptr(), self.q_bonds.data_ptr(),
                          self.modes_d.data_ptr(), p.stride(0), q.stride(0), self.out.data_ptr(),
                          self.out.stride(0), self.out_off.data_ptr(), self.bonds.data_ptr(),
                          self.work.data_ptr(), self.work_stride, self.status.data_ptr(),
                          self.pairs, self.d, float(error), int(max_rank or 0))
        check(K.lib().ttb_round_batch(C.byref(desc), K.stream()), "ttb_round_batch")
        return RoundResult(self.out, self.bonds, self.status, self.modes)


def round_sum_batch(p: PackedTrains, q: PackedTrains, error: float = 0.0,
                    max_rank: Optional[int] = None, plan: Optional[RoundPlan] = None
                    ) -> RoundResult:
    """Round ``p_i + q_i`` for every pair i (``truncate(error, max_rank)``)."""
    if p.count != q.count or p.modes != q.modes:
        raise ValueError("pairs must share count and modes")
    if plan is None:
        plan = RoundPlan(p.count, len(p.modes), p.modes, p.bonds, q.bonds, p.offsets, q.offsets)
    return plan.run(p.data, q.data, error, max_rank)
