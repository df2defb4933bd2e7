"""Many AMEn solves in one persistent launch (``ttb_amen_persistent``).

Each request becomes one thread block that runs the whole solve on the
device (``csrc/ttb_amen.cu``).  The host packs every request's operator,
right-hand side, initial guess and random residual start into a few large
buffers (one host-to-device copy), builds the task table, launches once and
reads back the bonds, stop reasons and residual histories.  A solve whose
bonds outgrow the slot capacity ``rmax`` is re-run with a larger one.

Argument semantics, validation and the ``SolverInfo`` produced are those of
``amen`` (``ttnumpy/solvers/amen.py:395-725``): direct local solves up to
``direct_solve_size`` unknowns, MINRES (``symmetric=True``) or restarted
GMRES beyond.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from . import kernels as K
from . import tensor_train
from ._lib import check
from .solvers.common import (
    LocalSolver,
    SolverInfo,
    StopReason,
    TruncationMode,
    _SolverSettings,
)
from .tensor_train import TensorTrain

P, I, L, D = C.c_void_p, C.c_int, C.c_longlong, C.c_double


Task = _lib.AmenTask


def _lib_handle():
    return K.lib()


def _host_cores(t) -> List[np.ndarray]:
    if isinstance(t, TensorTrain):
        return t.to_numpy()
    return [np.asarray(c, dtype=np.float64).reshape(c.shape if c.ndim == 4 else
                                                    (c.shape[0], c.shape[1], 1, c.shape[2]))
            for c in t]


def _orth(t) -> Optional[int]:
    return t.orth_center if isinstance(t, TensorTrain) else None


STATUS = {0: "ok", -1: "singular local system", -3: "slab too small", -4: "rank above rmax",
          -5: "unsupported settings", -6: "time limit", -7: "tensor-core pipeline gave up"}


@dataclass
class Result:
    x: Optional[TensorTrain]
    info: SolverInfo
    status: int
    device_ms: float = 0.0  # the block's run time on the device for this solve
    flops: float = 0.0      # FLOPs of its float64 dense and sparse products
    flops_tc: float = 0.0   # FLOPs of its 3xTF32 tensor-core products (mixed precision)
    refine: int = 0         # float64 refinement steps of its local solves (mixed precision)


class _Prepared:
    """One request's host data and resolved settings."""

    def __init__(self, A, b, x0, kwargs):
        kw = dict(kwargs)
        kick = kw.pop("kickrank", 4)
        eth = kw.pop("error_threshold", 1e-7)
        max_rank = kw.pop("max_rank", None)
        damp = kw.pop("residual_damp", 2.0)
        seed = kw.pop("seed", None)
        return_info = kw.pop("return_info", True)
        kw.pop("inplace", None)
        # persistent-engine option (not an argument of the reference's amen):
        # "fp64", or "mixed" for 3xTF32 inner solves with float64 refinement
        precision = kw.pop("precision", "fp64")
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
        self.precision = precision
        if kick <= 0:
            raise ValueError(f"kickrank must be a positive integer, got {kick}")
        if max_rank is not None and max_rank <= 0:
            raise ValueError(f"max_rank must be a positive integer, got {max_rank}")
        if damp < 1.0:
            raise ValueError(f"residual_damp must be >= 1, got {damp}")
        self.A = _host_cores(A)
        self.b = _host_cores(b)
        d = len(self.A)
        st = _SolverSettings.resolve(
            max_sweeps=kw.pop("max_sweeps", 1), residual_tol=kw.pop("residual_tol", None),
            stagnation_factor=kw.pop("stagnation_factor", "auto"),
            local_solver=kw.pop("local_solver", "auto"), symmetric=kw.pop("symmetric", False),
            direct_solve_size=kw.pop("direct_solve_size", 1000), return_info=return_info,
            local_rtol=kw.pop("local_rtol", None),
            allow_dense_fallback=kw.pop("allow_dense_fallback", False),
            truncation_steps=max(2 * (d - 1), 1))
        if kw:
            raise TypeError(f"unexpected arguments {sorted(kw)}")
        if st.allow_dense_fallback:
            raise ValueError("the persistent path has no dense fallback for local solves")
        modes = [c.shape[1] for c in self.b]
        if [c.shape[1] for c in self.A] != modes or [c.shape[2] for c in self.A] != modes:
            raise tensor_train.DimensionMismatch("operator and right-hand side modes differ")
        if x0 is None:
            ranks = [c.shape[0] for c in self.b] + [1]
            self.x0 = [np.ones((ranks[i], modes[i], 1, ranks[i + 1])) for i in range(d)]
            self.x0_oc = -1
        else:
            self.x0 = _host_cores(x0)
            oc = _orth(x0)
            self.x0_oc = -1 if oc is None else oc
        rng = np.random.default_rng(seed)
        zr = [1] + [kick] * (d - 1) + [1]
        self.z0 = [rng.random((zr[i], modes[i], 1, zr[i + 1])) for i in range(d)]
        self.b_oc = _orth(b)
        self.st, self.kick, self.eth, self.max_rank, self.damp = st, kick, eth, max_rank, damp
        self.d = d
        self.modes = modes

    def packed(self) -> np.ndarray:
        """Operator, right-hand side, initial guess and residual start, core
        after core, as one float64 vector (the layout a task reads)."""
        return np.concatenate([c.reshape(-1) for cores in (self.A, self.b, self.x0, self.z0)
                               for c in cores])

    def offsets(self) -> np.ndarray:
        """Start of every core in :meth:`packed` (A, b, x0, z0 cores in order)."""
        sizes = [c.size for cores in (self.A, self.b, self.x0, self.z0) for c in cores]
        return np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)

    def resident(self):
        """This request's inputs on the device (uploaded on the first call
        and kept): (packed cores, their offsets)."""
        if getattr(self, "_dev", None) is None:
            host = torch.from_numpy(self.packed()).pin_memory()
            self._dev = (host.to("cuda", non_blocking=True),
                         torch.from_numpy(self.offsets()).to("cuda", non_blocking=True))
        return self._dev

    def drop_resident(self) -> None:
        self._dev = None

    def dims(self) -> np.ndarray:
        d = self.d
        R = [c.shape[0] for c in self.A] + [1]
        rb = [c.shape[0] for c in self.b] + [1]
        xb = [c.shape[0] for c in self.x0] + [1]
        zb = [c.shape[0] for c in self.z0] + [1]
        return np.array(self.modes + R + rb + xb + zb, dtype=np.int32)


def slab_doubles(p: "_Prepared", rmax: int) -> int:
    """Device work area (doubles) of one request at slot capacity ``rmax``:
    the kernel's own bound (``ttb_amen_slab_doubles``), rounded up to 64."""
    dh = p.dims()
    arr = (C.c_int * len(dh))(*dh.tolist())
    size = _lib_handle().ttb_amen_slab_doubles(p.d, arr, p.kick, rmax,
                                               int(min(p.st.direct_solve_size, 1 << 30)))
    if size < 0:
        raise ValueError("train too long for the persistent path")
    return (size + 63) // 64 * 64


class PersistentBatch:
    """Requests packed on the device for the persistent kernel.

    Construction packs the inputs (one host-to-device copy), sizes and
    allocates the slabs and uploads the task table; :meth:`run` launches the
    kernel and returns the results.  The inputs are read-only to the kernel,
    so a batch can be run again.
    """

    def __init__(self, preps: List["_Prepared"], rmax: int, debug: bool = False,
                 time_limit: Optional[float] = None, resident: bool = False, cluster: int = 1):
        lib = _lib_handle()
        self.preps, self.rmax = preps, rmax
        self.cluster = max(1, int(cluster))  # thread blocks per solve
        n = len(preps)
        # inputs: per request already on the device (``resident``: uploaded
        # beforehand by _Prepared.resident), or packed here into one buffer
        # and copied from host memory
        if resident:
            devs = [p.resident() for p in preps]
            in_ptr = [d[0].data_ptr() for d in devs]
            off_ptr = [d[1].data_ptr() for d in devs]
            self.h2d_bytes = 0
            self.dev_in = self.dev_off = None
            self._resident = devs  # keeps the buffers alive with the batch
        else:
            host = np.concatenate([p.packed() for p in preps])
            offs = []
            pos = 0
            for p in preps:
                offs.append(p.offsets() + pos)
                pos += sum(c.size for cores in (p.A, p.b, p.x0, p.z0) for c in cores)
            self.h2d_bytes = host.nbytes
            self.dev_in = torch.from_numpy(host).pin_memory().to("cuda", non_blocking=True)
            self.dev_off = torch.from_numpy(np.concatenate(offs)).to("cuda")
            in_ptr = [self.dev_in.data_ptr()] * n
            off_ptr = []
            opos = 0
            for p in preps:
                off_ptr.append(self.dev_off.data_ptr() + 8 * opos)
                opos += 4 * p.d
            self._resident = None
        dims_host = [p.dims() for p in preps]
        dim_pos = np.cumsum([0] + [len(x) for x in dims_host])
        self.dev_dims = torch.from_numpy(np.concatenate(dims_host)).to("cuda")
        sizes = [slab_doubles(p, rmax) for p in preps]
        self.slab_pos = np.cumsum([0] + sizes)
        self.slabs = torch.empty(int(self.slab_pos[-1]), dtype=torch.float64, device="cuda")
        self.dmax = max(p.d for p in preps)
        smax = max(max(p.st.max_sweeps for p in preps), 1)
        self.resid = torch.zeros(n, 2 * smax + 16, dtype=torch.float64, device="cuda")
        self.result = torch.zeros(n, 6 + self.dmax, dtype=torch.int32, device="cuda")
        self.xoff = torch.zeros(n, self.dmax, dtype=torch.int64, device="cuda")
        tasks = (Task * n)()
        # blocks start in task order: longest solves first (estimated cost)
        self.order = sorted(range(n), key=lambda i: -_cost(preps[i]))
        slot = {i: j for j, i in enumerate(self.order)}
        for i, p in enumerate(preps):
            t = tasks[slot[i]]
            t.A = t.b = t.x0 = t.z0 = in_ptr[i]
            t.A_off, t.b_off, t.x0_off, t.z0_off = [off_ptr[i] + 8 * j * p.d for j in range(4)]
            t.dims = self.dev_dims.data_ptr() + 4 * int(dim_pos[i])
            t.slab = self.slabs.data_ptr() + 8 * int(self.slab_pos[i])
            t.slab_doubles = sizes[i]
            t.residuals = self.resid[i].data_ptr()
            t.result = self.result[i].data_ptr()
            t.x_offsets = self.xoff[i].data_ptr()
            st = p.st
            t.d, t.kickrank = p.d, p.kick
            t.max_rank = p.max_rank or 0
            t.max_sweeps = st.max_sweeps
            t.direct_solve_size = (int(min(st.direct_solve_size, 1 << 30))
                                   if st.iterative_solver is not None else (1 << 30))
            t.track_residual = int(st.track_residual)
            t.residual_mode = int(st.truncation_mode is TruncationMode.RESIDUAL)
            t.stagnation_on = int(st.stagnation_factor is not None)
            t.x0_orth_center = p.x0_oc
            t.b_orth_center = -1 if p.b_oc is None else p.b_oc
            t.residual_tol = st.residual_tol or 0.0
            t.error_threshold = p.eth
            t.residual_damp = p.damp
            t.stagnation_factor = st.stagnation_factor or 0.0
            # MINRES (symmetric) or restarted GMRES local solves at local_rtol
            t.local_rtol = st.local_rtol or 0.0
            t.local_gmres = int(st.iterative_solver is LocalSolver.GMRES)
            t.truncation_tol = st.truncation_tol or 0.0
            t.debug = int(debug)
            t.time_limit_ns = int(time_limit * 1e9) if time_limit else 0
            t.precision = 1 if p.precision == "mixed" else 0
        raw = np.frombuffer(bytes(tasks), dtype=np.uint8)
        self.dev_tasks = torch.from_numpy(raw.copy()).to("cuda")

    def launch(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        """Queue the kernel on ``stream`` (asynchronous)."""
        s = stream or torch.cuda.current_stream()
        if self.cluster > 1:
            check(K.lib().ttb_amen_persistent_cluster(
                C.c_void_p(self.dev_tasks.data_ptr()), len(self.preps), self.rmax, self.cluster,
                C.c_void_p(s.cuda_stream)), "ttb_amen_persistent_cluster")
            return
        check(K.lib().ttb_amen_persistent(C.c_void_p(self.dev_tasks.data_ptr()),
                                          len(self.preps), self.rmax, C.c_void_p(s.cuda_stream)),
              "ttb_amen_persistent")

    def capture(self) -> torch.cuda.CUDAGraph:
        """The batch's launch captured in a CUDA graph: ``graph.replay()``
        solves every request of the batch again (the kernel only reads the
        inputs, which may be updated in place between replays, and rewrites
        every result), then :meth:`collect` reads the results.  Run the batch
        once first, so that the one-time set-up of the library happens
        outside the capture."""
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.launch()
        return graph

    def gemm_flops(self) -> float:
        """FP64 FLOPs of the dense products of the last launch, all blocks."""
        resid_h = self.resid.cpu().numpy()
        return float(sum(resid_h[i, 2 * p.st.max_sweeps] for i, p in enumerate(self.preps)))

    PHASES = ("env", "solve", "zcore", "trunc_enrich", "gemm", "resid", "init")

    def breakdown(self):
        """Per solve: operator applications and SM cycles per phase of the
        last launch (environment updates, local solves, residual cores,
        truncation with enrichment, residual checks, set-up) and, under
        "gemm", the cycles of all dense products (inside those phases)."""
        resid_h = self.resid.cpu().numpy()
        out = []
        for i, p in enumerate(self.preps):
            base = 2 * p.st.max_sweeps
            row = {"applies": int(resid_h[i, base + 1]), "flops": float(resid_h[i, base])}
            for j, name in enumerate(self.PHASES):
                row[name] = float(resid_h[i, base + 2 + j])
            row["check"] = float(resid_h[i, base + 9])
            row["check_qr"] = float(resid_h[i, base + 12])
            row["n_qr2"] = int(resid_h[i, base + 13])
            out.append(row)
        return out

    def latencies_ms(self) -> List[float]:
        """Per solve of the last launch: milliseconds from the first block's
        start to this solve's end (device global timer)."""
        resid_h = self.resid.cpu().numpy()
        starts, ends = [], []
        for i, p in enumerate(self.preps):
            base = 2 * p.st.max_sweeps
            starts.append(resid_h[i, base + 10])
            ends.append(resid_h[i, base + 11])
        t0 = min(starts)
        return [(e - t0) * 1e-6 for e in ends]

    def collect(self) -> List[Result]:
        """Results of the last launch (synchronises with it)."""
        res_h = self.result.cpu().numpy()
        resid_h = self.resid.cpu().numpy()
        xoff_h = self.xoff.cpu().numpy()
        out = []
        for i, p in enumerate(self.preps):
            status = int(res_h[i, 0])
            info = SolverInfo()
            hb = 2 * p.st.max_sweeps
            dev_ms = (resid_h[i, hb + 11] - resid_h[i, hb + 10]) * 1e-6
            flops = float(resid_h[i, hb])
            extra = dict(flops_tc=float(resid_h[i, hb + 14]), refine=int(resid_h[i, hb + 15]))
            if status == -6:  # time limit: the sweeps completed before it
                info.num_sweeps_run = int(res_h[i, 1])
                info.residuals = [float(v) for v in resid_h[i, :info.num_sweeps_run]]
            if status != 0:
                out.append(Result(None, info, status, dev_ms, flops, **extra))
                continue
            sweeps = int(res_h[i, 1])
            info.num_sweeps_run = sweeps
            info.stop_reason = [StopReason.CONVERGED, StopReason.STAGNATED,
                                StopReason.MAX_SWEEPS][int(res_h[i, 2])]
            info.local_solves = int(res_h[i, 3])
            info.local_inexact = int(res_h[i, 4])
            if p.st.track_residual:
                info.residuals = [float(v) for v in resid_h[i, :sweeps]]
            ms = p.st.max_sweeps
            info.max_bonds = [int(v) for v in resid_h[i, ms:ms + sweeps]]
            bonds = [int(v) for v in res_h[i, 5:6 + p.d]]
            base = int(self.slab_pos[i])
            cores = []
            for k in range(p.d):
                o = base + int(xoff_h[i, k])
                size = bonds[k] * p.modes[k] * bonds[k + 1]
                cores.append(self.slabs[o:o + size].view(bonds[k], p.modes[k], 1,
                                                         bonds[k + 1]).clone())
            out.append(Result(TensorTrain._wrap(cores, orth_center=0), info, status, dev_ms,
                              flops, **extra))
        return out

    def run(self, stream: Optional[torch.cuda.Stream] = None) -> List[Result]:
        self.launch(stream)
        return self.collect()

    @property
    def device_bytes(self) -> int:
        """Device memory the batch holds: inputs, slabs and result tables."""
        return sum(t.numel() * t.element_size() for t in
                   (self.dev_in, self.dev_off, self.dev_dims, self.slabs, self.resid,
                    self.result, self.xoff) if t is not None)

    def release(self) -> None:
        """Drop the device buffers (results already collected stay valid:
        their cores were cloned out of the slabs)."""
        self.dev_in = self.dev_off = self.dev_dims = self.slabs = None
        self.resid = self.result = self.xoff = None
        self._resident = None


def initial_rmax(p: "_Prepared") -> int:
    """Slot capacity a request starts with: bonds of solutions on mode-2
    (QTT) trains stay far below 32, those of mode sizes up to 32 below 64,
    and larger modes reach the 70s at residual 1e-8, where starting at 64
    would cost a full re-run at twice the capacity."""
    n = max(p.modes)
    if n <= 4:
        return 32
    return 64 if n < 64 else 96


def cluster_size(p: "_Prepared") -> int:
    """Thread blocks a request's solve runs on: four for mode sizes of 64
    and up, whose local operator applications are the large products a
    cluster shares out (tens of seconds of work on one SM), one otherwise."""
    return 4 if max(p.modes) >= 64 else 1


def _cost(p: "_Prepared") -> float:
    """Relative cost estimate of a solve for the launch order: the local
    apply grows like n^3 R^2 at the bonds such problems reach, times d."""
    n = max(p.modes)
    R = max(c.shape[0] for c in p.A)
    return float(p.d) * n ** 3 * R ** 2


def prepare(requests: Sequence) -> List["_Prepared"]:
    """Validate and resolve ``[(A, b, x0, kwargs), ...]`` on the host."""
    return [_Prepared(A, b, x0, kw) for A, b, x0, kw in requests]


def amen_persistent(requests: Sequence, rmax: int = 64, max_rmax: int = 256,
                    stream: Optional[torch.cuda.Stream] = None,
                    time_limit: Optional[float] = None, cluster: int = 1) -> List[Result]:
    """Solve ``[(A, b, x0, kwargs), ...]`` in one persistent launch; solves
    whose bonds outgrow ``rmax`` are re-run with twice the capacity.  With
    ``time_limit`` (seconds) a solve still running after that long on the
    device stops with status -6; with ``cluster`` > 1 every solve runs on a
    cluster of that many thread blocks (same results)."""
    K.device_ok()
    preps = prepare(requests)
    results: List[Optional[Result]] = [None] * len(preps)
    todo = list(range(len(preps)))
    while todo:
        out = PersistentBatch([preps[i] for i in todo], rmax, time_limit=time_limit,
                              cluster=cluster).run(stream)
        retry = []
        for i, res in zip(todo, out):
            if res.status == -4 and rmax < max_rmax:
                retry.append(i)
            else:
                results[i] = res
        todo = retry
        rmax = min(2 * rmax, max_rmax)
    return results
