"""Device orchestration: node sets, operand folds and bilinear forms on the GPU.

A *job* is a list of (cont_i, cont_f) pairs sharing one grid, one potential
set and one (bound_i, bound_f) transition, i.e. the work of one energy point of
the reference's driver (``driver.py:907-1029``) or one ejected energy of its
ionization loop (``ionization.py:526-608``). The host plans each pair
(``plan.py``), the device builds the quadrature operators of every distinct
node set once, folds all operands, and evaluates every bilinear form in one
launch; the L=0 corrections and the outer tails are added in FP64 on the host.
"""
from __future__ import annotations

import collections
import ctypes
from dataclasses import dataclass, field
import functools
import hashlib
from itertools import repeat
import operator
import threading
from typing import Dict, List, NamedTuple, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .plan import (GridInfo, NodeSetKey, NodeSetPlan, OVERLAP_TOL, adaptive_dphi, cc_reference, diag_scale,
                   idx_limit, is_excitation, multipole_moments, plan_nodeset, safe_float, tail_limits)

ENGINES = ("dense", "semisep", "tc_bf16x3", "tc_bf16x6")
TC_TERMS = {"tc_bf16x3": 2, "tc_bf16x6": 3}


def tc_route_fraction() -> float:
    """Routing bound of the split-BF16 engines: an exchange form whose |I_L| exceeds this fraction of
    the largest |I_L| of its transition at any L is recomputed in FP64 (DWBA_B200_TC_ROUTE; <= 0
    disables the guard)."""
    import os
    try:
        return float(os.environ.get("DWBA_B200_TC_ROUTE", "0.1"))
    except ValueError:
        return 0.1


class TCGuard:
    """Accuracy guard of the split-BF16 exchange forms of one launch.

    The tensor-core forms carry an error of about 1e-6 of their scale |a|^T K_L |b| (FP32 values of
    K_L and FP32 accumulation), independent of the bf16 split. A transition's cross section is
    dominated by its largest integrals, so the guard recomputes in FP64 the forms whose |I_L| (from
    the tensor-core pass) exceeds ``theta`` times the largest |I_L| of their transition (``groups``:
    the transition of each form) at some L -- typically a few percent of the forms -- and keeps the
    tensor-core values of the rest, whose errors are small against the dominant integrals. The
    flagged forms are evaluated by the exact semiseparable form (the others masked to empty forms,
    which cost nothing) and merged into the result. Device-side only, no host sync, so it is
    captured in CUDA graphs with the rest of the launch sequence."""

    def __init__(self, forms_d: torch.Tensor, n: int, nl: int, dev, groups: np.ndarray, theta: float):
        self.n, self.theta, self.nl = n, theta, nl
        self.forms_d = forms_d
        g = np.ascontiguousarray(groups, dtype=np.int64)
        self.n_groups = int(g.max()) + 1 if len(g) else 0
        self.gidx = _dev(g, dev)
        self.gidx2 = self.gidx[:, None].expand(n, nl)
        self.desc32 = forms_d.view(torch.int32).view(n, _lib.FORM_DTYPE.itemsize // 4)
        self.masked = torch.empty_like(forms_d)
        self.masked32 = self.masked.view(torch.int32).view(n, _lib.FORM_DTYPE.itemsize // 4)
        self.mag = torch.empty((n, nl), dtype=torch.float64, device=dev)
        self.gmax = torch.empty((max(1, self.n_groups), nl), dtype=torch.float64, device=dev)
        self.exact = torch.empty((n, nl), dtype=torch.float64, device=dev)
        self.over = torch.empty((n, nl), dtype=torch.bool, device=dev)
        self.flag = torch.zeros(n, dtype=torch.bool, device=dev)
        self.rows = _lib.FORM_DTYPE.fields["n_rows"][1] // 4  # int32 column of n_rows (n_cols follows)

    def launch(self, lib, L_max: int, ds: np.ndarray, r_min: float, r_max: float, out: torch.Tensor) -> None:
        if self.theta <= 0 or self.n == 0:
            return
        st = _stream()
        torch.abs(out, out=self.mag)
        self.gmax.zero_()
        self.gmax.scatter_reduce_(0, self.gidx2, self.mag, reduce="amax", include_self=True)
        torch.gt(self.mag, self.theta * self.gmax.index_select(0, self.gidx), out=self.over)
        torch.any(self.over, dim=1, out=self.flag)
        self.masked.copy_(self.forms_d)
        keep = self.flag.to(torch.int32)
        c = self.rows
        self.masked32[:, c:c + 2] = self.desc32[:, c:c + 2] * keep[:, None]
        _lib.check(lib.dwba_bilinear_semisep_fp64(_ptr(self.masked), self.n, L_max, ds.ctypes.data, r_min, r_max,
                                                  _ptr(self.exact), st), "dwba_bilinear_semisep_fp64")
        out.copy_(torch.where(self.flag[:, None], self.exact, out))

    def n_routed(self) -> int:
        return int(self.flag.sum().item()) if self.theta > 0 else 0


def _ptr(t: Optional[torch.Tensor]) -> int:
    return 0 if t is None else int(t.data_ptr())


def _stream() -> int:
    return int(torch.cuda.current_stream().cuda_stream)


class RingRegions:
    """Region allocator of a ring buffer whose regions are freed in allocation order: ``alloc(n)``
    returns the next region [a, b) (256-byte aligned) and the keys of the earlier regions it
    overlaps, or that a wrap leaves behind, which must be released (waited for) before [a, b) is
    written. Live regions never overlap."""

    def __init__(self, size: int):
        self.size, self.head = size, 0
        self.live: "collections.deque[Tuple[int, int, object]]" = collections.deque()

    def alloc(self, n: int, key) -> Tuple[int, int, list]:
        need = (n + 255) // 256 * 256
        if need > self.size:
            raise ValueError("region larger than the ring")
        release = []
        if self.head + need > self.size:
            while self.live and self.live[0][0] >= self.head:  # past this pass's end
                release.append(self.live.popleft()[2])
            self.head = 0
        a, b = self.head, self.head + need
        while self.live and self.live[0][0] < b and a < self.live[0][1]:
            release.append(self.live.popleft()[2])
        self.live.append((a, b, key))
        self.head = b
        return a, b, release


class _Staging:
    """A ring of page-locked host memory per device for the small arrays a call uploads
    (descriptors): an array is copied into the ring and from there to the device by a kernel on the
    current stream (``dwba_copy_from_host``), so that it neither blocks the host nor queues behind a
    large transfer on the copy engines. A region of the ring is reused only after the event recorded
    behind its copy has completed."""

    SIZE = 32 << 20
    MAX = 4 << 20  # larger arrays go through torch's pinned memory and the copy engines
    _by_device: Dict[int, "_Staging"] = {}

    def __init__(self):
        self.buf = torch.empty(self.SIZE, dtype=torch.uint8, pin_memory=True)
        self.host = self.buf.numpy()
        self.ptr = self.buf.data_ptr()
        self.regions = RingRegions(self.SIZE)
        self.lock = threading.Lock()  # callers on several host threads share the ring

    _make_lock = threading.Lock()

    @classmethod
    def get(cls, index: int) -> "_Staging":
        st = cls._by_device.get(index)
        if st is None:
            with cls._make_lock:
                st = cls._by_device.get(index)
                if st is None:
                    st = cls._by_device[index] = cls()
        return st

    def copy(self, x: np.ndarray, out: torch.Tensor) -> None:
        raw = x.reshape(-1).view(np.uint8)
        n = len(raw)
        ev = torch.cuda.Event()
        with self.lock:
            a, _, release = self.regions.alloc(n, ev)
            for old in release:
                old.synchronize()  # the earlier copy from this region must have run
            self.host[a:a + n] = raw
            _lib.check(_lib.load().dwba_copy_from_host(out.data_ptr(), self.ptr + a, n, _stream()),
                       "dwba_copy_from_host")
            ev.record()


def _dev(x: np.ndarray, device) -> torch.Tensor:
    """A host array on the device. To a GPU, a small array goes through the staging ring (copied by
    a kernel, _Staging) and a large one through pinned memory as an asynchronous copy on the current
    stream: neither blocks the host, and later changes to ``x`` do not reach the copy."""
    x = np.ascontiguousarray(x)
    t = torch.from_numpy(x)
    dev = torch.device(device)
    if dev.type != "cuda":
        return t.to(device)
    if 0 < x.nbytes <= _Staging.MAX:
        out = torch.empty_like(t, device=dev)
        _Staging.get(out.device.index).copy(x, out)
        return out
    return t.pin_memory().to(device, non_blocking=True)


class DeviceGrid:
    """Device copies of one radial grid (r, log r, Simpson weights) and its node-set cache."""

    def __init__(self, g: GridInfo, device):
        self.info = g
        self.device = device
        self.r = _dev(g.r, device)
        self.logr = torch.log(self.r)
        self.w = _dev(g.w, device)
        self.nodesets: Dict[NodeSetKey, "DeviceNodeSet"] = {}

    def nbytes(self) -> int:
        return sum(ns.nbytes for ns in self.nodesets.values()) + 3 * 8 * self.info.N


class DeviceNodeSet(NamedTuple):
    """Operators of one node set: device addresses inside ``block`` (which keeps them alive)."""
    plan: NodeSetPlan
    block: torch.Tensor
    ta_ptr: int
    bx_ptr: int
    nbytes: int

    @property
    def ta(self) -> torch.Tensor:
        return self._view(self.ta_ptr, 3 * self.plan.key.n1)

    @property
    def bx(self) -> torch.Tensor:
        return self._view(self.bx_ptr, (self.nbytes // 8) - 3 * self.plan.key.n1)

    def _view(self, ptr: int, n: int) -> torch.Tensor:
        off = (ptr - self.block.data_ptr()) // 8
        return self.block.narrow(0, off, n)


class CCTables:
    _cache: Dict[Tuple[int, str], Tuple[torch.Tensor, torch.Tensor]] = {}

    @classmethod
    def get(cls, n: int, device) -> Tuple[torch.Tensor, torch.Tensor]:
        key = (n, str(device))
        v = cls._cache.get(key)
        if v is None:
            x, w = cc_reference(n)
            v = (_dev(np.asarray(x, dtype=np.float64), device), _dev(np.asarray(w, dtype=np.float64), device))
            cls._cache[key] = v
        return v


_KEY_N1 = operator.itemgetter(1)  # NodeSetKey.n1


class NodeSetBatch:
    """Descriptors of the node sets a job uses; ``launch()`` (re)builds their banded operators.

    ``fused`` (a mask over ``plans``): sets whose operators are applied at once to their pair's
    multi-folds (``dwba_build_nodesets_folded``) instead of being stored: they get no operator
    memory, are not cached, and launch with the fold descriptors given by ``set_fused_folds``."""

    def __init__(self, dg: DeviceGrid, plans: Sequence[NodeSetPlan], n_cc: int, rebuild: bool = False,
                 fused: Optional[np.ndarray] = None):
        self.dg, self.n_cc = dg, n_cc
        dev = dg.device
        N = dg.info.N
        cache = dg.nodesets
        plans = list(plans)
        fused = np.zeros(len(plans), dtype=bool) if fused is None else np.asarray(fused, dtype=bool)
        self.fused_idx = np.nonzero(fused)[0]
        self.n_fused = len(self.fused_idx)
        self.fused_recs = None
        self.fused_folds_d = None
        self.fused_groups = [(0, 0, self.n_fused)]
        if self.n_fused:
            fp = list(map(plans.__getitem__, self.fused_idx.tolist()))
            f_key, f_nb, f_br, f_l1, f_l2 = zip(*fp)  # fields of every fused set, without a Python loop
            fr = np.zeros(self.n_fused, dtype=_lib.NODESET_DTYPE)
            fr["r"], fr["logr"] = _ptr(dg.r), _ptr(dg.logr)
            fr["n_grid"], fr["n1"] = N, list(map(_KEY_N1, f_key))
            fr["n_breaks"], fr["log1"], fr["log2"] = f_nb, f_l1, f_l2
            self._fused_breaks = f_br
            if any(map(operator.is_not, f_br, repeat(None))):
                br_len = np.array([0 if b is None else len(b) for b in self._fused_breaks], dtype=np.int64)
                self._fused_br = _dev(np.concatenate([np.asarray(b, dtype=np.float64) for b in self._fused_breaks
                                                      if b is not None]), dev)
                off = np.concatenate([[0], np.cumsum(br_len)[:-1]])
                has = br_len > 0
                fr["breaks"][has] = np.uint64(_ptr(self._fused_br)) + np.uint64(8) * off[has].astype(np.uint64)
            self.fused_recs = fr
            self.fused_recs_d = _dev(fr.view(np.uint8), dev)
            self.fccx, self.fccw = CCTables.get(n_cc, dev)
            self.fused_status = torch.zeros(1, dtype=torch.int32, device=dev)
        keep = np.nonzero(~fused)[0]
        plans = list(map(plans.__getitem__, keep.tolist()))
        cached = [cache.get(p.key) for p in plans]
        todo = plans if rebuild else [p for p, c in zip(plans, cached) if c is None]
        self.n = len(todo)
        # operator addresses of every planned set, in the plans' order (and a 0 for "no set"); the
        # fused sets have none
        self.ta_all = np.zeros(len(fused) + 1, dtype=np.uint64)
        self.bx_all = np.zeros(len(fused) + 1, dtype=np.uint64)
        self._keep = keep
        if not todo:
            self.ta_all[keep] = [c.ta_ptr for c in cached]
            self.bx_all[keep] = [c.bx_ptr for c in cached]
            return
        self.ccx, self.ccw = CCTables.get(n_cc, dev)
        n = len(todo)
        self.keep = []
        # operators of the sets not cached yet: one allocation for the batch, addresses by offset
        fresh_mask = np.array([c is None for c in cached], dtype=bool) if rebuild else np.ones(n, dtype=bool)
        n1s = np.array([p.key.n1 for p in todo], dtype=np.int64)
        sizes = np.where(fresh_mask, 3 * n1s + 5 * N, 0)
        offs = np.concatenate([[0], np.cumsum(sizes)[:-1]])
        block = torch.empty(int(sizes.sum()), dtype=torch.float64, device=dev) if fresh_mask.any() else None
        ta_p = np.zeros(n, dtype=np.uint64)
        bx_p = np.zeros(n, dtype=np.uint64)
        if block is not None:
            base = np.uint64(_ptr(block))
            ta_p[fresh_mask] = base + np.uint64(8) * offs[fresh_mask].astype(np.uint64)
            bx_p[fresh_mask] = ta_p[fresh_mask] + np.uint64(8) * (3 * n1s[fresh_mask]).astype(np.uint64)
        # Coulomb breakpoint lists (eta != 0) of every set: one upload, addresses by offset
        br_len = np.array([0 if p.breaks is None else len(p.breaks) for p in todo], dtype=np.int64)
        br_p = np.zeros(n, dtype=np.uint64)
        if br_len.any():
            br_all = _dev(np.concatenate([np.asarray(p.breaks, dtype=np.float64) for p in todo
                                          if p.breaks is not None]), dev)
            self.keep.append(br_all)
            br_off = np.concatenate([[0], np.cumsum(br_len)[:-1]])
            has = br_len > 0
            br_p[has] = np.uint64(_ptr(br_all)) + np.uint64(8) * br_off[has].astype(np.uint64)
        nb = (8 * (3 * n1s + 5 * N)).tolist()
        ta_l, bx_l = ta_p.tolist(), bx_p.tolist()
        for i, p in enumerate(todo):
            if fresh_mask[i]:
                cache[p.key] = DeviceNodeSet(p, block, ta_l[i], bx_l[i], nb[i])
        if rebuild and not fresh_mask.all():
            old = [i for i in range(n) if not fresh_mask[i]]
            ta_p[old] = [cached[i].ta_ptr for i in old]
            bx_p[old] = [cached[i].bx_ptr for i in old]
        if rebuild:
            self.ta_all[keep], self.bx_all[keep] = ta_p, bx_p
        else:
            done = {id(p): i for i, p in enumerate(todo)}
            for j, (p, c) in enumerate(zip(plans, cached)):
                k = done.get(id(p))
                self.ta_all[keep[j]], self.bx_all[keep[j]] = (ta_p[k], bx_p[k]) if k is not None else \
                    (c.ta_ptr, c.bx_ptr)
        recs = np.zeros(n, dtype=_lib.NODESET_DTYPE)
        recs["r"], recs["logr"] = _ptr(dg.r), _ptr(dg.logr)
        recs["breaks"], recs["ta"], recs["bx"] = br_p, ta_p, bx_p
        recs["n_grid"], recs["n1"] = N, n1s
        recs["n_breaks"] = np.array([p.n_breaks for p in todo], dtype=np.int32)
        recs["log1"] = np.array([int(p.log1) for p in todo], dtype=np.int32)
        recs["log2"] = np.array([int(p.log2) for p in todo], dtype=np.int32)
        self.recs = recs
        self.recs_d = _dev(recs.view(np.uint8), dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)

    def reorder_fused(self, perm: np.ndarray, groups: List[Tuple[int, int, int]]) -> None:
        """Put the fused sets in the order ``perm`` (of their current order) and launch them in
        ``groups`` (part k of a chunked wave upload, first set, end set): each group after its part
        of the waves is on the device. Call before ``set_fused_folds``, whose folds follow the new order."""
        perm = np.asarray(perm, dtype=np.int64)
        self.fused_idx = self.fused_idx[perm]
        self.fused_recs = _take(self.fused_recs, perm)
        self.fused_recs_d = _dev(self.fused_recs.view(np.uint8), self.dg.device)
        self.fused_groups = list(groups)

    def set_fused_folds(self, folds: np.ndarray) -> None:
        """The two multi-folds (T, then B) of every fused set, in the order of ``fused_idx``."""
        assert len(folds) == 2 * self.n_fused
        self.fused_folds = folds
        self.fused_folds_d = _dev(folds.view(np.uint8), self.dg.device) if len(folds) else None

    def algorithmic_bytes(self) -> float:
        """Bytes a build must move: the operators written (3 n1 + 5 N doubles per set) and the grid
        read (r and log r, 2 N doubles per set); a fused set writes no operators but reads its
        folds' functions and writes their outputs (``fold_bytes`` of its multi-folds)."""
        N = float(self.dg.info.N)
        b = 0.0
        if self.n:
            b += float(np.sum(8.0 * (3.0 * self.recs["n1"].astype(np.float64) + 7.0 * N)))
        if self.n_fused:
            b += self.n_fused * 8.0 * 2.0 * N + fused_fold_bytes(self.fused_folds)
        return b

    def launch(self, waves: Optional["WaveMatrix"] = None) -> None:
        """Stored sets first (they read only the grid), then the fused sets, which read their pair's
        waves: with ``waves``, each group of ``fused_groups`` after its part of the wave upload."""
        lib = _lib.load()
        N = self.dg.info.N
        for s0 in range(0, self.n, 65535):
            n = min(65535, self.n - s0)
            _lib.check(lib.dwba_build_nodesets(_ptr(self.recs_d) + s0 * _lib.NODESET_DTYPE.itemsize, n, N,
                                               _ptr(self.ccx), _ptr(self.ccw), self.n_cc, _ptr(self.status),
                                               _stream()), "dwba_build_nodesets")
        pending = waves is not None and waves.chunks is not None
        for k, g0, g1 in (self.fused_groups if pending else [(-1, 0, self.n_fused)]):
            if pending:
                waves.wait_chunk(k)
            for s0 in range(g0, g1, 65535):
                n = min(65535, g1 - s0)
                _lib.check(lib.dwba_build_nodesets_folded(
                    _ptr(self.fused_recs_d) + s0 * _lib.NODESET_DTYPE.itemsize,
                    _ptr(self.fused_folds_d) + 2 * s0 * _lib.FOLD_MULTI_DTYPE.itemsize, n, N, _ptr(self.fccx),
                    _ptr(self.fccw), self.n_cc, _ptr(self.fused_status), _stream()), "dwba_build_nodesets_folded")

    def check(self) -> None:
        if self.n and int(self.status.item()) != 0:
            raise _lib.DWBAError(_lib.DWBA_ERR_RANGE, "dwba_build_nodesets")
        if self.n_fused and int(self.fused_status.item()) != 0:
            raise _lib.DWBAError(_lib.DWBA_ERR_RANGE, "dwba_build_nodesets_folded")


def fused_fold_bytes(folds: np.ndarray) -> float:
    """Bytes the multi-folds of fused node sets move: each distinct function read once over its
    longest use and every output written."""
    if folds is None or not len(folds):
        return 0.0
    reads: Dict[int, float] = {}
    writes = 0.0
    for m in folds:
        n_src = float(m["n_src"])
        for p_ in [int(m["g"])] + [int(x) for x in m["f"][:m["n_f"]]]:
            if p_ and n_src > reads.get(p_, 0.0):
                reads[p_] = n_src
        writes += float(m["n_clear"]) * int(m["n_f"])
    return 8.0 * (sum(reads.values()) + writes)


@dataclass
class PairPlan:
    n1: int
    osc: bool
    nodeset: Optional[NodeSetPlan]
    corr_dir: float = 0.0
    corr_ex: float = 0.0
    tail: Optional[np.ndarray] = None


@dataclass
class Transition:
    """One (bound_i, bound_f) pair: u_f is a bound orbital (excitation) or an ejected wave (ionization)."""
    u_i: np.ndarray
    u_f: np.ndarray
    excitation: bool


@dataclass
class Job:
    """Work sharing one grid and potentials: every transition with every (cont_i, cont_f) pair.

    One energy point of the reference's excitation driver is one transition with all its
    (l_i, l_f) pairs (``driver.py:907-1029``); one ejected energy of its ionization loop is a
    set of transitions (one per ejected wave) (``ionization.py:526-608``).
    """
    grid: GridInfo
    V_core: np.ndarray
    U_i: np.ndarray
    U_f: Optional[np.ndarray]
    transitions: List[Transition]
    pairs: List[Tuple[object, object]]
    L_max: int
    use_oscillatory_quadrature: bool = True
    oscillatory_method: str = "advanced"
    CC_nodes: int = 5
    phase_increment: float = 1.5708
    min_grid_fraction: float = 0.10
    k_threshold: float = 0.5
    tails_on_device: bool = True
    # tails per unit multipole moment (t_L / M_L) instead of the tails themselves, for callers that
    # apply the moments themselves (the differentiable path)
    tails_per_unit_moment: bool = False


def _wave_scalars(w):
    return (float(w.k_au), int(w.l), int(getattr(w, "idx_match", -1)), float(getattr(w, "eta", 0.0)),
            float(getattr(w, "phase_shift", 0.0)), float(getattr(w, "sigma_l", 0.0)))


def _packed_pair_arrays(scal: np.ndarray):
    """_pair_arrays from the packed scalars (P x 12: k, l, idx_match, eta, phase_shift, sigma_l of
    cont_i then cont_f)."""
    a = scal
    out = dict(k_i=a[:, 0], l_i=a[:, 1].astype(np.int64), im_i=a[:, 2].astype(np.int64), e_i=a[:, 3], d_i=a[:, 4],
               s_i=a[:, 5], k_f=a[:, 6], l_f=a[:, 7].astype(np.int64), im_f=a[:, 8].astype(np.int64), e_f=a[:, 9],
               d_f=a[:, 10], s_f=a[:, 11])
    return {k: np.ascontiguousarray(v) for k, v in out.items()}


def _pair_arrays(pairs):
    """Scalar metadata of every pair's two waves as arrays (each distinct wave read once)."""
    memo: Dict[int, tuple] = {}

    def sc(w):
        v = memo.get(id(w))
        if v is None:
            v = memo[id(w)] = _wave_scalars(w)
        return v
    a = np.array([sc(ci) + sc(cf) for ci, cf in pairs], dtype=np.float64).reshape(len(pairs), 12)
    out = dict(k_i=a[:, 0], l_i=a[:, 1].astype(np.int64), im_i=a[:, 2].astype(np.int64), e_i=a[:, 3], d_i=a[:, 4],
               s_i=a[:, 5], k_f=a[:, 6], l_f=a[:, 7].astype(np.int64), im_f=a[:, 8].astype(np.int64), e_f=a[:, 9],
               d_f=a[:, 10], s_f=a[:, 11])
    return {k: np.ascontiguousarray(v) for k, v in out.items()}


def _idx_limits(job: Job, pa, t: Transition, cupy: bool = False, memo: Optional[dict] = None) -> np.ndarray:
    """Vectorised ``idx_limit`` (dwba_matrix_elements.py:909-1022) for every pair of one transition.
    ``cupy``: the CuPy path's rule (``:1676-1720``, ``_refine_idx_limit_physics`` :688-777), which counts the
    final state's extent only for a bound final state. ``memo``: a dict shared by the transitions of
    one job: the transition enters only through the bound states' 99 % extent, so the pair-only part
    is computed once and a transition whose extent changes no pair's limit reuses the result."""
    g = job.grid
    N, r = g.N, g.r
    base = memo.get("base") if memo is not None else None
    if base is None:
        n1 = np.full(len(pa["k_i"]), N, dtype=np.int64)
        for im in (pa["im_i"], pa["im_f"]):
            m = (im > 0) & (im < N)
            n1 = np.where(m, np.minimum(n1, im + 1), n1)
        kmin = np.minimum(pa["k_i"], pa["k_f"])
        kmax = np.maximum(pa["k_i"], pa["k_f"])
        k_eff = np.where(kmin > 0.1, kmin, kmax)
        lmax = np.maximum(pa["l_i"], pa["l_f"])
        with np.errstate(divide="ignore", invalid="ignore"):
            r_turn = (lmax + 0.5) / k_eff
        idx_turn = np.minimum(np.searchsorted(r, np.where(k_eff > 1e-3, r_turn, 0.0)), N - 20)
        mgf = int(N * job.min_grid_fraction)
        min_idx = np.where(k_eff > 1e-3, np.minimum(np.maximum(idx_turn + 20, mgf), N), max(1, mgf))
        n1 = np.where(n1 < min_idx, min_idx, n1)
        base = (n1, kmin, lmax, int(n1.min()) if len(n1) else N)
        if memo is not None:
            memo["base"] = base
    n1, kmin, lmax, n1_min = base
    idx99 = max(0, g.extent99(t.u_i), g.extent99(t.u_f) if (t.excitation or not cupy) else 0)
    key = idx99 if idx99 > n1_min else -1  # -1: the extent moves no limit
    if memo is not None and key in memo:
        return memo[key].copy()
    n1 = np.where(idx99 > n1, min(N, idx99 + 1), n1)
    ke = 0.5 * kmin ** 2
    uabs = np.abs(job.U_i) if job.U_f is None else np.maximum(np.abs(job.U_i), np.abs(job.U_f))
    cent = lmax * (lmax + 1)
    i0 = np.maximum(0, n1 - 1)
    veff0 = uabs[i0] + cent / (2.0 * r[i0] ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        sel = np.nonzero((ke > 1e-10) & (veff0 / ke > 0.03))[0]
    if len(sel):
        T = n1[sel, None] + np.arange(500)[None, :]
        valid = T < N
        Tc = np.minimum(T, N - 1)
        veff = uabs[Tc] + cent[sel, None] / (2.0 * r[Tc] ** 2)
        ok = valid & (veff / ke[sel, None] < 0.03)
        has = ok.any(axis=1)
        first = np.argmax(ok, axis=1)
        n1[sel] = np.where(has, T[np.arange(len(sel)), first] + 1, n1[sel])
    if memo is not None:
        memo[key] = n1.copy()
    return n1


def _dphis(job: Job, n1: np.ndarray, k_total: np.ndarray, eta_total: np.ndarray) -> np.ndarray:
    """Vectorised adaptive phase step (oscillatory_integrals.py:1716-1755, :1456-1509)."""
    g = job.grid
    d0 = min(max(np.pi / 16, float(job.phase_increment)), np.pi / 4)
    mx = np.zeros(len(n1))
    neutral = np.abs(eta_total) <= 1e-10
    idx = np.maximum(n1 - 2, 0)
    mx[neutral] = np.abs(k_total[neutral] * g.dr_prefix_max[idx[neutral]])
    if (~neutral).any():
        rm = np.maximum(0.5 * (g.r[:-1] + g.r[1:]), 1e-10)
        for key in set(zip(k_total[~neutral].tolist(), eta_total[~neutral].tolist())):
            sel = (~neutral) & (k_total == key[0]) & (eta_total == key[1])
            cm = np.maximum.accumulate(np.abs((key[0] + key[1] / rm) * g.dr))
            mx[sel] = cm[idx[sel]]
    d = np.full(len(n1), d0)
    under = (mx > np.pi / 4) & (k_total >= 1e-10) & (n1 >= 2)
    scale = np.pi / 4 / np.maximum(mx, 1e-12)
    d_eff = d0 * np.maximum(0.25, np.minimum(1.0, scale))
    d = np.where(under, np.clip(d_eff, np.pi / 16, np.pi / 4), d)
    return d


WAVE_CHUNKS = 8  # parts of a side-stream wave upload that kernels can wait for one by one


def _in_order(idx, rows, N: int, block: np.ndarray) -> Optional[int]:
    """First row of ``out`` when the rows ``idx`` of a gather are consecutive and take the block's
    rows 0, 1, ... in order with exactly N columns (the block then copies straight into them)."""
    n = len(idx)
    if block.shape[0] != n or block.shape[1] != N:
        return None
    i = np.asarray(idx, dtype=np.int64)
    r = np.asarray(rows, dtype=np.int64)
    if r[0] != 0 or not (np.all(np.diff(r) == 1) and np.all(np.diff(i) == 1)):
        return None
    return int(i[0])


_COPY_STREAMS: Dict[int, "torch.cuda.Stream"] = {}


def _copy_stream(device) -> "torch.cuda.Stream":
    """A side stream per device for large host-to-device transfers."""
    idx = torch.device(device).index
    idx = torch.cuda.current_device() if idx is None else idx
    st = _COPY_STREAMS.get(idx)
    if st is None:
        st = _COPY_STREAMS[idx] = torch.cuda.Stream(device=idx)
    return st


class Prestaged(NamedTuple):
    """Rows [r0, r0 + n) of a pinned host matrix already on their way to rows [0, n) of ``out`` (a
    device matrix with room for ``out.shape[0] - n`` more rows), in parts with an event after each."""
    out: torch.Tensor
    base_ptr: int
    row_bytes: int
    r0: int
    n: int
    chunks: list


def prestage_waves(pairs, N: int, n_extra: int, device) -> Optional[Prestaged]:
    """Start the copy of a batch's waves before the batch is packed, when its first and last waves
    are rows of one page-locked C-contiguous host matrix of N columns whose rows between them hold
    the pairs' two waves in turn (2 P rows, the order packing numbers them in). The upload checks
    every wave's address against that block afterwards and otherwise copies as usual; a block
    copied in vain costs device bandwidth, not correctness."""
    try:
        c0, c1 = pairs[0][0].chi_of_r, pairs[-1][1].chi_of_r
    except (AttributeError, IndexError, TypeError):
        return None
    b = getattr(c0, "base", None)
    if (b is None or getattr(c1, "base", None) is not b or not isinstance(b, np.ndarray) or b.ndim != 2 or
            b.dtype != np.float64 or not b.flags.c_contiguous or b.shape[1] != N or
            not isinstance(c0, np.ndarray) or not isinstance(c1, np.ndarray) or c0.dtype != np.float64 or
            c1.dtype != np.float64 or c0.shape != (N,) or c1.shape != (N,)):
        return None
    bp, rb = b.__array_interface__["data"][0], 8 * N
    o0, o1 = c0.__array_interface__["data"][0] - bp, c1.__array_interface__["data"][0] - bp
    if o0 % rb or o1 % rb:
        return None
    r0, r1 = o0 // rb, o1 // rb
    n = r1 - r0 + 1
    if not (0 <= r0 <= r1 < b.shape[0]) or n != 2 * len(pairs):
        return None
    src = torch.from_numpy(b[r0:r1 + 1])
    if not src.is_pinned():
        return None
    dev = torch.device(device)
    out = torch.empty((n + max(1, n_extra), N), dtype=torch.float64, device=dev)
    cs = _copy_stream(out.device)
    cs.wait_stream(torch.cuda.current_stream(out.device))  # out belongs to the current stream
    chunks = []
    with torch.cuda.stream(cs):
        cuts = [n * k // WAVE_CHUNKS for k in range(WAVE_CHUNKS + 1)]
        for a, c in zip(cuts[:-1], cuts[1:]):
            if c > a:
                out[a:c].copy_(src[a:c], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(cs)
                chunks.append((a, c, ev))
    out.record_stream(cs)
    return Prestaged(out, bp + r0 * rb, rb, r0, n, chunks)


class WaveMatrix:
    """Distinct 1-D functions of a job as rows of one host matrix (dedup by host buffer)."""

    def __init__(self, N):
        self.N = N
        self.arrays: List[np.ndarray] = []
        self._uploaded: Dict[str, Tuple[int, torch.Tensor]] = {}
        self._by_id: Dict[int, int] = {}
        self._keep: List[object] = []
        self._ptrs: Dict[int, Tuple[int, np.ndarray]] = {}  # first row -> (count, data addresses)
        self.ready: Optional[torch.cuda.Event] = None  # end of a side-stream upload not yet waited for
        # side-stream upload of a block copied in row order: (first row, end row, event after it) of
        # each of its WAVE_CHUNKS parts, so that kernels reading only early rows can start sooner
        self.chunks: Optional[List[Tuple[int, int, torch.cuda.Event]]] = None
        self.prestaged: Optional[Prestaged] = None  # waves already on their way (prestage_waves)

    def wait_ready(self) -> None:
        """Order the current stream after a side-stream upload (``upload(..., side_stream=True)``);
        the kernels' launchers call it before their first launch."""
        if self.ready is not None:
            torch.cuda.current_stream().wait_event(self.ready)
            self.ready = None
        self.chunks = None

    def chunk_of(self, rows: np.ndarray) -> np.ndarray:
        """For each row of the device matrix, the part of a chunked upload after which it is on the
        device (len(chunks) when the whole upload must be waited for, 0 when nothing is pending)."""
        rows = np.asarray(rows, dtype=np.int64)
        if self.chunks is None:
            return np.zeros(len(rows), dtype=np.int64)
        out = np.full(len(rows), len(self.chunks), dtype=np.int64)
        for k, (lo, hi, _) in enumerate(self.chunks):
            out[(rows >= lo) & (rows < hi)] = k
        return out

    def wait_chunk(self, k: int) -> None:
        """Order the current stream after part k of a chunked upload (after all of it for k beyond
        the parts)."""
        if self.chunks is None or k >= len(self.chunks):
            self.wait_ready()
        else:
            torch.cuda.current_stream().wait_event(self.chunks[k][2])

    def add_distinct(self, arrays: Sequence[np.ndarray], ptrs: Optional[np.ndarray] = None) -> int:
        """Append arrays known to be distinct C-contiguous objects of N float64 values that are not
        rows yet (a packed batch's waves, with their data addresses), in order; returns the row of
        the first."""
        first = len(self.arrays)
        self._by_id.update(zip(map(id, arrays), range(first, first + len(arrays))))
        self.arrays.extend(arrays)
        self._keep.extend(arrays)
        if ptrs is not None:
            self._ptrs[first] = (len(arrays), np.asarray(ptrs, dtype=np.int64))
        return first

    def add(self, arr: np.ndarray) -> int:
        """Row of ``arr`` (one row per distinct array object; the object is kept alive with it)."""
        i = self._by_id.get(id(arr))
        if i is None:
            i = self._by_id[id(arr)] = len(self.arrays)
            a = arr if type(arr) is np.ndarray else np.asarray(arr)
            self.arrays.append(a if len(a) == self.N else a[: self.N])
            self._keep.append(arr)  # keeps id(arr) from being reused while the memo holds it
        return i

    def matrix(self) -> np.ndarray:
        if not hasattr(self, "_m"):
            self._m = np.stack([np.asarray(a, dtype=np.float64) for a in self.arrays]) if self.arrays \
                else np.zeros((1, self.N))
        return self._m

    @staticmethod
    def _row_of(a: np.ndarray, N: int, ptr: int, base_ptrs: dict):
        """(base, row) when ``a`` (data at ``ptr``) is a full row of a C-contiguous float64 2-D host
        matrix, else None."""
        b = a.base
        if (b is None or not isinstance(b, np.ndarray) or b.ndim != 2 or b.dtype != np.float64 or
                not b.flags.c_contiguous or b.shape[1] < N or a.dtype != np.float64 or a.ndim != 1 or
                a.strides != (8,)):
            return None
        bp = base_ptrs.get(id(b))
        if bp is None:
            bp = base_ptrs[id(b)] = b.__array_interface__["data"][0]
        off = ptr - bp
        rb = 8 * b.shape[1]
        if off % rb != 0:
            return None
        return b, off // rb

    def upload(self, device, side_stream: bool = False) -> torch.Tensor:
        """Copy every row to the device. Rows taken from one C-contiguous host matrix (in any
        order) are copied with that matrix in one transfer (asynchronous when it is pinned) and
        gathered on the device; other rows that are consecutive in memory go as one block.

        ``side_stream``: the large transfers and their gathers run on a copy stream of the device,
        so that the small synchronous copies the caller issues meanwhile (descriptors) do not wait
        behind them in the current stream; ``ready`` records their end, and whoever launches
        kernels reading the matrix calls ``wait_ready()`` first."""
        N = self.N
        n = len(self.arrays)
        cached = self._uploaded.get(str(device))
        if cached is not None and cached[0] == n:
            return cached[1]  # already on the device (no rows added since)
        pre, self.prestaged = self.prestaged, None
        if side_stream and pre is not None and self._takes(pre):
            return self._adopt(pre, device)
        out = torch.empty((max(1, n), N), dtype=torch.float64, device=device)
        done = np.zeros(n, dtype=bool)
        groups: Dict[int, list] = {}
        base_ptrs: Dict[int, int] = {}
        grouped = np.zeros(n, dtype=bool)
        # runs of packed rows (addresses known): those lying in the rows of the matrix behind their
        # first array are grouped with it by address arithmetic, without a pass per array
        for first, (cnt, addr) in self._ptrs.items():
            b = self.arrays[first].base
            if not (isinstance(b, np.ndarray) and b.ndim == 2 and b.dtype == np.float64 and b.flags.c_contiguous
                    and b.shape[1] >= N):
                continue
            bp = b.__array_interface__["data"][0]
            rb = 8 * b.shape[1]
            off = addr - bp
            ok = (off >= 0) & (off % rb == 0) & (off // rb < b.shape[0])
            idx = first + np.nonzero(ok)[0]
            if len(idx):
                grp = groups.setdefault(id(b), [b, [], []])
                grp[1].extend(idx.tolist())
                grp[2].extend((off[ok] // rb).tolist())
                grouped[idx] = True
        for i in np.nonzero(~grouped)[0].tolist():
            a = self.arrays[i]
            rb = self._row_of(a, N, a.__array_interface__["data"][0], base_ptrs)
            if rb is not None:
                groups.setdefault(id(rb[0]), [rb[0], [], []])
                groups[id(rb[0])][1].append(i)
                groups[id(rb[0])][2].append(rb[1])
        big = []
        for base, idx, rows in groups.values():
            # the contiguous block of the matrix's rows that the group spans goes as one copy when
            # the group uses at least half of it (e.g. all pairs of a batch, or one chunk of them)
            r_arr = np.asarray(rows, dtype=np.int64)
            lo, hi = int(r_arr.min()), int(r_arr.max()) + 1
            if len(idx) < 2 or 2 * len(np.unique(r_arr)) < hi - lo:
                continue  # a small share of its span: per-row copies below
            big.append((base[lo:hi], idx, r_arr - lo))
            done[idx] = True
        side = bool(side_stream and big and out.is_cuda)
        if side:
            # the grouped blocks go first, on the copy stream, so that the transfer starts at once;
            # the index arrays of the gathers and the remaining rows follow as asynchronous copies
            # through pinned staging (the rows on the current stream), none of them blocking the host
            cs = _copy_stream(out.device)
            cs.wait_stream(torch.cuda.current_stream(out.device))  # out belongs to the current stream
            chunks = []
            with torch.cuda.stream(cs):
                blocks = []
                for block, idx, rows in big:
                    src = torch.from_numpy(block)
                    o = _in_order(idx, rows, N, block)
                    if o is not None and src.is_pinned() and not chunks:
                        # the block's rows are these rows of out, in order: no gather; copied in
                        # parts with an event after each
                        nb = len(idx)
                        cuts = [nb * k // WAVE_CHUNKS for k in range(WAVE_CHUNKS + 1)]
                        for a, b in zip(cuts[:-1], cuts[1:]):
                            if b > a:
                                out[o + a:o + b].copy_(src[a:b], non_blocking=True)
                                ev = torch.cuda.Event()
                                ev.record(cs)
                                chunks.append((o + a, o + b, ev))
                        blocks.append(None)
                    elif o is not None:  # the block's rows are these rows of out, in order: no gather
                        out[o:o + len(idx)].copy_(src, non_blocking=src.is_pinned())
                        blocks.append(None)
                    else:
                        blocks.append(src.to(device, non_blocking=src.is_pinned()))
                for (_, idx, rows), dev_block in zip(big, blocks):
                    if dev_block is not None:
                        sel, dst = _dev(rows, device), _dev(np.asarray(idx, dtype=np.int64), device)
                        out.index_copy_(0, dst, dev_block.index_select(0, sel)[:, :N])
            self._copy_rows(out, done, N, n, stage=True)
            out.record_stream(cs)
            self.ready = torch.cuda.Event()
            self.ready.record(cs)
            self.chunks = chunks or None
        else:
            # every small (synchronous) copy first -- the rows outside the grouped matrices and the
            # index arrays of the gathers -- so that none of them waits behind a large asynchronous
            # copy in the stream; the grouped blocks (asynchronous from pinned memory) last
            self._copy_rows(out, done, N, n)
            direct = [_in_order(idx, rows, N, block) for block, idx, rows in big]
            gathers = [(torch.as_tensor(rows, device=device),
                        torch.as_tensor(np.asarray(idx, dtype=np.int64), device=device), block)
                       for (block, idx, rows), o in zip(big, direct) if o is None]
            for (block, idx, _), o in zip(big, direct):
                if o is not None:
                    src = torch.from_numpy(block)
                    out[o:o + len(idx)].copy_(src, non_blocking=src.is_pinned())
            for sel, dst, block in gathers:
                src = torch.from_numpy(block)
                dev_block = src.to(device, non_blocking=src.is_pinned())
                out.index_copy_(0, dst, dev_block.index_select(0, sel)[:, :N])
        self._uploaded[str(device)] = (n, out)
        return out

    def _takes(self, pre: Prestaged) -> bool:
        """Whether the prestaged block holds exactly this matrix's first rows: the packed waves, in
        order, at the block's addresses (and room for the rest)."""
        first = self._ptrs.get(0)
        if first is None or first[0] != pre.n or len(self.arrays) > pre.out.shape[0]:
            return False
        want = pre.base_ptr + pre.row_bytes * np.arange(pre.n, dtype=np.int64)
        return bool(np.array_equal(first[1], want))

    def _adopt(self, pre: Prestaged, device) -> torch.Tensor:
        """Rows [0, n) are the prestaged block (its parts become ``chunks``); the other rows follow
        as in ``upload``, after which ``ready`` covers everything."""
        out, N, n = pre.out, self.N, len(self.arrays)
        done = np.zeros(n, dtype=bool)
        done[:pre.n] = True
        self._copy_rows(out, done, N, n, stage=True)
        cs = _copy_stream(out.device)
        self.ready = torch.cuda.Event()
        self.ready.record(cs)
        self.chunks = list(pre.chunks)
        self._uploaded[str(device)] = (n, out)
        return out

    def _copy_rows(self, out: torch.Tensor, done: np.ndarray, N: int, n: int, stage: bool = False) -> None:
        """Rows not taken from a grouped matrix: consecutive ones in memory as one block, the others
        one by one (``stage``: pageable rows through pinned staging memory, asynchronously)."""
        todo = np.nonzero(~done[:n])[0].tolist()
        k = 0
        while k < len(todo):
            i = todo[k]
            a = self.arrays[i]
            p0 = a.__array_interface__["data"][0]
            j = i + 1
            ok = a.flags.c_contiguous and a.dtype == np.float64 and len(a) == N
            while ok and j < n and not done[j]:
                b = self.arrays[j]
                if not (b.flags.c_contiguous and b.dtype == np.float64 and len(b) == N and
                        b.__array_interface__["data"][0] == p0 + 8 * N * (j - i)):
                    break
                j += 1
            if ok and j - i > 1 and a.base is not None:
                block = np.lib.stride_tricks.as_strided(a, shape=(j - i, N), strides=(8 * N, 8))
            else:
                j = i + 1
                block = np.ascontiguousarray(a, dtype=np.float64).reshape(1, N)
            src = torch.from_numpy(block)
            if stage and out.is_cuda and block.nbytes <= _Staging.MAX and not src.is_pinned():
                # small rows by the staging ring's kernel copy: a copy-engine transfer would wait
                # behind the large one on the side stream, and every later launch on this stream with it
                _Staging.get(out.device.index).copy(np.ascontiguousarray(block), out[i:j])
            else:
                if stage and out.is_cuda and not src.is_pinned():
                    src = src.pin_memory()
                out[i:j].copy_(src, non_blocking=src.is_pinned())
            k += j - i  # rows i..j-1 are consecutive entries of todo


@dataclass
class JobPlan:
    """Host plan of a job, as arrays over (transition, pair).

    n1: integration limit; osc: oscillatory branch (per pair); ns_index: node set of the pair
    (index into ``nodesets``, -1 when there is none); corr_dir/corr_ex: L=0 corrections;
    tails: outer tails of the direct term evaluated on the host, keyed by (t, p);
    tail_tp/tail_wave/tail_rm/tail_rmax/tail_mode: the tails left to the device kernel (one
    record per (t, p)); moments: multipole moments M_L of each transition (T, L_max+1)."""
    n1: np.ndarray
    osc: np.ndarray
    ns_index: np.ndarray
    nodesets: List[NodeSetPlan]
    corr_dir: np.ndarray
    corr_ex: np.ndarray
    tails: Dict[Tuple[int, int], np.ndarray]
    tail_tp: np.ndarray = None
    tail_wave: np.ndarray = None
    tail_rm: np.ndarray = None
    tail_rmax: np.ndarray = None
    tail_mode: np.ndarray = None
    moments: np.ndarray = None
    tail_limits: Tuple[int, float] = (4096, np.pi / 2)

    @property
    def n_tail_dev(self) -> int:
        return 0 if self.tail_tp is None else len(self.tail_tp)

    def pair(self, t: int, p: int) -> PairPlan:
        k = int(self.ns_index[t, p])
        return PairPlan(n1=int(self.n1[t, p]), osc=bool(self.osc[p]), nodeset=self.nodesets[k] if k >= 0 else None,
                        corr_dir=float(self.corr_dir[t, p]), corr_ex=float(self.corr_ex[t, p]),
                        tail=self.tails.get((t, p)))


def _unique_rows(a: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """np.unique(a, axis=0, return_inverse=True) for a 2-D float array: the distinct rows in
    lexicographic order and the row of each input among them (by a stable lexsort of the columns,
    which is several times faster than numpy's structured-row sort; same result)."""
    order = np.lexsort(a.T[::-1])
    srt = a[order]
    new = np.ones(len(a), dtype=bool)
    if len(a) > 1:
        new[1:] = np.any(srt[1:] != srt[:-1], axis=1)
    grp = np.cumsum(new) - 1
    inv = np.empty(len(a), dtype=np.int64)
    inv[order] = grp
    return srt[new], inv


_new_key = functools.partial(tuple.__new__, NodeSetKey)  # from one tuple of the fields, no Python frame
_new_plan = functools.partial(tuple.__new__, NodeSetPlan)


def plan_job(job: Job, waves: Optional[WaveMatrix] = None) -> JobPlan:
    """Host planning (vectorised over pairs): integration limit, branch, node set, L=0
    corrections and outer tails for every (transition, pair)."""
    g = job.grid
    N, r, w = g.N, g.r, g.w
    P, T = len(job.pairs), len(job.transitions)
    packed = getattr(job, "_packed", None)
    pa = _packed_pair_arrays(packed.scalars) if packed is not None else _pair_arrays(job.pairs)
    k_total = pa["k_i"] + pa["k_f"]
    eta_total = pa["e_i"] + pa["e_f"]
    osc = np.asarray(job.use_oscillatory_quadrature & (k_total > job.k_threshold), dtype=bool)
    V_diff = job.V_core - job.U_i
    v_live = bool(np.any(V_diff))
    max_seg, max_dphi = tail_limits()
    legacy = job.oscillatory_method == "legacy"
    if waves is None:
        waves = WaveMatrix(N)
    if packed is not None and packed.owner is not waves and not waves.arrays:
        packed.first, packed.owner = waves.add_distinct(packed.arrays, packed.ptrs), waves
    if packed is not None and packed.owner is waves:
        # rows of the packed waves (added to this matrix in the packed order)
        wi_idx, wf_idx = packed.rows_i + packed.first, packed.rows_f + packed.first
    else:
        wi_idx = np.array([waves.add(ci.chi_of_r) for ci, _ in job.pairs], dtype=np.int64)
        wf_idx = np.array([waves.add(cf.chi_of_r) for _, cf in job.pairs], dtype=np.int64)
    n1_all = np.zeros((T, P), dtype=np.int64)
    ns_index = np.full((T, P), -1, dtype=np.int64)
    corr_dir = np.zeros((T, P))
    corr_ex = np.zeros((T, P))
    tails: Dict[Tuple[int, int], np.ndarray] = {}
    dev_tp, dev_wave, dev_rm, dev_rmax = [], [], [], []
    moments_all = np.zeros((T, job.L_max + 1))
    nodesets: List[NodeSetPlan] = []
    ns_pos: Dict[NodeSetKey, int] = {}
    idx_memo: dict = {}
    for ti, t in enumerate(job.transitions):
        n1 = _idx_limits(job, pa, t, memo=idx_memo)
        n1_all[ti] = n1
        # distinct node sets of this transition (pairs of one energy share k_total and eta); a
        # transition with the same integration limits as the previous one has the same node sets
        cand = np.nonzero(osc & (n1 >= 2))[0]
        if ti > 0 and np.array_equal(n1, n1_all[ti - 1]):
            ns_index[ti] = ns_index[ti - 1]
        elif len(cand):
            d = _dphis(job, n1, k_total, eta_total)
            keys = np.stack([n1[cand].astype(np.float64), k_total[cand], d[cand], eta_total[cand]], axis=1)
            uk, inv = _unique_rows(keys)
            pos = np.empty(len(uk), dtype=np.int64)
            # breakpoint counts of the linspace (eta == 0) sets for all keys at once, with the
            # arithmetic of plan_nodeset; Coulomb sets go through plan_nodeset one by one
            u_n1 = uk[:, 0].astype(np.int64)
            span = r[u_n1 - 1] - r[0]
            with np.errstate(divide="ignore", invalid="ignore"):
                n_lin = np.ceil(span / (uk[:, 2] / uk[:, 1])) + 1
                step = span / (n_lin - 1)
            lin_ok = (uk[:, 1] >= 1e-10) & (n_lin >= 2) & (step > 1e-12)
            keys = list(map(_new_key, zip(repeat(id(g)), u_n1.tolist(), uk[:, 1].tolist(), uk[:, 2].tolist(),
                                          uk[:, 3].tolist(), repeat(int(job.CC_nodes)))))
            if bool(np.all(np.abs(uk[:, 3]) < 1e-10)) and not any(map(ns_pos.__contains__, keys)):
                # linspace sets only, none seen before (the usual case): built in bulk, in key order
                ok = np.nonzero(lin_ok)[0]
                pos[:] = -1
                pos[ok] = len(nodesets) + np.arange(len(ok))
                nodesets.extend(map(_new_plan, zip([keys[u] for u in ok.tolist()],
                                                   n_lin[ok].astype(np.int64).tolist(), repeat(None),
                                                   g.log_prefixes(u_n1[ok].tolist()),
                                                   repeat(g.log_full))))
                ns_pos.update(zip(keys, pos.tolist()))
                keys = ()
            for u, key in enumerate(keys):
                rec = key[1:5]  # n1, k_total, dphi, eta_total
                q = ns_pos.get(key)
                if q is None:
                    if abs(rec[3]) < 1e-10:
                        nsp = (NodeSetPlan(key, int(n_lin[u]), None, g.log_prefix(key.n1), g.log_full)
                               if lin_ok[u] else None)
                    else:
                        nsp = plan_nodeset(g, key)
                    q = -1 if nsp is None else len(nodesets)
                    if nsp is not None:
                        nodesets.append(nsp)
                    ns_pos[key] = q
                pos[u] = q
            ns_index[ti, cand] = pos[np.ravel(inv)]
        # L=0 corrections with the limited Simpson weights (dwba_matrix_elements.py:1028-1046, :1249-1296)
        if v_live:
            # per pair with the reference's own expressions (np.dot of rho_w and V_diff), so the
            # rounding does not depend on how many pairs share the call
            W = waves.matrix()
            for nv in np.unique(n1):
                sel = np.nonzero(n1 == nv)[0]
                wl = w.copy()
                wl[nv:] = 0.0
                s2 = np.sum(wl * t.u_f * t.u_i)
                wl_uf = wl * t.u_f
                for p in sel:
                    chi_i, chi_f = W[wi_idx[p]], W[wf_idx[p]]
                    wl_cf = wl * chi_f
                    if abs(s2) > OVERLAP_TOL:
                        corr_dir[ti, p] = np.dot(wl_cf * chi_i, V_diff) * s2
                    s2e = np.sum(wl_cf * t.u_i)
                    if abs(s2e) > OVERLAP_TOL:
                        corr_ex[ti, p] = np.dot(wl_uf * chi_i, V_diff) * s2e
        # outer tails of the direct term (dwba_matrix_elements.py:1213-1241 advanced/full_split; :1256-1267 legacy)
        want = (job.L_max >= 1) & (n1 < N - 10) & t.excitation & (
            (legacy & job.use_oscillatory_quadrature) | ((not legacy) & osc))
        if want.any():
            moments = multipole_moments(g, t.u_i, t.u_f, job.L_max)
            if job.tails_per_unit_moment:
                moments = np.ones(job.L_max + 1)
            moments_all[ti] = moments
            for p in np.nonzero(want)[0]:
                wave = np.array([pa["k_i"][p], pa["l_i"][p], pa["d_i"][p], pa["e_i"][p], pa["s_i"][p],
                                 pa["k_f"][p], pa["l_f"][p], pa["d_f"][p], pa["e_f"][p], pa["s_f"][p]])
                r_m, r_end = float(r[n1[p] - 1]), float(r[-1])
                # the device kernel covers the Filon/Levin branches; pairs whose mid-interval
                # frequency selects the adaptive-quadrature branch stay on the host
                if job.tails_on_device and not job.tails_per_unit_moment and (
                        legacy or _lib.tail_on_device(wave, r_m, r_end)):
                    dev_tp.append((ti, int(p)))
                    dev_wave.append(wave)
                    dev_rm.append(r_m)
                    dev_rmax.append(r_end)
                else:
                    tails[(ti, int(p))] = _lib.outer_tails(wave, r_m, r_end, job.L_max, moments,
                                                           1 if legacy else 0, max_seg, max_dphi)
    job._waves = waves
    job._wave_idx = (wi_idx, wf_idx)
    nd = len(dev_tp)
    return JobPlan(n1=n1_all, osc=osc, ns_index=ns_index, nodesets=nodesets, corr_dir=corr_dir, corr_ex=corr_ex,
                   tails=tails, tail_tp=np.array(dev_tp, dtype=np.int64).reshape(nd, 2),
                   tail_wave=np.array(dev_wave, dtype=np.float64).reshape(nd, 10),
                   tail_rm=np.array(dev_rm, dtype=np.float64), tail_rmax=np.array(dev_rmax, dtype=np.float64),
                   tail_mode=np.full(nd, 1 if legacy else 0, dtype=np.int32), moments=moments_all,
                   tail_limits=(max_seg, max_dphi))


def _take(a: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """a[idx] for a structured descriptor array, copied as raw rows (numpy copies structured
    records field by field, which costs milliseconds for a few thousand descriptors)."""
    rows = a.view(np.uint8).reshape(len(a), a.dtype.itemsize)
    return rows[idx].view(a.dtype).reshape(-1)


def _interleave(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """[x0, y0, x1, y1, ...] for two structured arrays of one dtype and length, as raw rows."""
    n, isz = len(x), x.dtype.itemsize
    out = np.empty((2 * n, isz), dtype=np.uint8)
    out[0::2] = x.view(np.uint8).reshape(n, isz)
    out[1::2] = y.view(np.uint8).reshape(n, isz)
    return out.view(x.dtype).reshape(-1)


def expand_multi(multi: np.ndarray) -> np.ndarray:
    """The single folds a set of multi-folds stands for (same operator, factors and output)."""
    n = int(np.sum(multi["n_f"])) if len(multi) else 0
    out = np.zeros(n, dtype=_lib.FOLD_DTYPE)
    if n == 0:
        return out
    g = np.repeat(np.arange(len(multi)), multi["n_f"])
    pos = np.arange(n) - np.repeat(np.cumsum(multi["n_f"]) - multi["n_f"], multi["n_f"])
    out["op"], out["g"] = multi["op"][g], multi["g"][g]
    out["f"], out["out"] = multi["f"][g, pos], multi["out"][g, pos]
    for k in ("half_band", "n_out", "n_src", "n_clear"):
        out[k] = multi[k][g]
    return out


@dataclass
class DirectPlan:
    """How the exact engines evaluate the forms of one prepared job (indices into its forms).

    A direct form whose column operand is its transition's full-grid b = w u_f u_i (the Filon
    direct term and the no-interval branch) is a dot product of the pair's folded density with
    the transition's multipole potential phi_L = K_L b, the reference's inner integral int_r2
    (oscillatory_integrals.py:2571), which every pair of the transition shares. ``pot_b``: device
    address of each transition's b (0 when no form of it takes this path); ``dot_fo`` / ``dot_t``:
    those forms and their transitions; ``ss_fo``: the forms left to the semiseparable kernel."""
    pot_b: np.ndarray
    dot_fo: np.ndarray
    dot_t: np.ndarray
    ss_fo: np.ndarray


class FormLaunch:
    """Device descriptors of the exact forms of one or several prepared jobs: one multipole potential
    per transition with Filon direct forms, the dot forms against them (runs of ``DOT_RUN`` sharing a
    potential, padded with empty descriptors) and the remaining forms as semiseparable forms, whose
    results go to a compact buffer scattered into the result rows. ``entries``: per job
    (forms_host, plan, N, r_ptr, dot_rows, ss_rows) with dot_rows / ss_rows the result rows (of
    ``out``) of plan.dot_fo / plan.ss_fo."""

    def __init__(self, entries, out: torch.Tensor, nl: int, dev):
        self.out, self.nl = out, nl
        row = np.uint64(8 * nl)
        out_p = np.uint64(_ptr(out))
        phi_len = [int(np.count_nonzero(pl.pot_b)) * nl * N for _, pl, N, _, _, _ in entries]
        self.phi = torch.empty(max(1, sum(phi_len)), dtype=torch.float64, device=dev)
        base = np.uint64(_ptr(self.phi))
        pots, dots, ss_forms, ss_rows = [], [], [], []
        off = 0
        for (fh, pl, N, r_ptr, dot_rows, ss_out), ln in zip(entries, phi_len):
            used = np.nonzero(pl.pot_b)[0]
            phi_t = np.zeros(len(pl.pot_b), dtype=np.uint64)
            phi_t[used] = base + np.uint64(8) * (np.uint64(off) + np.uint64(nl * N) * np.arange(len(used), dtype=np.uint64))
            off += ln
            p = np.zeros(len(used), dtype=_lib.POTENTIAL_DTYPE)
            p["r"], p["b"], p["phi"] = r_ptr, pl.pot_b[used], phi_t[used]
            p["n_rows"] = p["n_cols"] = p["stride"] = N
            pots.append(p)
            if len(pl.dot_fo):
                # group by transition, each group padded to whole runs of DOT_RUN
                order = np.argsort(pl.dot_t, kind="stable")
                t_s = pl.dot_t[order]
                cnt = np.bincount(t_s, minlength=len(pl.pot_b))
                padded = (cnt + _lib.DOT_RUN - 1) // _lib.DOT_RUN * _lib.DOT_RUN
                start = np.concatenate([[0], np.cumsum(padded)[:-1]])
                first = np.concatenate([[0], np.cumsum(cnt)[:-1]])
                pos = start[t_s] + (np.arange(len(t_s)) - first[t_s])
                d = np.zeros(int(padded.sum()), dtype=_lib.DOT_DTYPE)
                fo = pl.dot_fo[order]
                d["a"][pos] = fh["a"][fo]
                d["phi"][pos] = phi_t[t_s]
                d["out"][pos] = out_p + row * np.asarray(dot_rows, dtype=np.uint64)[order]
                d["n_rows"][pos] = fh["n_rows"][fo]
                d["stride"] = N
                dots.append(d)
            if len(pl.ss_fo):
                ss_forms.append(_take(fh, pl.ss_fo))
                ss_rows.append(np.asarray(ss_out, dtype=np.int64))
        pots = np.concatenate(pots) if pots else np.zeros(0, dtype=_lib.POTENTIAL_DTYPE)
        dots = np.concatenate(dots) if dots else np.zeros(0, dtype=_lib.DOT_DTYPE)
        self.n_pots, self.n_dots = len(pots), len(dots)
        self.pots_d = _dev(pots.view(np.uint8), dev) if len(pots) else None
        self.dots_d = _dev(dots.view(np.uint8), dev) if len(dots) else None
        self.n_ss = int(sum(len(f) for f in ss_forms))
        if self.n_ss:
            self.ss_forms_host = np.concatenate(ss_forms)
            self.ss_forms_d = _dev(self.ss_forms_host.view(np.uint8), dev)
            self.ss_rows_d = _dev(np.concatenate(ss_rows), dev)
            self.out_ss = torch.empty((self.n_ss, nl), dtype=torch.float64, device=dev)
        self.pots_host, self.dots_host = pots, dots

    def launch(self, lib, L_max: int, ds: np.ndarray, r_min: float, r_max: float, marks: Optional[list] = None,
               parts=("potentials", "dots", "semisep")) -> None:
        """Enqueue the potentials, the dot forms and the semiseparable forms (those of ``parts``).
        With ``marks`` (a list), a CUDA event is recorded after each of the three and appended as
        (name, event)."""
        st = _stream()

        def mark(name):
            if marks is not None:
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(torch.cuda.current_stream())
                marks.append((name, ev))
        if self.n_pots and "potentials" in parts:
            _lib.check(lib.dwba_multipole_potentials(_ptr(self.pots_d), self.n_pots, L_max, ds.ctypes.data, r_min, r_max,
                                                     st), "dwba_multipole_potentials")
        mark("potentials")
        if self.n_dots and "dots" in parts:
            _lib.check(lib.dwba_dot_forms(_ptr(self.dots_d), self.n_dots, L_max, st), "dwba_dot_forms")
        mark("dots")
        if self.n_ss and "semisep" in parts:
            _lib.check(lib.dwba_bilinear_semisep_fp64(_ptr(self.ss_forms_d), self.n_ss, L_max, ds.ctypes.data, r_min,
                                                      r_max, _ptr(self.out_ss), st), "dwba_bilinear_semisep_fp64")
            self.out.index_copy_(0, self.ss_rows_d, self.out_ss)
        mark("semisep")

    def stage_bytes(self) -> Dict[str, float]:
        """Algorithmic bytes of each of the three launches (see ``algorithmic_bytes``)."""
        out = {"potentials": 0.0, "dots": 0.0, "semisep": 0.0}
        if self.n_pots:
            p = self.pots_host
            out["potentials"] = float(np.sum(8.0 * (2.0 * p["n_cols"] + self.nl * p["n_rows"].astype(np.float64))))
        if self.n_dots:
            d = self.dots_host
            runs = d[::_lib.DOT_RUN]
            out["dots"] = float(np.sum(8.0 * d["n_rows"].astype(np.float64))) + \
                float(np.sum(8.0 * self.nl * runs["stride"].astype(np.float64)))
        if self.n_ss:
            f = self.ss_forms_host
            m = np.maximum(f["n_rows"], f["n_cols"]).astype(np.float64)
            out["semisep"] = float(np.sum(8.0 * (f["n_rows"].astype(np.float64) + f["n_cols"] + m)))
        return out

    def algorithmic_bytes(self) -> float:
        """Operand bytes: each potential reads b and r and writes (L_max+1) rows; each dot form reads a
        (the potential's tiles are read once per run); each semiseparable form reads a, b and r."""
        b = 0.0
        if self.n_pots:
            p = self.pots_host
            b += float(np.sum(8.0 * (2.0 * p["n_cols"] + self.nl * p["n_rows"].astype(np.float64))))
        if self.n_dots:
            d = self.dots_host
            b += float(np.sum(8.0 * d["n_rows"].astype(np.float64)))
            runs = d[::_lib.DOT_RUN]
            b += float(np.sum(8.0 * self.nl * runs["stride"].astype(np.float64)))
        if self.n_ss:
            f = self.ss_forms_host
            m = np.maximum(f["n_rows"], f["n_cols"]).astype(np.float64)
            b += float(np.sum(8.0 * (f["n_rows"].astype(np.float64) + f["n_cols"] + m)))
        return b


FUSE_MIN_SETS = 64  # fuse node sets with their folds when a job has at least this many single-pair sets


def fusable_sets(plans: "JobPlan", T: int) -> Optional[np.ndarray]:
    """Mask over ``plans.nodesets``: the sets whose every use is one pair's phase-split entries with at
    most FOLD_MULTI - 1 transitions (one multi-fold group per operator), or None if a set has other
    uses. Such a set is applied to its pair's folds at once instead of being stored -- worthwhile when
    many distinct sets each serve one pair (e.g. a batch of pairs at different energies); a set that
    serves several pairs (all pairs of one energy) is built once and stored."""
    n_sets = len(plans.nodesets)
    if n_sets == 0:
        return None
    use = (plans.ns_index >= 0) & plans.osc[None, :]
    t_i, p_i = np.nonzero(use)
    k = plans.ns_index[t_i, p_i]
    ok = np.zeros(n_sets, dtype=bool)
    if not len(k):
        return ok
    first_p = np.full(n_sets, -1, dtype=np.int64)
    first_p[k[::-1]] = p_i[::-1]  # some pair of each set
    single = np.ones(n_sets, dtype=bool)
    single[k[p_i != first_p[k]]] = False  # another pair uses it
    n_t = np.bincount(k, minlength=n_sets)
    ok = single & (n_t >= 1) & (n_t <= _lib.FOLD_MULTI - 1)
    return ok


class PreparedJob:
    """A job planned on the host with its inputs and descriptors resident on the device.

    ``launch()`` enqueues every kernel on the current stream: node-set operators (those not
    yet cached for the grid, or all of them with ``rebuild_nodesets``), operand folds and the
    bilinear forms. ``collect()`` copies the results back once and adds the host-side L=0
    corrections and outer tails. Results are indexed [transition, pair, L]. With ``early_nodesets``
    the constructor enqueues the node sets as soon as their descriptors exist (the first
    ``launch()`` then enqueues the rest). With ``early_direct``
    (exact engine, every direct form through the potentials), the direct rows are copied back
    before the exchange forms run, and ``collect_direct()`` returns them first.
    """

    def __init__(self, job: Job, dg: DeviceGrid, engine: str = "dense", plans=None,
                 rebuild_nodesets: bool = False, fuse_folds: Optional[bool] = None, early_direct: bool = False,
                 early_nodesets: bool = False):
        if engine not in ENGINES:
            raise ValueError(f"unknown engine {engine!r}; choose from {ENGINES}")
        if job.L_max < 0:
            raise ValueError("radial_ME_all_L: L_max must be >= 0.")
        if job.L_max > _lib.DWBA_MAX_L:
            raise ValueError(f"L_max > {_lib.DWBA_MAX_L} is not supported")
        self.job, self.dg, self.engine = job, dg, engine
        self.lib = lib = _lib.load()
        dev = dg.device
        g = job.grid
        N = g.N
        self.nl = nl = job.L_max + 1
        self.plans = plans = plan_job(job) if plans is None else plans
        T, P = len(job.transitions), len(job.pairs)
        self.T, self.P = T, P
        # 1. node sets (operators cached per grid and key; rebuilt every launch when rebuild_nodesets);
        # sets that serve a single pair are applied to its folds at once when fusing (see fusable_sets)
        fused = fusable_sets(plans, T) if fuse_folds is not False else None
        if fuse_folds is None and fused is not None and int(fused.sum()) < FUSE_MIN_SETS:
            fused = None
        self.nodesets = NodeSetBatch(dg, plans.nodesets, job.CC_nodes, rebuild=rebuild_nodesets, fused=fused)
        # 2. functions on the device: continuum waves (planner order) + bound functions
        waves = getattr(job, "_waves", None) or WaveMatrix(N)
        wi_idx, wf_idx = getattr(job, "_wave_idx", (None, None))
        if wi_idx is None:
            wi_idx = np.array([waves.add(ci.chi_of_r) for ci, _ in job.pairs], dtype=np.int64)
            wf_idx = np.array([waves.add(cf.chi_of_r) for _, cf in job.pairs], dtype=np.int64)
        tidx = [(waves.add(t.u_i), waves.add(t.u_f)) for t in job.transitions]
        self.waves = waves
        self.wave_rows = (np.asarray(wi_idx), np.asarray(wf_idx), tidx)
        self.F = F = waves.upload(dev)
        self.h2d_bytes = len(waves.arrays) * N * 8
        Fp = np.uint64(_ptr(F))
        row = np.uint64(8 * N)
        fptr = lambda i: Fp + row * np.asarray(i, dtype=np.uint64)  # noqa: E731
        # 3. operand folds: per (t, p) a_dir, a_ex, b_ex, b_dir(standard); one full-grid b_dir per transition
        SL = 4
        n_slots = SL * T * P + T
        ops = torch.empty((n_slots, N), dtype=torch.float64, device=dev)
        Op = np.uint64(_ptr(ops))
        wl_cache: Dict[int, torch.Tensor] = {}

        def wl_ptr(n1):  # Simpson weights zeroed past n1 (dwba_matrix_elements.py:1025-1026)
            t_ = wl_cache.get(n1)
            if t_ is None:
                t_ = dg.w.clone()
                t_[n1:] = 0.0
                wl_cache[n1] = t_
            return t_.data_ptr()

        ta_ptr, bx_ptr = self.nodesets.ta_all, self.nodesets.bx_all
        w_ptr, r_ptr = np.uint64(_ptr(dg.w)), np.uint64(_ptr(dg.r))
        fold_parts, forms = [], np.zeros(2 * T * P, dtype=_lib.FORM_DTYPE)
        pidx = np.arange(P, dtype=np.int64)
        ci_p, cf_p = fptr(wi_idx), fptr(wf_idx)

        def mk(op, f, g_, out, h, n_out, n_src, n_clear):
            a = np.zeros(len(out), dtype=_lib.FOLD_DTYPE)
            a["op"], a["f"], a["g"], a["out"] = op, f, g_, out
            a["half_band"], a["n_out"], a["n_src"], a["n_clear"] = h, n_out, n_src, n_clear
            return a

        A_parts = []  # node-set branch entries, grouped into multi-folds after the loop
        for ti, (iu_i, iu_f) in enumerate(tidx):
            ui_p, uf_p = fptr(iu_i), fptr(iu_f)
            b_full = Op + row * np.uint64(SL * T * P + ti)  # filon inner integral runs over all N
            fold_parts.append(mk(w_ptr, uf_p, ui_p, np.array([b_full]), 0, N, N, N))
            n1 = plans.n1[ti]
            k = plans.ns_index[ti]
            base = (SL * (ti * P + pidx)).astype(np.uint64)
            a_dir, a_ex, b_ex, b_dir = (Op + row * (base + np.uint64(q)) for q in range(SL))
            fo = 2 * (ti * P + pidx)
            nb = np.minimum(N, n1 + 2)
            A = plans.osc & (k >= 0)
            B = plans.osc & (k < 0)
            C = ~plans.osc
            if A.any():
                nA = int(A.sum())
                A_parts.append((np.full(nA, ti), pidx[A], k[A], a_dir[A], a_ex[A], b_ex[A], n1[A], nb[A],
                                np.full(nA, uf_p, dtype=np.uint64), np.full(nA, ui_p, dtype=np.uint64), fo[A]))
                forms["r"][fo[A]], forms["a"][fo[A]], forms["b"][fo[A]] = r_ptr, a_dir[A], b_full
                forms["n_rows"][fo[A]], forms["n_cols"][fo[A]] = n1[A], N
                forms["r"][fo[A] + 1], forms["a"][fo[A] + 1], forms["b"][fo[A] + 1] = r_ptr, a_ex[A], b_ex[A]
                forms["n_rows"][fo[A] + 1], forms["n_cols"][fo[A] + 1] = n1[A], nb[A]
            if B.any():
                # no valid phase interval: weighted dot products over r[:n1] x r[:N]
                # (oscillatory_integrals.py:2580-2587, :2694-2699)
                fold_parts.append(mk(w_ptr, cf_p[B], ci_p[B], a_dir[B], 0, n1[B], N, n1[B]))
                fold_parts.append(mk(w_ptr, uf_p, ci_p[B], a_ex[B], 0, n1[B], N, n1[B]))
                fold_parts.append(mk(w_ptr, cf_p[B], ui_p, b_ex[B], 0, N, N, N))
                forms["r"][fo[B]], forms["a"][fo[B]], forms["b"][fo[B]] = r_ptr, a_dir[B], b_full
                forms["n_rows"][fo[B]], forms["n_cols"][fo[B]] = n1[B], N
                forms["r"][fo[B] + 1], forms["a"][fo[B] + 1], forms["b"][fo[B] + 1] = r_ptr, a_ex[B], b_ex[B]
                forms["n_rows"][fo[B] + 1], forms["n_cols"][fo[B] + 1] = n1[B], N
            if C.any():
                # standard Simpson path with limited weights (dwba_matrix_elements.py:1242-1245, :1287-1289)
                wl = np.array([wl_ptr(int(v)) for v in n1[C]], dtype=np.uint64)
                fold_parts.append(mk(wl, cf_p[C], ci_p[C], a_dir[C], 0, n1[C], N, n1[C]))
                fold_parts.append(mk(wl, uf_p, ci_p[C], a_ex[C], 0, n1[C], N, n1[C]))
                fold_parts.append(mk(wl, cf_p[C], ui_p, b_ex[C], 0, n1[C], N, n1[C]))
                fold_parts.append(mk(wl, uf_p, ui_p, b_dir[C], 0, n1[C], N, n1[C]))
                forms["r"][fo[C]], forms["a"][fo[C]], forms["b"][fo[C]] = r_ptr, a_dir[C], b_dir[C]
                forms["n_rows"][fo[C]], forms["n_cols"][fo[C]] = n1[C], n1[C]
                forms["r"][fo[C] + 1], forms["a"][fo[C] + 1], forms["b"][fo[C] + 1] = r_ptr, a_ex[C], b_ex[C]
                forms["n_rows"][fo[C] + 1], forms["n_cols"][fo[C] + 1] = n1[C], n1[C]
        # node-set branch: one multi-fold per (pair, node set) and operator -- T with g = chi_i for
        # a_dir (f = chi_f) and a_ex of every transition (f = u_f), B with g = chi_f for b_ex of every
        # transition (f = u_i); a_dir no longer depends on the transition, so its direct forms share it
        multi = np.zeros(0, dtype=_lib.FOLD_MULTI_DTYPE)
        if A_parts:
            cols = [np.concatenate(c) for c in zip(*A_parts)]
            t_a, p_a, k_a, adir_a, aex_a, bex_a, n1_a, nb_a, uf_a, ui_a, fo_a = cols
            # by pair, then node set, then transition (a stable sort of one composite key: the order
            # of np.lexsort((t_a, k_a, p_a)), which takes several times as long)
            nk, nt = int(k_a.max()) + 1, int(t_a.max()) + 1
            order = np.argsort((p_a * nk + k_a) * nt + t_a, kind="stable")
            t_a, p_a, k_a, adir_a, aex_a, bex_a, n1_a, nb_a, uf_a, ui_a, fo_a = (c[order] for c in cols)
            n = len(p_a)
            new_run = np.ones(n, dtype=bool)
            new_run[1:] = (p_a[1:] != p_a[:-1]) | (k_a[1:] != k_a[:-1])
            run_start = np.maximum.accumulate(np.where(new_run, np.arange(n), 0))
            pos_run = np.arange(n) - run_start
            per = _lib.FOLD_MULTI - 1  # transitions per group (one f slot of T holds a_dir)
            new_grp = new_run | (pos_run % per == 0)
            gid = np.cumsum(new_grp) - 1
            G = int(gid[-1]) + 1
            first = np.nonzero(new_grp)[0]
            pos = np.arange(n) - first[gid]
            cnt = np.bincount(gid, minlength=G)
            mT = np.zeros(G, dtype=_lib.FOLD_MULTI_DTYPE)
            mB = np.zeros(G, dtype=_lib.FOLD_MULTI_DTYPE)
            pf, kf = p_a[first], k_a[first]
            mT["op"], mT["g"] = ta_ptr[kf], ci_p[pf]
            mT["f"][:, 0], mT["out"][:, 0] = cf_p[pf], adir_a[first]
            mT["f"][gid, 1 + pos], mT["out"][gid, 1 + pos] = uf_a, aex_a
            mT["n_f"], mT["half_band"] = 1 + cnt, 1
            mT["n_out"] = mT["n_src"] = mT["n_clear"] = n1_a[first]
            mB["op"], mB["g"] = bx_ptr[kf], cf_p[pf]
            mB["f"][gid, pos], mB["out"][gid, pos] = ui_a, bex_a
            mB["n_f"], mB["half_band"] = cnt, 2
            mB["n_out"], mB["n_src"], mB["n_clear"] = nb_a[first], N, nb_a[first]
            forms["a"][fo_a] = adir_a[first][gid]
            # T and B multi-folds of one pair launched next to each other, so that the continuum
            # wave both read (chi_f) is still in L2 for the second
            multi = _interleave(mT, mB)
            ns = self.nodesets
            if ns.n_fused:
                # the groups of fused sets (one per set) go with the node-set launch, in its order
                pos = np.full(len(ns.ta_all), -1, dtype=np.int64)
                pos[ns.fused_idx] = np.arange(ns.n_fused)
                q = pos[kf]
                fg = q >= 0
                if int(np.count_nonzero(fg)) != ns.n_fused or \
                        int(np.count_nonzero(np.bincount(q[fg], minlength=ns.n_fused))) != ns.n_fused:
                    raise RuntimeError("fused node sets must serve exactly one multi-fold group each")
                sel = np.nonzero(fg)[0][np.argsort(q[fg], kind="stable")]  # groups in node-set order
                if waves.chunks is not None:
                    # sets whose pair's waves arrive in an earlier part of the upload go first, in
                    # groups that each wait only for their part
                    pp = pf[sel]
                    ch = waves.chunk_of(np.maximum(wi_idx[pp], wf_idx[pp]))
                    perm = np.argsort(ch, kind="stable")
                    cs = ch[perm]
                    starts = np.concatenate([[0], np.nonzero(np.diff(cs))[0] + 1])
                    ends = np.concatenate([starts[1:], [len(cs)]])
                    ns.reorder_fused(perm, [(int(cs[a]), int(a), int(b)) for a, b in zip(starts, ends)])
                    sel = sel[perm]
                ns.set_fused_folds(_interleave(_take(mT, sel), _take(mB, sel)))
                multi = _take(multi, np.nonzero(np.repeat(~fg, 2))[0])
        elif self.nodesets.n_fused:
            raise RuntimeError("fused node sets without multi-folds")
        self._nodesets_enqueued = False
        if early_nodesets:
            # the node sets (and the folds applied with them) need nothing built below: enqueued
            # now, they run while the rest of the descriptors are made; launch() then skips them once
            self.nodesets.launch(waves)
            self._nodesets_enqueued = True
        self.multi_host = multi
        self.n_multi = len(multi)
        self.multi_d = _dev(multi.view(np.uint8), dev) if len(multi) else None
        folds = np.concatenate(fold_parts)
        nf = len(folds)
        self.n_folds = nf
        self.folds_host = folds
        self.fold_singles = np.concatenate([folds, expand_multi(multi)])
        self.folds_d = _dev(folds.view(np.uint8), dev)
        self.ops, self.wl_cache = ops, wl_cache
        # 4. bilinear form descriptors
        self.n_forms = 2 * T * P
        self.forms_d = _dev(forms.view(np.uint8), dev)
        self.n_tail = plans.n_tail_dev
        # rows [0, n_forms): bilinear forms (direct, exchange interleaved); then one row per device tail
        self.out = torch.empty((self.n_forms + self.n_tail, nl), dtype=torch.float64, device=dev)
        if self.n_tail:
            self.moments_d = _dev(np.ascontiguousarray(plans.moments), dev)
            self.tails_d = _dev(self.tail_records(_ptr(self.out), self.n_forms).view(np.uint8), dev)
        self.ds = diag_scale(job.L_max)
        self.forms_host = forms
        # the direct forms on a transition's full-grid b go through its multipole potential
        b_full_p = Op + row * (np.uint64(SL * T * P) + np.arange(T, dtype=np.uint64))
        d_rows = np.arange(0, 2 * T * P, 2, dtype=np.int64)
        d_t = d_rows // (2 * P)
        via_pot = (forms["b"][d_rows] == b_full_p[d_t]) & (forms["n_cols"][d_rows] == N) & (forms["n_rows"][d_rows] > 0)
        pot_b = np.where(np.bincount(d_t[via_pot], minlength=T) > 0, b_full_p, np.uint64(0))
        tc = engine in TC_TERMS
        ss_fo = d_rows[~via_pot] if tc else np.sort(np.concatenate([d_rows[~via_pot], d_rows + 1]))
        self.direct_plan = DirectPlan(pot_b=pot_b, dot_fo=d_rows[via_pot], dot_t=d_t[via_pot], ss_fo=ss_fo)
        self.early_direct = None
        if engine == "semisep":
            dp = self.direct_plan
            self.form_launch = FormLaunch([(forms, dp, N, _ptr(dg.r), dp.dot_fo, dp.ss_fo)], self.out, nl, dev)
            if early_direct and len(dp.ss_fo) and bool(np.all(dp.ss_fo % 2 == 1)):
                # every direct form goes through the potentials and dot forms, so the direct rows are
                # final before the semiseparable (exchange) forms run
                self.early_direct = {
                    "dev": torch.empty((T * P, nl), dtype=torch.float64, device=dev),
                    "host": torch.empty((T * P, nl), dtype=torch.float64, pin_memory=True),
                    "tails": torch.empty((max(1, self.n_tail), nl), dtype=torch.float64, pin_memory=True),
                    "event": torch.cuda.Event(), "done": None}
        if engine in TC_TERMS:
            # direct forms: potentials and dot products, the rest exact O(N L); exchange forms: tensor cores
            self.forms_ex_d = _dev(np.ascontiguousarray(forms[1::2]).view(np.uint8), dev)
            self.out_dir = torch.empty((T * P, nl), dtype=torch.float64, device=dev)
            self.out_ex = torch.empty((T * P, nl), dtype=torch.float64, device=dev)
            self.tc_guard = TCGuard(self.forms_ex_d, T * P, nl, dev, np.repeat(np.arange(T), P), tc_route_fraction())
            dp = self.direct_plan
            self.form_launch = FormLaunch([(forms, dp, N, _ptr(dg.r), dp.dot_fo // 2, dp.ss_fo // 2)], self.out_dir,
                                          nl, dev)
            ws = int(lib.dwba_tc_workspace_bytes(T * P, N, job.L_max, TC_TERMS[engine]))
            if ws < 0:
                raise ValueError("invalid tensor-core form sizes")
            self.tc_ws = torch.empty(max(ws, 256), dtype=torch.uint8, device=dev)
            self.tc_status = torch.zeros(1, dtype=torch.int32, device=dev)
        if engine == "dense":
            m = np.maximum(forms["n_rows"], forms["n_cols"]).astype(np.int32)
            prefix = np.zeros(self.n_forms + 1, dtype=np.int64)
            n_cta = lib.dwba_dense_chunk_prefix(m.ctypes.data, self.n_forms, prefix.ctypes.data)
            if n_cta < 0:
                raise ValueError("invalid form sizes")
            self.n_cta = int(n_cta)
            self.prefix_d = _dev(prefix, dev)
            self.partial = torch.empty(self.n_cta * nl, dtype=torch.float64, device=dev)

    def tail_records(self, out_ptr: int, row0: int) -> np.ndarray:
        """Device tail records writing rows row0.. of a (rows, L_max+1) float64 buffer at out_ptr."""
        pl, nl = self.plans, self.nl
        n = pl.n_tail_dev
        rec = np.zeros(n, dtype=_lib.TAIL_DTYPE)
        if n:
            rec["wave"] = pl.tail_wave
            rec["r_m"], rec["r_max"], rec["mode"] = pl.tail_rm, pl.tail_rmax, pl.tail_mode
            rec["moments"] = np.uint64(_ptr(self.moments_d)) + np.uint64(8 * nl) * pl.tail_tp[:, 0].astype(np.uint64)
            rec["out"] = np.uint64(out_ptr) + np.uint64(8 * nl) * (np.uint64(row0) + np.arange(n, dtype=np.uint64))
        return rec

    def launch_tails(self) -> None:
        if self.n_tail and self.job.L_max >= 1:
            seg, dphi = self.plans.tail_limits
            _lib.check(self.lib.dwba_outer_tails_batch(_ptr(self.tails_d), self.n_tail, self.job.L_max, seg, dphi,
                                                       _stream()), "dwba_outer_tails_batch")

    def add_host_terms(self, I_dir, I_exc, tail_rows) -> None:
        """Outer tails (host- and device-evaluated) and L=0 corrections, then the non-finite guard."""
        self.add_direct_host_terms(I_dir, tail_rows)
        self.add_exchange_host_terms(I_exc)

    def add_direct_host_terms(self, I_dir, tail_rows) -> None:
        pl = self.plans
        for (ti, p_i), tail in pl.tails.items():
            I_dir[ti, p_i] += tail
        if self.n_tail:
            I_dir[pl.tail_tp[:, 0], pl.tail_tp[:, 1], 1:] += tail_rows[:, 1:]
        I_dir[:, :, 0] += pl.corr_dir
        I_dir[~np.isfinite(I_dir)] = 0.0

    def add_exchange_host_terms(self, I_exc) -> None:
        I_exc[:, :, 0] += self.plans.corr_ex
        I_exc[~np.isfinite(I_exc)] = 0.0

    def launch_folds(self) -> None:
        lib, nf = self.lib, self.n_folds
        for s0 in range(0, nf, 65535):
            n = min(65535, nf - s0)
            _lib.check(lib.dwba_fold(_ptr(self.folds_d) + s0 * _lib.FOLD_DTYPE.itemsize, n, self.job.grid.N,
                                     _stream()), "dwba_fold")
        for s0 in range(0, self.n_multi, 65535):
            n = min(65535, self.n_multi - s0)
            _lib.check(lib.dwba_fold_multi(_ptr(self.multi_d) + s0 * _lib.FOLD_MULTI_DTYPE.itemsize, n,
                                           self.job.grid.N, _stream()), "dwba_fold_multi")

    def launch_forms_direct(self) -> None:
        """Tensor-core engines: the direct forms share b per transition and take the exact FP64 path
        (multipole potentials and dot products; semiseparable forms for the rest)."""
        g = self.job.grid
        self.form_launch.launch(self.lib, self.job.L_max, self.ds, float(g.r[0]), float(g.r[-1]))

    def launch_forms_exchange(self) -> None:
        """Tensor-core engines: exchange forms on tcgen05 (split bf16 K_L B, FP64 epilogue), then the
        accuracy guard (forms with strong cancellation recomputed in FP64)."""
        job, g = self.job, self.job.grid
        _lib.check(self.lib.dwba_bilinear_tc_bf16(_ptr(self.forms_ex_d), self.T * self.P, _ptr(self.dg.r), g.N,
                                                  job.L_max, TC_TERMS[self.engine], self.ds.ctypes.data,
                                                  _ptr(self.tc_ws), self.tc_ws.numel(), _ptr(self.tc_status),
                                                  _ptr(self.out_ex), _stream()), "dwba_bilinear_tc_bf16")
        self.tc_guard.launch(self.lib, job.L_max, self.ds, float(g.r[0]), float(g.r[-1]), self.out_ex)

    def tensor_flops(self) -> Tuple[float, float]:
        """(dense-equivalent, executed) tensor flops of the exchange forms per launch."""
        N = self.job.grid.N
        n_pad = (N + 63) // 64 * 64
        bn = 256
        f_pad = (self.T * self.P + bn - 1) // bn * bn
        n_iblk = (N + 127) // 128
        prods = 3 if TC_TERMS[self.engine] == 2 else 6
        useful = float(np.sum(2.0 * self.forms_host["n_rows"][1::2].astype(np.float64) *
                              self.forms_host["n_cols"][1::2])) * self.nl
        executed = 2.0 * (n_iblk * 128) * n_pad * f_pad * self.nl * prods
        return useful, executed

    def launch_forms(self) -> None:
        lib, job = self.lib, self.job
        if self.engine in TC_TERMS:
            self.launch_forms_direct()
            self.launch_forms_exchange()
            return
        if self.engine == "dense":
            _lib.check(lib.dwba_bilinear_dense_fp64(_ptr(self.forms_d), self.n_forms, job.L_max, self.ds.ctypes.data,
                                                    _ptr(self.prefix_d), self.n_cta, _ptr(self.partial),
                                                    self.partial.numel(), _ptr(self.out), _stream()),
                       "dwba_bilinear_dense_fp64")
        else:
            self.form_launch.launch(lib, job.L_max, self.ds, float(job.grid.r[0]), float(job.grid.r[-1]))

    def launch(self) -> None:
        if self._nodesets_enqueued:
            self._nodesets_enqueued = False  # enqueued by the constructor (early_nodesets)
        else:
            self.nodesets.launch(self.waves)  # stored sets at once, fused sets as their waves arrive
        self.waves.wait_ready()
        if self.early_direct is not None:
            # direct forms and tails first; their rows go back to the host while the exchange
            # forms run (collect_direct)
            self.launch_folds()
            job = self.job
            self.form_launch.launch(self.lib, job.L_max, self.ds, float(job.grid.r[0]), float(job.grid.r[-1]),
                                    parts=("potentials", "dots"))
            self.launch_tails()
            ed = self.early_direct
            ed["dev"].copy_(self.out[0:self.n_forms:2])
            ed["host"].copy_(ed["dev"], non_blocking=True)
            if self.n_tail:
                ed["tails"].copy_(self.out[self.n_forms:], non_blocking=True)
            ed["event"].record()
            ed["done"] = None
            self.form_launch.launch(self.lib, job.L_max, self.ds, float(job.grid.r[0]), float(job.grid.r[-1]),
                                    parts=("semisep",))
            return
        self.launch_folds()
        self.launch_forms()
        self.launch_tails()

    def algorithmic_flops(self) -> float:
        """Dense-equivalent work: 2 n_rows n_cols flops per (form, L)."""
        f = self.forms_host
        return float(np.sum(2.0 * f["n_rows"].astype(np.float64) * f["n_cols"])) * self.nl

    def fold_bytes(self) -> float:
        """Bytes the fold launches must move at least once: every distinct operand array (band
        operator, density factors) read over its longest use, and every output written. Arrays
        several folds share (a bound state, one pair's operator) count once."""
        reads: Dict[int, float] = {}
        writes = 0.0

        def rd(ptrs, lengths):
            for p_, n_ in zip(np.asarray(ptrs).ravel().tolist(), np.asarray(lengths, dtype=np.float64).ravel().tolist()):
                if p_ and n_ > reads.get(p_, 0.0):
                    reads[p_] = n_
        f = self.folds_host
        if len(f):
            rd(f["op"], (2.0 * f["half_band"] + 1.0) * f["n_out"])
            rd(f["f"], f["n_src"])
            rd(f["g"], f["n_src"])
            writes += float(np.sum(f["n_clear"].astype(np.float64)))
        m = self.multi_host
        if len(m):
            rd(m["op"], (2.0 * m["half_band"] + 1.0) * m["n_out"])
            rd(m["g"], m["n_src"])
            for t in range(_lib.FOLD_MULTI):
                use = m["n_f"] > t
                rd(m["f"][use, t], m["n_src"][use])
                writes += float(np.sum(m["n_clear"][use].astype(np.float64)))
        return 8.0 * (sum(reads.values()) + writes)

    def algorithmic_bytes(self) -> float:
        """Operand bytes of the exact evaluation: potentials (b and r read, rows written), dot forms
        (a read once, each potential tile once per run) and semiseparable forms (a, b and r)."""
        fl = getattr(self, "form_launch", None)
        if fl is not None and self.engine == "semisep":
            return fl.algorithmic_bytes()
        f = self.forms_host
        m = np.maximum(f["n_rows"], f["n_cols"]).astype(np.float64)
        return float(np.sum(8.0 * (f["n_rows"].astype(np.float64) + f["n_cols"] + m)))

    def collect_direct(self) -> np.ndarray:
        """I_dir as a (T, P, L_max+1) array as soon as the direct forms and tails have run (their
        rows are copied back before the exchange forms), for a caller that handles them while the
        device finishes; ``collect()`` then returns the same array. Only with ``early_direct``."""
        ed = self.early_direct
        if ed is None:
            raise RuntimeError("collect_direct: this job evaluates its direct forms with the exchange forms")
        if ed["done"] is None:
            ed["event"].synchronize()
            I_dir = ed["host"].numpy().reshape(self.T, self.P, self.nl).copy()
            self.add_direct_host_terms(I_dir, ed["tails"].numpy() if self.n_tail else None)
            ed["done"] = I_dir
        return ed["done"]

    def collect(self):
        """(I_dir, I_exc) as (T, P, L_max+1) float64 arrays."""
        nf = self.n_forms
        if self.early_direct is not None:
            I_dir = self.collect_direct()
            res = self.out[1:nf:2].cpu().numpy()  # synchronises
            self.nodesets.check()
            I_exc = res.reshape(self.T, self.P, self.nl).copy()
            self.add_exchange_host_terms(I_exc)
            return I_dir, I_exc
        if self.engine in TC_TERMS:
            self.out[0:nf:2] = self.out_dir
            self.out[1:nf:2] = self.out_ex
        res = self.out.cpu().numpy()  # single device->host transfer (synchronises)
        self.nodesets.check()
        if self.engine in TC_TERMS and int(self.tc_status.item()) != 0:
            raise _lib.DWBAError(_lib.DWBA_ERR_RANGE, "dwba_bilinear_tc_bf16: a bounded wait expired")
        T, P, nl = self.T, self.P, self.nl
        I_dir = res[0:nf:2].reshape(T, P, nl).copy()
        I_exc = res[1:nf:2].reshape(T, P, nl).copy()
        self.add_host_terms(I_dir, I_exc, res[nf:])
        return I_dir, I_exc


class MultiPrepared:
    """Several prepared jobs (typically one per energy point, each with its own grid) evaluated
    with shared launches: one node-set launch, one fold launch and one bilinear-form launch for
    all of them (every descriptor carries its own grid pointer and sizes). The launch sequence
    does no host synchronisation and no allocation, so it can be captured in a CUDA graph and
    replayed (``capture()`` / ``replay()``). With the tensor-core engines the exchange forms of all
    jobs go in one ragged tensor-core launch (one segment per grid)."""

    def __init__(self, parts: List[PreparedJob]):
        if not parts:
            raise ValueError("no jobs")
        self.parts = parts
        self.engine = parts[0].engine
        if any(p.engine != self.engine for p in parts):
            raise ValueError("all jobs of a batch use one engine")
        dev = parts[0].dg.device
        self.lib = _lib.load()
        self.L_max = max(p.job.L_max for p in parts)
        if any(p.job.L_max != self.L_max for p in parts):
            raise ValueError("all jobs of a batch share L_max")
        self.nl = self.L_max + 1
        # node sets of every part (each record names its own grid); fused sets with their folds
        recs = [p.nodesets.recs for p in parts if p.nodesets.n]
        self.n_sets = int(sum(len(r) for r in recs))
        frecs = [p.nodesets.fused_recs for p in parts if p.nodesets.n_fused]
        self.n_fused = int(sum(len(r) for r in frecs))
        self.max_grid = max(p.job.grid.N for p in parts)
        if self.n_sets or self.n_fused:
            cc = {p.nodesets.n_cc for p in parts if p.nodesets.n or p.nodesets.n_fused}
            if len(cc) != 1:
                raise ValueError("all jobs of a batch share CC_nodes")
            self.n_cc = cc.pop()
            self.ccx, self.ccw = CCTables.get(self.n_cc, dev)
            self.ns_status = torch.zeros(1, dtype=torch.int32, device=dev)
        if self.n_sets:
            self.recs_d = _dev(np.concatenate(recs).view(np.uint8), dev)
        if self.n_fused:
            self.frecs_d = _dev(np.concatenate(frecs).view(np.uint8), dev)
            self.ffolds_d = _dev(np.concatenate([p.nodesets.fused_folds for p in parts if p.nodesets.n_fused])
                                 .view(np.uint8), dev)
        folds = np.concatenate([p.folds_host for p in parts])
        self.n_folds = len(folds)
        self.folds_d = _dev(folds.view(np.uint8), dev)
        multi = np.concatenate([p.multi_host for p in parts])
        self.n_multi = len(multi)
        self.multi_d = _dev(multi.view(np.uint8), dev) if len(multi) else None
        forms = np.concatenate([p.forms_host for p in parts])
        self.n_forms = len(forms)
        self.forms_host = forms
        self.forms_d = _dev(forms.view(np.uint8), dev)
        self.n_tail = int(sum(p.n_tail for p in parts))
        self.out = torch.empty((self.n_forms + self.n_tail, self.nl), dtype=torch.float64, device=dev)
        self.ds = diag_scale(self.L_max)
        self.offsets = np.cumsum([0] + [p.n_forms for p in parts])
        self.tail_offsets = self.n_forms + np.cumsum([0] + [p.n_tail for p in parts])
        if self.n_tail:
            trec = np.concatenate([p.tail_records(_ptr(self.out), int(self.tail_offsets[k]))
                                   for k, p in enumerate(parts)])
            self.tails_d = _dev(trec.view(np.uint8), dev)
            self.tail_limits = parts[0].plans.tail_limits
        self.r_min = min(float(p.job.grid.r[0]) for p in parts)
        self.r_max = max(float(p.job.grid.r[-1]) for p in parts)
        if self.engine == "dense":
            m = np.maximum(forms["n_rows"], forms["n_cols"]).astype(np.int32)
            prefix = np.zeros(self.n_forms + 1, dtype=np.int64)
            self.n_cta = int(self.lib.dwba_dense_chunk_prefix(m.ctypes.data, self.n_forms, prefix.ctypes.data))
            if self.n_cta < 0:
                raise ValueError("invalid form sizes")
            self.prefix_d = _dev(prefix, dev)
            self.partial = torch.empty(self.n_cta * self.nl, dtype=torch.float64, device=dev)
        self.graph = None
        if self.engine == "semisep":
            # one potential launch, one dot-form launch and one semiseparable launch for all jobs
            ent = [(p.forms_host, p.direct_plan, p.job.grid.N, _ptr(p.dg.r), self.offsets[k] + p.direct_plan.dot_fo,
                    self.offsets[k] + p.direct_plan.ss_fo) for k, p in enumerate(parts)]
            self.form_launch = FormLaunch(ent, self.out, self.nl, dev)
        # tensor-core engines: the direct forms of every job in one exact launch sequence (each
        # descriptor names its own grid); the exchange forms of all jobs in ONE ragged tensor-core
        # launch (one segment per distinct grid, so the transitions of an energy share the form
        # tiles), then one accuracy guard over all of them; the jobs' tails go round-robin (largest
        # grid first) over side streams forked from and joined back into the launching stream.
        # The jobs' own direct / exchange output rows become views of the shared ones (jobs of a
        # MultiPrepared are launched through it only).
        self.side_streams = []
        self.tc_order = []
        self.tc = None
        if self.engine in TC_TERMS:
            nt = TC_TERMS[self.engine]
            self.side_streams = [torch.cuda.Stream(device=dev) for _ in range(min(4, len(parts)))]
            self.tc_order = sorted(range(len(parts)), key=lambda k: -parts[k].job.grid.N)
            n_dir = int(sum(p.T * p.P for p in parts))
            self.tc_out_dir = torch.empty((n_dir, self.nl), dtype=torch.float64, device=dev)
            d_off = np.cumsum([0] + [p.T * p.P for p in parts])
            ent = [(p.forms_host, p.direct_plan, p.job.grid.N, _ptr(p.dg.r), d_off[k] + p.direct_plan.dot_fo // 2,
                    d_off[k] + p.direct_plan.ss_fo // 2) for k, p in enumerate(parts)]
            self.form_launch = FormLaunch(ent, self.tc_out_dir, self.nl, dev)
            off = 0
            for k, p in enumerate(parts):
                n = p.T * p.P
                p.out_dir = self.tc_out_dir[off:off + n]
                off += n
            by_grid: Dict[tuple, List[int]] = {}
            for k, p in enumerate(parts):
                r = np.ascontiguousarray(p.job.grid.r, dtype=np.float64)
                by_grid.setdefault((len(r), hashlib.sha1(r.tobytes()).hexdigest()), []).append(k)
            groups = sorted(by_grid.values(), key=lambda v: -parts[v[0]].job.grid.N)
            order = [k for ks in groups for k in ks]  # the jobs' exchange forms, grouped by grid
            fe = np.concatenate([np.ascontiguousarray(parts[k].forms_host[1::2]) for k in order])
            n_ex = len(fe)
            self.tc = {"forms": _dev(fe.view(np.uint8), dev), "n": n_ex, "nt": nt,
                       "status": torch.zeros(1, dtype=torch.int32, device=dev),
                       "out": torch.empty((n_ex, self.nl), dtype=torch.float64, device=dev)}
            fbase, obase = _ptr(self.tc["forms"]), _ptr(self.tc["out"])
            segs = np.zeros(len(groups), dtype=_lib.TC_SEGMENT_DTYPE)
            f0 = 0
            for q, ks in enumerate(groups):
                n = int(sum(parts[k].T * parts[k].P for k in ks))
                segs[q] = (fbase + f0 * _lib.FORM_DTYPE.itemsize, _ptr(parts[ks[0]].dg.r),
                           obase + f0 * 8 * self.nl, n, parts[ks[0]].job.grid.N)
                f0 += n
            self.tc["segs"] = segs
            self.set_tile(None)
            off = 0
            gids, g0 = [], 0
            for k in order:
                p = parts[k]
                n = p.T * p.P
                p.out_ex = self.tc["out"][off:off + n]
                p.tc_status = self.tc["status"]
                p.tc_ws = None  # the shared workspace serves it
                off += n
                gids.append(g0 + np.repeat(np.arange(p.T), p.P))  # transition of each form
                g0 += p.T
            self.tc["guard"] = TCGuard(self.tc["forms"], n_ex, self.nl, dev, np.concatenate(gids),
                                       tc_route_fraction())
            self.r_lo_tc = min(float(p.job.grid.r[0]) for p in parts)
            self.r_hi_tc = max(float(p.job.grid.r[-1]) for p in parts)

    def launch_tensor(self) -> None:
        """The ragged tensor-core launch alone, on the current stream (for timing its tiles)."""
        tc = self.tc
        segs = tc["segs"]
        _lib.check(self.lib.dwba_bilinear_tc_bf16_ragged(segs.ctypes.data, len(segs), self.L_max, tc["nt"],
                                                         tc["tile"].ctypes.data, self.ds.ctypes.data, _ptr(tc["ws"]),
                                                         tc["ws"].numel(), _ptr(tc["status"]), _stream()),
                   "dwba_bilinear_tc_bf16_ragged")

    def set_tile(self, tile: Optional[dict]) -> None:
        """Tile of the ragged tensor-core launch: dict(bn=128|256, stages=..., order=0|1) or None for the
        default; (re)sizes the shared workspace. Capture the graph again after a change."""
        if self.tc is None:
            return
        t = np.zeros(1, dtype=_lib.TC_TILE_DTYPE)
        if tile:
            t["bn"], t["stages"], t["order"] = tile.get("bn", 0), tile.get("stages", 0), tile.get("order", 0)
        segs = self.tc["segs"]
        ws = int(self.lib.dwba_tc_ragged_workspace_bytes(segs.ctypes.data, len(segs), self.L_max, self.tc["nt"],
                                                          t.ctypes.data))
        if ws < 0:
            raise ValueError(f"invalid tensor-core tile or form sizes: {tile}")
        old = self.tc.get("ws")
        if old is None or old.numel() < ws:
            self.tc["ws"] = torch.empty(max(ws, 256), dtype=torch.uint8, device=self.parts[0].dg.device)
        self.tc["tile"] = t
        self.tile = dict(tile) if tile else None

    def launch(self, marks: Optional[list] = None) -> None:
        """The launch sequence. With ``marks`` (a list), a CUDA event is recorded on the stream after
        each stage and appended as (stage, event): "start", "nodesets", "folds", "forms", "tails"."""
        lib = self.lib
        st = _stream()

        def mark(name):
            if marks is not None:
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(torch.cuda.current_stream())
                marks.append((name, ev))
        for p in self.parts:
            p.waves.wait_ready()
        mark("start")
        if self.n_sets:
            for s0 in range(0, self.n_sets, 65535):
                n = min(65535, self.n_sets - s0)
                _lib.check(lib.dwba_build_nodesets(_ptr(self.recs_d) + s0 * _lib.NODESET_DTYPE.itemsize, n,
                                                   self.max_grid, _ptr(self.ccx), _ptr(self.ccw), self.n_cc,
                                                   _ptr(self.ns_status), st), "dwba_build_nodesets")
        for s0 in range(0, self.n_fused, 65535):
            n = min(65535, self.n_fused - s0)
            _lib.check(lib.dwba_build_nodesets_folded(_ptr(self.frecs_d) + s0 * _lib.NODESET_DTYPE.itemsize,
                                                      _ptr(self.ffolds_d) + 2 * s0 * _lib.FOLD_MULTI_DTYPE.itemsize,
                                                      n, self.max_grid, _ptr(self.ccx), _ptr(self.ccw), self.n_cc,
                                                      _ptr(self.ns_status), st), "dwba_build_nodesets_folded")
        mark("nodesets")
        for s0 in range(0, self.n_folds, 65535):
            n = min(65535, self.n_folds - s0)
            _lib.check(lib.dwba_fold(_ptr(self.folds_d) + s0 * _lib.FOLD_DTYPE.itemsize, n, self.max_grid, st),
                       "dwba_fold")
        for s0 in range(0, self.n_multi, 65535):
            n = min(65535, self.n_multi - s0)
            _lib.check(lib.dwba_fold_multi(_ptr(self.multi_d) + s0 * _lib.FOLD_MULTI_DTYPE.itemsize, n,
                                           self.max_grid, st), "dwba_fold_multi")
        mark("folds")
        if self.engine == "dense":
            _lib.check(lib.dwba_bilinear_dense_fp64(_ptr(self.forms_d), self.n_forms, self.L_max, self.ds.ctypes.data,
                                                    _ptr(self.prefix_d), self.n_cta, _ptr(self.partial),
                                                    self.partial.numel(), _ptr(self.out), st),
                       "dwba_bilinear_dense_fp64")
        elif self.engine == "semisep":
            self.form_launch.launch(lib, self.L_max, self.ds, self.r_min, self.r_max)
        else:
            main = torch.cuda.current_stream()
            nt = TC_TERMS[self.engine]
            for stage in ("forms", "tails"):
                for sd in self.side_streams:
                    sd.wait_stream(main)
                if stage == "forms":
                    # direct forms on the main stream, beside the one ragged tensor-core launch (and
                    # its guard) on a side stream
                    self.form_launch.launch(lib, self.L_max, self.ds, self.r_min, self.r_max)
                    tc = self.tc
                    sd = self.side_streams[0]
                    segs = tc["segs"]
                    _lib.check(lib.dwba_bilinear_tc_bf16_ragged(segs.ctypes.data, len(segs), self.L_max, nt,
                                                                tc["tile"].ctypes.data, self.ds.ctypes.data,
                                                                _ptr(tc["ws"]), tc["ws"].numel(), _ptr(tc["status"]),
                                                                int(sd.cuda_stream)),
                               "dwba_bilinear_tc_bf16_ragged")
                    with torch.cuda.stream(sd):
                        tc["guard"].launch(lib, self.L_max, self.ds, self.r_lo_tc, self.r_hi_tc, tc["out"])
                else:
                    for q, k in enumerate(self.tc_order):
                        with torch.cuda.stream(self.side_streams[q % len(self.side_streams)]):
                            self.parts[k].launch_tails()
                for sd in self.side_streams:
                    main.wait_stream(sd)
                mark(stage)
            return
        mark("forms")
        if self.n_tail and self.L_max >= 1:
            seg, dphi = self.tail_limits
            _lib.check(lib.dwba_outer_tails_batch(_ptr(self.tails_d), self.n_tail, self.L_max, seg, dphi, st),
                       "dwba_outer_tails_batch")
        mark("tails")

    def capture(self) -> None:
        """Record the launch sequence once in a CUDA graph (warm-up launch first)."""
        self.launch()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch()
        self.graph = g

    def replay(self) -> None:
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def collect(self):
        """[(I_dir, I_exc) per part], each (T, P, L_max+1)."""
        if self.engine in TC_TERMS:
            return [p.collect() for p in self.parts]
        res = self.out.cpu().numpy()
        if (self.n_sets or self.n_fused) and int(self.ns_status.item()) != 0:
            raise _lib.DWBAError(_lib.DWBA_ERR_RANGE, "dwba_build_nodesets")
        outs = []
        for k, p in enumerate(self.parts):
            part = res[self.offsets[k]:self.offsets[k + 1]]
            T, P, nl = p.T, p.P, p.nl
            I_dir = part[0::2].reshape(T, P, nl).copy()
            I_exc = part[1::2].reshape(T, P, nl).copy()
            p.add_host_terms(I_dir, I_exc, res[self.tail_offsets[k]:self.tail_offsets[k + 1]])
            outs.append((I_dir, I_exc))
        return outs
