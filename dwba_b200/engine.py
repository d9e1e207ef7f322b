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

import ctypes
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .plan import (GridInfo, NodeSetKey, NodeSetPlan, OVERLAP_TOL, adaptive_dphi, cc_reference, diag_scale,
                   idx_limit, is_excitation, multipole_moments, plan_nodeset, safe_float, tail_limits)

ENGINES = ("dense", "semisep")


def _ptr(t: Optional[torch.Tensor]) -> int:
    return 0 if t is None else int(t.data_ptr())


def _stream() -> int:
    return int(torch.cuda.current_stream().cuda_stream)


def _require_device():
    if not torch.cuda.is_available():
        raise RuntimeError("dwba_b200: no CUDA device is available (the engine has no CPU fallback)")
    _lib.load()


def _dev(x: np.ndarray, device) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(x)).to(device, non_blocking=False)


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


@dataclass
class DeviceNodeSet:
    plan: NodeSetPlan
    ta: torch.Tensor
    bx: torch.Tensor
    nbytes: int


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


class NodeSetBatch:
    """Descriptors of the node sets a job uses; ``launch()`` (re)builds their banded operators."""

    def __init__(self, dg: DeviceGrid, plans: Sequence[NodeSetPlan], n_cc: int, rebuild: bool = False):
        self.dg, self.n_cc = dg, n_cc
        dev = dg.device
        N = dg.info.N
        todo = list(plans) if rebuild else [p for p in plans if p.key not in dg.nodesets]
        self.n = len(todo)
        if not todo:
            return
        self.ccx, self.ccw = CCTables.get(n_cc, dev)
        recs = np.zeros(len(todo), dtype=_lib.NODESET_DTYPE)
        self.keep = []
        for i, p in enumerate(todo):
            old = dg.nodesets.get(p.key)
            ta = old.ta if old is not None else torch.empty(3 * p.key.n1, dtype=torch.float64, device=dev)
            bx = old.bx if old is not None else torch.empty(5 * N, dtype=torch.float64, device=dev)
            br = _dev(p.breaks, dev) if p.breaks is not None else None
            self.keep.append(br)
            recs[i] = (_ptr(dg.r), _ptr(dg.logr), _ptr(br), _ptr(ta), _ptr(bx), N, p.key.n1, p.n_breaks,
                       int(p.log1), int(p.log2), 0)
            dg.nodesets[p.key] = DeviceNodeSet(p, ta, bx, 8 * (3 * p.key.n1 + 5 * N))
        self.recs_d = _dev(recs.view(np.uint8), dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)

    def launch(self) -> None:
        if self.n == 0:
            return
        lib = _lib.load()
        N = self.dg.info.N
        for s0 in range(0, self.n, 65535):
            n = min(65535, self.n - s0)
            _lib.check(lib.dwba_build_nodesets(_ptr(self.recs_d) + s0 * _lib.NODESET_DTYPE.itemsize, n, N,
                                               _ptr(self.ccx), _ptr(self.ccw), self.n_cc, _ptr(self.status),
                                               _stream()), "dwba_build_nodesets")

    def check(self) -> None:
        if self.n and int(self.status.item()) != 0:
            raise _lib.DWBAError(_lib.DWBA_ERR_RANGE, "dwba_build_nodesets")


@dataclass
class PairPlan:
    n1: int
    osc: bool
    nodeset: Optional[NodeSetPlan]
    corr_dir: float = 0.0
    corr_ex: float = 0.0
    tail: Optional[np.ndarray] = None


@dataclass
class Job:
    """One energy point: shared grid/potentials/transition, many continuum pairs."""
    grid: GridInfo
    V_core: np.ndarray
    U_i: np.ndarray
    U_f: Optional[np.ndarray]
    u_i: np.ndarray
    u_f: np.ndarray
    excitation: bool
    pairs: List[Tuple[object, object]]
    L_max: int
    use_oscillatory_quadrature: bool = True
    oscillatory_method: str = "advanced"
    CC_nodes: int = 5
    phase_increment: float = 1.5708
    min_grid_fraction: float = 0.10
    k_threshold: float = 0.5


def plan_job(job: Job) -> List[PairPlan]:
    """Host planning of every pair (integration limit, branch, node set, L=0 corrections, tails)."""
    g = job.grid
    N = g.N
    r, w = g.r, g.w
    V_diff = job.V_core - job.U_i
    moments = None
    max_seg, max_dphi = tail_limits()
    plans = []
    for ci, cf in job.pairs:
        k_i, k_f, l_i, l_f = float(ci.k_au), float(cf.k_au), int(ci.l), int(cf.l)
        n1 = idx_limit(g, job.U_i, job.U_f, job.u_i, job.u_f, k_i, k_f, l_i, l_f,
                       int(getattr(ci, "idx_match", -1)), int(getattr(cf, "idx_match", -1)), job.min_grid_fraction)
        e_i, e_f = float(getattr(ci, "eta", 0.0)), float(getattr(cf, "eta", 0.0))
        k_total, eta_total = k_i + k_f, e_i + e_f
        osc = bool(job.use_oscillatory_quadrature and k_total > job.k_threshold)
        ns = None
        if osc and n1 >= 2:
            d = adaptive_dphi(g, n1, k_total, job.phase_increment, eta_total)
            ns = plan_nodeset(g, NodeSetKey(id(g), n1, k_total, d, eta_total, int(job.CC_nodes)))
        pp = PairPlan(n1=n1, osc=osc, nodeset=ns)
        # L=0 corrections with the limited Simpson weights (dwba_matrix_elements.py:1028-1046, :1249-1296)
        wl = w.copy()
        wl[n1:] = 0.0
        chi_i, chi_f = ci.chi_of_r[:N], cf.chi_of_r[:N]
        s2 = np.sum(wl * job.u_f * job.u_i)
        if abs(s2) > OVERLAP_TOL:
            pp.corr_dir = float(np.dot(wl * chi_f * chi_i, V_diff) * s2)
        s2e = np.sum(wl * chi_f * job.u_i)
        if abs(s2e) > OVERLAP_TOL:
            pp.corr_ex = float(np.dot(wl * job.u_f * chi_i, V_diff) * s2e)
        # outer tails of the direct term (dwba_matrix_elements.py:1213-1241 advanced/full_split; :1256-1267 legacy)
        legacy = job.oscillatory_method == "legacy"
        want = job.L_max >= 1 and n1 < N - 10 and job.excitation and (
            (legacy and job.use_oscillatory_quadrature) or (not legacy and osc))
        if want:
            if moments is None:
                moments = multipole_moments(g, job.u_i, job.u_f, job.L_max)
            wave = [k_i, l_i, float(getattr(ci, "phase_shift", 0.0)), e_i, float(getattr(ci, "sigma_l", 0.0)),
                    k_f, l_f, float(getattr(cf, "phase_shift", 0.0)), e_f, float(getattr(cf, "sigma_l", 0.0))]
            pp.tail = _lib.outer_tails(wave, float(r[n1 - 1]), float(r[-1]), job.L_max, moments, 1 if legacy else 0,
                                       max_seg, max_dphi)
        plans.append(pp)
    return plans


class _Pool:
    """Device copies of the distinct 1-D functions of a job (dedup by host buffer)."""

    def __init__(self, device, N):
        self.device = device
        self.N = N
        self.idx: Dict[int, int] = {}
        self.host: List[np.ndarray] = []

    def add(self, arr: np.ndarray) -> int:
        a = np.ascontiguousarray(arr[: self.N], dtype=np.float64)
        key = arr.__array_interface__["data"][0]
        i = self.idx.get(key)
        if i is None:
            i = len(self.host)
            self.idx[key] = i
            self.host.append(a)
        return i

    def upload(self) -> torch.Tensor:
        stacked = np.stack(self.host) if self.host else np.zeros((1, self.N))
        pinned = torch.from_numpy(stacked).pin_memory()
        return pinned.to(self.device, non_blocking=True)


class PreparedJob:
    """A job planned on the host with its inputs and descriptors resident on the device.

    ``launch()`` enqueues every kernel on the current stream (node sets are built in
    ``__init__`` and cached per grid); ``collect()`` copies the results back once
    and adds the host-side L=0 corrections and outer tails.
    """

    def __init__(self, job: Job, dg: DeviceGrid, engine: str = "dense", plans: Optional[List[PairPlan]] = None,
                 rebuild_nodesets: bool = False):
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
        # 1. node sets (operators cached per grid and key; rebuilt every launch when rebuild_nodesets)
        uniq = {}
        for p in plans:
            if p.nodeset is not None:
                uniq.setdefault(p.nodeset.key, p.nodeset)
        self.nodesets = NodeSetBatch(dg, list(uniq.values()), job.CC_nodes, rebuild=rebuild_nodesets)
        # 2. functions on the device
        pool = _Pool(dev, N)
        iu_i, iu_f = pool.add(job.u_i), pool.add(job.u_f)
        fidx = [(pool.add(ci.chi_of_r), pool.add(cf.chi_of_r)) for ci, cf in job.pairs]
        self.F = F = pool.upload()
        self.h2d_bytes = int(F.numel()) * 8
        fptr = lambda i: _ptr(F) + 8 * N * i  # noqa: E731
        # 3. operand folds: per pair a_dir, a_ex, b_ex, b_dir(standard path); the filon b_dir is shared
        n_p = len(job.pairs)
        SL = 4
        ops = torch.empty((SL * n_p + 1, N), dtype=torch.float64, device=dev)
        op_ptr = lambda k: _ptr(ops) + 8 * N * k  # noqa: E731
        folds = np.zeros(SL * n_p + 1, dtype=_lib.FOLD_DTYPE)
        forms = np.zeros(2 * n_p, dtype=_lib.FORM_DTYPE)
        w_ptr = _ptr(dg.w)
        r_ptr = _ptr(dg.r)
        wl_cache: Dict[int, torch.Tensor] = {}

        def wl(n1):  # Simpson weights zeroed past n1 (dwba_matrix_elements.py:1025-1026)
            t = wl_cache.get(n1)
            if t is None:
                t = dg.w.clone()
                t[n1:] = 0.0
                wl_cache[n1] = t
            return t

        b_dir_full = op_ptr(SL * n_p)  # full-grid Simpson weights: the filon inner integral runs over all N
        nf = 0
        folds[nf] = (w_ptr, fptr(iu_f), fptr(iu_i), b_dir_full, 0, N, N, N)
        nf += 1
        for p_i, (pp, (ic_i, ic_f)) in enumerate(zip(plans, fidx)):
            a_dir, a_ex, b_ex, b_dir = (op_ptr(SL * p_i + k) for k in range(SL))
            n1 = pp.n1
            if pp.osc and pp.nodeset is not None:
                ns = dg.nodesets[pp.nodeset.key]
                nb = min(N, n1 + 2)
                folds[nf] = (_ptr(ns.ta), fptr(ic_f), fptr(ic_i), a_dir, 1, n1, n1, n1)
                folds[nf + 1] = (_ptr(ns.ta), fptr(iu_f), fptr(ic_i), a_ex, 1, n1, n1, n1)
                folds[nf + 2] = (_ptr(ns.bx), fptr(ic_f), fptr(iu_i), b_ex, 2, nb, N, nb)
                nf += 3
                forms[2 * p_i] = (r_ptr, a_dir, b_dir_full, n1, N)
                forms[2 * p_i + 1] = (r_ptr, a_ex, b_ex, n1, nb)
            elif pp.osc:
                # no valid phase interval: weighted dot products over r[:n1] x r[:N]
                # (oscillatory_integrals.py:2580-2587, :2694-2699)
                folds[nf] = (w_ptr, fptr(ic_f), fptr(ic_i), a_dir, 0, n1, N, n1)
                folds[nf + 1] = (w_ptr, fptr(iu_f), fptr(ic_i), a_ex, 0, n1, N, n1)
                folds[nf + 2] = (w_ptr, fptr(ic_f), fptr(iu_i), b_ex, 0, N, N, N)
                nf += 3
                forms[2 * p_i] = (r_ptr, a_dir, b_dir_full, n1, N)
                forms[2 * p_i + 1] = (r_ptr, a_ex, b_ex, n1, N)
            else:
                # standard Simpson path with limited weights (dwba_matrix_elements.py:1242-1245, :1287-1289)
                wlp = _ptr(wl(n1))
                folds[nf] = (wlp, fptr(ic_f), fptr(ic_i), a_dir, 0, n1, N, n1)
                folds[nf + 1] = (wlp, fptr(iu_f), fptr(ic_i), a_ex, 0, n1, N, n1)
                folds[nf + 2] = (wlp, fptr(ic_f), fptr(iu_i), b_ex, 0, n1, N, n1)
                folds[nf + 3] = (wlp, fptr(iu_f), fptr(iu_i), b_dir, 0, n1, N, n1)
                nf += 4
                forms[2 * p_i] = (r_ptr, a_dir, b_dir, n1, n1)
                forms[2 * p_i + 1] = (r_ptr, a_ex, b_ex, n1, n1)
        self.n_folds = nf
        self.folds_d = _dev(folds[:nf].view(np.uint8), dev)
        self.ops, self.wl_cache = ops, wl_cache
        # 4. bilinear form descriptors
        self.n_forms = 2 * n_p
        self.forms_d = _dev(forms.view(np.uint8), dev)
        self.out = torch.empty((2 * n_p, nl), dtype=torch.float64, device=dev)
        self.ds = diag_scale(job.L_max)
        self.forms_host = forms
        if engine == "dense":
            m = np.maximum(forms["n_rows"], forms["n_cols"]).astype(np.int32)
            prefix = np.zeros(2 * n_p + 1, dtype=np.int64)
            n_cta = lib.dwba_dense_chunk_prefix(m.ctypes.data, 2 * n_p, prefix.ctypes.data)
            if n_cta < 0:
                raise ValueError("invalid form sizes")
            self.n_cta = int(n_cta)
            self.prefix_d = _dev(prefix, dev)
            self.partial = torch.empty(self.n_cta * nl, dtype=torch.float64, device=dev)

    def launch_folds(self) -> None:
        lib, nf = self.lib, self.n_folds
        for s0 in range(0, nf, 65535):
            n = min(65535, nf - s0)
            _lib.check(lib.dwba_fold(_ptr(self.folds_d) + s0 * _lib.FOLD_DTYPE.itemsize, n, self.job.grid.N,
                                     _stream()), "dwba_fold")

    def launch_forms(self) -> None:
        lib, job = self.lib, self.job
        if self.engine == "dense":
            _lib.check(lib.dwba_bilinear_dense_fp64(_ptr(self.forms_d), self.n_forms, job.L_max, self.ds.ctypes.data,
                                                    _ptr(self.prefix_d), self.n_cta, _ptr(self.partial),
                                                    self.partial.numel(), _ptr(self.out), _stream()),
                       "dwba_bilinear_dense_fp64")
        else:
            _lib.check(lib.dwba_bilinear_semisep_fp64(_ptr(self.forms_d), self.n_forms, job.L_max,
                                                      self.ds.ctypes.data, float(job.grid.r[0]),
                                                      float(job.grid.r[-1]), _ptr(self.out), _stream()),
                       "dwba_bilinear_semisep_fp64")

    def launch(self) -> None:
        self.nodesets.launch()
        self.launch_folds()
        self.launch_forms()

    def algorithmic_flops(self) -> float:
        """Dense-equivalent work: 2 n_rows n_cols flops per (form, L)."""
        f = self.forms_host
        return float(np.sum(2.0 * f["n_rows"].astype(np.float64) * f["n_cols"])) * self.nl

    def collect(self):
        res = self.out.cpu().numpy()  # single device->host transfer (synchronises)
        self.nodesets.check()
        I_dir = res[0::2].copy()
        I_exc = res[1::2].copy()
        for p_i, pp in enumerate(self.plans):
            if pp.tail is not None:
                I_dir[p_i] += pp.tail
            I_dir[p_i, 0] += pp.corr_dir
            I_exc[p_i, 0] += pp.corr_ex
        I_dir[~np.isfinite(I_dir)] = 0.0
        I_exc[~np.isfinite(I_exc)] = 0.0
        return I_dir, I_exc


def run_job(job: Job, dg: DeviceGrid, engine: str = "dense", plans: Optional[List[PairPlan]] = None):
    """Evaluate every pair of a job. Returns (I_dir, I_exc) as (n_pairs, L_max+1) float64 arrays."""
    pj = PreparedJob(job, dg, engine, plans)
    pj.launch()
    return pj.collect()
