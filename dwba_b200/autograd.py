"""Differentiable radial integrals (new; the reference computes no gradients).

``RadialIntegrals`` evaluates, for one transition and a list of (cont_i, cont_f) pairs, the same
I_L^dir and I_L^exc as ``radial_ME_all_L`` (dwba_matrix_elements.py:780-1300), as a torch tensor of
shape (P, 2, L_max+1) (index 0: direct, 1: exchange) that is differentiable with respect to the
radial functions and potentials: chi_i, chi_f (P, N), u_i, u_f, V_core, U_i (N).

    I_L = a^T K_L b + c_L + t_L

* the bilinear part a^T K_L b runs on the CUDA engine forward (any engine) and backward
  (dwba_bilinear_semisep_backward_fp64: dLoss/da = K_g b, dLoss/db = K_g a with
  K_g = sum_L g_L K_L, exact FP64, or dwba_bilinear_tc_bf16_backward on the tensor cores;
  then dwba_fold_adjoint for the banded folds);
* the L=0 correction c_L (dwba_matrix_elements.py:1249-1296) and the outer tail
  t_L = tau_L M_L (dwba_matrix_elements.py:1213-1241; tau_L = tail per unit multipole moment,
  M_L = sum w r^L u_f u_i) are torch expressions, differentiated by autograd.

Held constant (piecewise constant in the inputs, or scalar wave data): the integration limit n1
(idx_limit), the phase-split node sets, the branch choices, the gates |.| > 1e-12 and the
scalar wave parameters (k, l, delta, eta, sigma) that enter the tails.
"""
from __future__ import annotations

from types import SimpleNamespace
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .dwba_matrix_elements import GPUCache, _engine_name, _make_job
from .engine import TC_TERMS, PreparedJob, plan_job
from .plan import OVERLAP_TOL

__all__ = ["RadialIntegrals"]


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _dev(a: np.ndarray, dev) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)


class _State:
    prepared: PreparedJob


class _BilinearFn(torch.autograd.Function):
    """a^T K_L b of every (pair, kind) of one prepared job; inputs are the radial functions."""

    @staticmethod
    def forward(ctx, chi_i, chi_f, u_i, u_f, state):
        pj = state.prepared
        pj.launch()
        if pj.engine in TC_TERMS:
            raw = torch.stack([pj.out_dir, pj.out_ex], dim=1)
        else:
            raw = pj.out[:pj.n_forms].view(pj.P, 2, pj.nl)
        ctx.state = state
        return raw.clone()

    @staticmethod
    def backward(ctx, gI):
        pj = ctx.state.prepared
        lib = _lib.load()
        dev = pj.F.device
        N, nl, nf = pj.job.grid.N, pj.nl, pj.n_forms
        G = gI.detach().to(torch.float64).contiguous().view(nf, nl)
        GA = torch.zeros((nf, N), dtype=torch.float64, device=dev)
        GB = torch.zeros((nf, N), dtype=torch.float64, device=dev)
        fh = pj.forms_host
        row = np.uint64(8 * N)
        idx = np.arange(nf, dtype=np.uint64)
        desc = np.zeros(nf, dtype=_lib.FORM_GRAD_DTYPE)
        desc["r"], desc["a"], desc["b"] = fh["r"], fh["a"], fh["b"]
        desc["ga"] = np.uint64(_ptr(GA)) + row * idx
        desc["gb"] = np.uint64(_ptr(GB)) + row * idx
        desc["n_rows"], desc["n_cols"] = fh["n_rows"], fh["n_cols"]
        desc_d = _dev(desc, dev)
        g = pj.job.grid
        bwd = getattr(ctx.state, "backward", "fp64")
        if bwd in TC_TERMS:
            nt = TC_TERMS[bwd]
            ws_bytes = int(lib.dwba_tc_backward_workspace_bytes(nf, N, pj.job.L_max, nt))
            if ws_bytes < 0:
                raise ValueError("invalid tensor-core form sizes")
            ws = torch.empty(max(ws_bytes, 256), dtype=torch.uint8, device=dev)
            status = torch.zeros(1, dtype=torch.int32, device=dev)
            _lib.check(lib.dwba_bilinear_tc_bf16_backward(_ptr(desc_d), nf, _ptr(pj.dg.r), N, pj.job.L_max, nt,
                                                          pj.ds.ctypes.data, _ptr(G), _ptr(ws), ws.numel(),
                                                          _ptr(status), _stream()),
                       "dwba_bilinear_tc_bf16_backward")
            if int(status.item()) != 0:
                raise _lib.DWBAError(_lib.DWBA_ERR_RANGE, "dwba_bilinear_tc_bf16_backward: a bounded wait expired")
        else:
            _lib.check(lib.dwba_bilinear_semisep_backward_fp64(_ptr(desc_d), nf, pj.job.L_max, pj.ds.ctypes.data,
                                                               _ptr(G), float(g.r[0]), float(g.r[-1]), _stream()),
                       "dwba_bilinear_semisep_backward_fp64")
        # gradients of the folded operands (rows of pj.ops), summed over the forms that read them
        ops = pj.ops
        Op = np.uint64(_ptr(ops))
        as_idx = lambda a: torch.as_tensor(np.asarray(a, dtype=np.int64), device=dev)  # noqa: E731
        gops = torch.zeros_like(ops)
        gops.index_add_(0, as_idx((fh["a"] - Op) // row), GA)
        gops.index_add_(0, as_idx((fh["b"] - Op) // row), GB)
        # adjoint of every fold: z = Op^T y, then d(f*g) -> f, g
        fo = pj.fold_singles
        nfo = len(fo)
        Z = torch.zeros((nfo, N), dtype=torch.float64, device=dev)
        adj = np.zeros(nfo, dtype=_lib.FOLD_ADJ_DTYPE)
        adj["op"] = fo["op"]
        adj["y"] = np.uint64(_ptr(gops)) + row * ((fo["out"] - Op) // row)
        adj["z"] = np.uint64(_ptr(Z)) + row * np.arange(nfo, dtype=np.uint64)
        adj["half_band"], adj["n_out"], adj["n_src"] = fo["half_band"], fo["n_out"], fo["n_src"]
        adj_d = _dev(adj, dev)
        for s0 in range(0, nfo, 65535):
            n = min(65535, nfo - s0)
            _lib.check(lib.dwba_fold_adjoint(_ptr(adj_d) + s0 * _lib.FOLD_ADJ_DTYPE.itemsize, n, N, _stream()),
                       "dwba_fold_adjoint")
        F = pj.F
        Fp = np.uint64(_ptr(F))
        f_rows = as_idx((fo["f"] - Fp) // row)
        g_rows = as_idx((fo["g"] - Fp) // row)
        grad_F = torch.zeros_like(F)
        grad_F.index_add_(0, f_rows, Z * F[g_rows])
        grad_F.index_add_(0, g_rows, Z * F[f_rows])
        wi, wf, tidx = pj.wave_rows
        return grad_F[as_idx(wi)], grad_F[as_idx(wf)], grad_F[tidx[0][0]], grad_F[tidx[0][1]], None


def _attrs(obj) -> dict:
    """Attributes of a wave/bound object (dataclass, namespace or plain object)."""
    keys = ("l", "k_au", "phase_shift", "idx_match", "eta", "sigma_l", "r_match", "energy_au", "n_index",
            "chi_of_r", "u_of_r")
    return {k: getattr(obj, k) for k in keys if hasattr(obj, k)}


class RadialIntegrals:
    """Differentiable I_L^dir, I_L^exc for one transition and a list of pairs.

    ``grid``: RadialGrid-like (r, w_simpson, w_trapz); ``bound_i``/``bound_f``: objects with the
    reference's BoundOrbital attributes (their u_of_r is replaced by the ``u_i``/``u_f`` of each
    call); ``pairs``: (cont_i, cont_f) objects with the ContinuumWave attributes (their chi_of_r is
    replaced by the rows of ``chi_i``/``chi_f``). Options as in ``radial_ME_all_L``.
    Calling the object with torch float64 CUDA tensors returns (P, 2, L_max+1).
    ``backward``: "fp64" (exact O(N L) FP64 kernels) or "tc_bf16x3" / "tc_bf16x6" (the K_L products
    of the gradients on the tensor cores with FP32 accumulation, weighted and summed over L in FP64).
    """

    def __init__(self, grid, bound_i, bound_f, pairs: Sequence, L_max: int, U_f_array: Optional[np.ndarray] = None,
                 engine: Optional[str] = None, gpu_cache: Optional[GPUCache] = None, backward: str = "fp64",
                 **options):
        self.grid, self.bound_i, self.bound_f = grid, bound_i, bound_f
        self.pairs = list(pairs)
        self.L_max = int(L_max)
        self.U_f = U_f_array
        eng = _engine_name(engine)
        # the autotuned names choose per call; the differentiable path uses one fixed forward engine
        self.engine = {"auto": "semisep", "auto_split": "tc_bf16x3"}.get(eng, eng)
        if backward != "fp64" and backward not in TC_TERMS:
            raise ValueError(f"backward must be 'fp64' or one of {sorted(TC_TERMS)}")
        self.backward = backward
        self.cache = gpu_cache or GPUCache(grid)
        self.options = dict(use_oscillatory_quadrature=options.get("use_oscillatory_quadrature", True),
                            oscillatory_method=options.get("oscillatory_method", "advanced"),
                            CC_nodes=options.get("CC_nodes", 5), phase_increment=options.get("phase_increment", 1.5708),
                            min_grid_fraction=options.get("min_grid_fraction", 0.10),
                            k_threshold=options.get("k_threshold", 0.5))

    def __call__(self, V_core: torch.Tensor, U_i: torch.Tensor, u_i: torch.Tensor, u_f: torch.Tensor,
                 chi_i: torch.Tensor, chi_f: torch.Tensor) -> torch.Tensor:
        P = len(self.pairs)
        N = self.cache.info.N
        for name, t, shape in (("V_core", V_core, (N,)), ("U_i", U_i, (N,)), ("u_i", u_i, (N,)), ("u_f", u_f, (N,)),
                               ("chi_i", chi_i, (P, N)), ("chi_f", chi_f, (P, N))):
            if tuple(t.shape) != shape or t.dtype != torch.float64 or not t.is_cuda:
                raise ValueError(f"{name}: expected a float64 CUDA tensor of shape {shape}")
        host = lambda t: t.detach().cpu().numpy()  # noqa: E731
        ci_h, cf_h = host(chi_i), host(chi_f)
        bi = SimpleNamespace(**{**_attrs(self.bound_i), "u_of_r": host(u_i)})
        bf = SimpleNamespace(**{**_attrs(self.bound_f), "u_of_r": host(u_f)})
        pairs = [(SimpleNamespace(**{**_attrs(ci), "chi_of_r": ci_h[p]}),
                  SimpleNamespace(**{**_attrs(cf), "chi_of_r": cf_h[p]})) for p, (ci, cf) in enumerate(self.pairs)]
        V_h, Ui_h = host(V_core), host(U_i)
        job = _make_job(self.grid, V_h, Ui_h, bi, bf, pairs, self.L_max, self.U_f, self.options, self.cache)
        job.tails_per_unit_moment = True
        plans = plan_job(job)
        state = _State()
        # the backward applies the transposed node-set operators, so they must be stored (not fused)
        state.prepared = PreparedJob(job, self.cache.dg, self.engine, plans=plans, fuse_folds=False)
        state.backward = self.backward
        I = _BilinearFn.apply(chi_i, chi_f, u_i, u_f, state)
        dev = chi_i.device
        nl = self.L_max + 1
        w, r = self.cache.dg.w, self.cache.dg.r
        n1 = torch.as_tensor(plans.n1[0], device=dev)
        # L=0 corrections with the Simpson weights limited to n1 (gated on the overlaps)
        corr = torch.zeros((P, 2, nl), dtype=torch.float64, device=dev)
        if np.any(V_h - Ui_h):
            wl = w[None, :] * (torch.arange(N, device=dev)[None, :] < n1[:, None])
            vd = V_core - U_i
            s2 = (wl * (u_f * u_i)[None, :]).sum(1)
            d_dir = (wl * chi_f * chi_i * vd[None, :]).sum(1)
            s2e = (wl * chi_f * u_i[None, :]).sum(1)
            d_ex = (wl * chi_i * (u_f * vd)[None, :]).sum(1)
            zero = torch.zeros_like(s2)
            corr[:, 0, 0] = torch.where(s2.detach().abs() > OVERLAP_TOL, d_dir * s2, zero)
            corr[:, 1, 0] = torch.where(s2e.detach().abs() > OVERLAP_TOL, d_ex * s2e, zero)
        # outer tails of the direct term: tau_L (per unit moment) times M_L
        tail = torch.zeros((P, 2, nl), dtype=torch.float64, device=dev)
        if plans.tails and self.L_max >= 1:
            tau = np.zeros((P, nl))
            for (_, p), t in plans.tails.items():
                tau[p] = t
            Ls = torch.arange(nl, device=dev, dtype=torch.float64)
            M = ((w * u_f * u_i)[None, :] * r[None, :] ** Ls[:, None]).sum(1)
            M = torch.where(M.detach().abs() > 1e-12, M, torch.zeros_like(M))
            M = torch.cat([torch.zeros(1, dtype=torch.float64, device=dev), M[1:]])
            tail[:, 0, :] = torch.as_tensor(tau, device=dev) * M[None, :]
        return I + corr + tail
