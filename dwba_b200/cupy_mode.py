"""The quadrature of the reference's CuPy path, as an engine mode (``semantics="cupy"``).

The reference has two implementations of the radial integrals whose results differ (by a few
percent on excitation and up to an order of magnitude on ionization): the CPU path
``radial_ME_all_L`` (``dwba_matrix_elements.py:780-1300``), which the default mode reproduces, and
the CuPy path ``radial_ME_all_L_gpu`` (``:1563-2549``), which this mode reproduces:
* integration limit: the final state's 99 % extent counts only for a bound final state (``:688-777``);
* phase intervals: a linspace on [r_0, r_{n1-1}] with the raw step phase_increment / k_total (no
  adaptive clamp, no Coulomb phase), at least two of them, else the standard Simpson form (``:1350-1414``);
* Clenshaw-Curtis weights from the table rule for every node count (``:1316-1347``);
* interpolation linear in r on r[:n1] (``cp.interp``); direct: the outer CC sum of rho1 against the
  full-grid inner integral int_r2 (``:2330-2420``, ``_gpu_filon_direct`` :1416-1465);
* exchange: the inner CC sum on r[:n1] with the kernel at each node formed from the interpolated
  1/r_> and log-ratio (``_gpu_filon_exchange`` :1469-1560, ``:2072-2091``), on the GPU by
  ``dwba_cupy_exchange_ops`` / ``dwba_cupy_exchange_forms``;
* L=0 corrections without the overlap gate; the legacy tail from the moments of r[:n1].
Every integral is evaluated on the GPU (node-set operators, folds, multipole potentials, dot and
semiseparable forms, the CuPy exchange forms), exactly in FP64 whatever engine the caller names;
outer tails and L=0 corrections are added on the host in FP64; node sets are built per call.
"""
from __future__ import annotations

from typing import Dict, Tuple

import numpy as np
import torch

from . import _lib
from .engine import DirectPlan, FormLaunch, Job, WaveMatrix, _dev, _idx_limits, _pair_arrays, _ptr, _stream
from .plan import diag_scale, multipole_moments, tail_limits


def cc_table_rule(n: int) -> Tuple[np.ndarray, np.ndarray]:
    """The CuPy path's Clenshaw-Curtis reference table for n nodes (``dwba_matrix_elements.py:1316-1347``):
    nodes cos(pi j/(n-1)) from +1 down to -1, weights (2/(n-1)) (1 - 2 sum_j cos(2 j theta)/(4 j^2 - 1)),
    the last term halved for odd n."""
    theta = np.pi * np.arange(n) / (n - 1)
    x = np.cos(theta)
    jm = (n - 1) // 2
    sums = np.zeros(n)
    if jm > 0:
        jv = np.arange(1, jm + 1)
        sums = np.sum(np.cos(2 * jv[:, None] * theta[None, :]) / (4 * jv ** 2 - 1)[:, None], axis=0)
        if (n - 1) % 2 == 0:
            sums = sums + 0.5 * np.cos(2 * jm * theta) / (4 * jm ** 2 - 1)
    return x, (2.0 / (n - 1)) * (1 - 2 * sums)


class CupyPreparedJob:
    """A job evaluated with the CuPy path's quadrature; results indexed [transition, pair, L]."""

    def __init__(self, job: Job, dg):
        self.job, self.dg = job, dg
        self.lib = _lib.load()
        dev = dg.device
        g = job.grid
        N, r = g.N, g.r
        self.nl = nl = job.L_max + 1
        T, P = len(job.transitions), len(job.pairs)
        self.T, self.P = T, P
        pa = _pair_arrays(job.pairs)
        k_total = pa["k_i"] + pa["k_f"]
        osc = bool(job.use_oscillatory_quadrature) & (k_total > job.k_threshold)
        waves = WaveMatrix(N)
        wi = np.array([waves.add(ci.chi_of_r) for ci, _ in job.pairs], dtype=np.int64)
        wf = np.array([waves.add(cf.chi_of_r) for _, cf in job.pairs], dtype=np.int64)
        tidx = [(waves.add(t.u_i), waves.add(t.u_f)) for t in job.transitions]
        self.F = F = waves.upload(dev)
        Fp, row = np.uint64(_ptr(F)), np.uint64(8 * N)

        def fp(i):
            return Fp + row * np.uint64(i)
        n1 = np.stack([_idx_limits(job, pa, t, cupy=True) for t in job.transitions])  # (T, P)
        self.n1 = n1
        span = r[n1 - 1] - r[0]
        with np.errstate(divide="ignore", invalid="ignore"):
            n_int = np.maximum(1, np.ceil(span / (job.phase_increment / k_total[None, :])))
            n_int = np.where(np.isfinite(n_int), n_int, 1).astype(np.int64)
            step = span / n_int
        A = osc[None, :] & (k_total[None, :] >= 1e-6) & (n_int >= 2) & (step > 1e-12)
        self.A = A
        # node sets: one per distinct (n1, k_total) of the phase-split entries
        keys: Dict[Tuple[int, float], Tuple[int, int]] = {}
        set_of = np.full((T, P), -1, dtype=np.int64)
        for t, p in zip(*np.nonzero(A)):
            kk = (int(n1[t, p]), float(k_total[p]))
            if kk not in keys:
                keys[kk] = (len(keys), int(n_int[t, p]))
            set_of[t, p] = keys[kk][0]
        self.set_of = set_of
        S = len(keys)
        n1s = np.array([k[0] for k in keys], dtype=np.int64)
        nbr = np.array([v[1] + 1 for v in keys.values()], dtype=np.int64)
        sz = 3 * n1s + 5 * N + 4 * nl * n1s
        offs = np.concatenate([[0], np.cumsum(sz)[:-1]]).astype(np.uint64)
        self.set_block = torch.empty(max(1, int(sz.sum())), dtype=torch.float64, device=dev)
        base = np.uint64(_ptr(self.set_block))
        ta = base + np.uint64(8) * offs
        bx = ta + np.uint64(8) * (3 * n1s).astype(np.uint64)
        opsp = bx + np.uint64(8 * 5 * N)
        self.n_sets = S
        self.max_n1 = int(n1s.max()) if S else 0
        if S:
            recs = np.zeros(S, dtype=_lib.NODESET_DTYPE)
            recs["r"], recs["logr"], recs["ta"], recs["bx"] = _ptr(dg.r), _ptr(dg.logr), ta, bx
            recs["n_grid"], recs["n1"], recs["n_breaks"] = N, n1s, nbr
            crec = np.zeros(S, dtype=_lib.CUPY_SET_DTYPE)
            crec["r"], crec["logr"], crec["ops"] = _ptr(dg.r), _ptr(dg.logr), opsp
            crec["n1"], crec["n_breaks"], crec["L_max"] = n1s, nbr, job.L_max
            self.recs_d, self.crec_d = _dev(recs.view(np.uint8), dev), _dev(crec.view(np.uint8), dev)
            x, wt = cc_table_rule(job.CC_nodes)
            self.ccx, self.ccw = _dev(np.asarray(x, dtype=np.float64), dev), _dev(np.asarray(wt, dtype=np.float64), dev)
            self.ns_status = torch.zeros(1, dtype=torch.int32, device=dev)
        # operand rows: per (t, p) a_dir, a_ex, b_dir, b_ex (the last two for the standard branch), and
        # one full-grid b = w u_f u_i per transition
        SL = 4
        self.ops = torch.empty((SL * T * P + T, N), dtype=torch.float64, device=dev)
        Op = np.uint64(_ptr(self.ops))
        folds, cforms = [], []
        forms = np.zeros(2 * T * P, dtype=_lib.FORM_DTYPE)
        self.out = torch.empty((2 * T * P, nl), dtype=torch.float64, device=dev)
        outp = np.uint64(_ptr(self.out))
        b_full = Op + row * (np.uint64(SL * T * P) + np.arange(T, dtype=np.uint64))
        r_p = _ptr(dg.r)
        for t, (iu_i, iu_f) in enumerate(tidx):
            folds.append((_ptr(dg.w), fp(iu_f), fp(iu_i), b_full[t], 0, N))
            for p in range(P):
                fo = 2 * (t * P + p)
                slot = Op + row * np.uint64(SL * (t * P + p))
                a_dir, a_ex, b_dir, b_ex = (slot + row * np.uint64(q) for q in range(SL))
                v = int(n1[t, p])
                if A[t, p]:
                    k = set_of[t, p]
                    folds.append((ta[k], fp(wf[p]), fp(wi[p]), a_dir, 1, v))
                    folds.append((ta[k], fp(iu_f), fp(wi[p]), a_ex, 1, v))
                    forms[fo] = (r_p, a_dir, b_full[t], v, N)
                    cforms.append((r_p, a_ex, fp(wf[p]), fp(iu_i), opsp[k], outp + np.uint64(8 * nl * (fo + 1)), v,
                                   job.L_max))
                else:
                    wv = _ptr(dg.w)
                    folds.append((wv, fp(wf[p]), fp(wi[p]), a_dir, 0, v))
                    folds.append((wv, fp(iu_f), fp(iu_i), b_dir, 0, v))
                    folds.append((wv, fp(iu_f), fp(wi[p]), a_ex, 0, v))
                    folds.append((wv, fp(wf[p]), fp(iu_i), b_ex, 0, v))
                    forms[fo] = (r_p, a_dir, b_dir, v, v)
                    forms[fo + 1] = (r_p, a_ex, b_ex, v, v)
        fh = np.zeros(len(folds), dtype=_lib.FOLD_DTYPE)
        for i, (op, f_, g_, o, h, n) in enumerate(folds):
            fh[i] = (int(op), int(f_), int(g_), int(o), h, n, n, n)
        self.n_folds = len(fh)
        self.folds_d = _dev(fh.view(np.uint8), dev)
        d_rows = np.arange(0, 2 * T * P, 2, dtype=np.int64).reshape(T, P)
        dot_fo = d_rows[A]
        dot_t = np.repeat(np.arange(T), P).reshape(T, P)[A]
        ss_fo = np.sort(np.concatenate([d_rows[~A], d_rows[~A] + 1]))
        pot_b = np.where(A.any(axis=1), b_full, np.uint64(0))
        dp = DirectPlan(pot_b=pot_b, dot_fo=dot_fo, dot_t=dot_t, ss_fo=ss_fo)
        self.form_launch = FormLaunch([(forms, dp, N, r_p, dot_fo, ss_fo)], self.out, nl, dev)
        cf = np.zeros(len(cforms), dtype=_lib.CUPY_FORM_DTYPE)
        for i, c in enumerate(cforms):
            cf[i] = tuple(int(x) for x in c)
        self.n_cforms = len(cf)
        self.cforms_d = _dev(cf.view(np.uint8), dev) if len(cf) else None
        self.ds = diag_scale(job.L_max)
        self._host_terms(pa, n1, A)

    def _host_terms(self, pa, n1, A):
        """L=0 corrections (no overlap gate, Simpson weights on r[:n1]) and the outer tails of the
        phase-split entries (``dwba_matrix_elements.py:2430-2520``)."""
        job, g = self.job, self.job.grid
        N, r, w = g.N, g.r, g.w
        T, P, nl = self.T, self.P, self.nl
        chi_i = [np.asarray(job.pairs[p][0].chi_of_r)[:N] for p in range(P)]
        chi_f = [np.asarray(job.pairs[p][1].chi_of_r)[:N] for p in range(P)]
        V_diff = job.V_core - job.U_i
        self.corr_dir = np.zeros((T, P))
        self.corr_ex = np.zeros((T, P))
        self.tails = np.zeros((T, P, nl))
        max_seg, max_dphi = tail_limits()
        legacy = job.oscillatory_method == "legacy"
        for t, tr in enumerate(job.transitions):
            mom_full = multipole_moments(g, tr.u_i, tr.u_f, job.L_max)
            for p in range(P):
                v = int(n1[t, p])
                wl = w[:v]
                ci, cf = chi_i[p][:v], chi_f[p][:v]
                self.corr_dir[t, p] = np.dot(wl * cf * ci, V_diff[:v]) * np.sum(wl * tr.u_f[:v] * tr.u_i[:v])
                self.corr_ex[t, p] = np.dot(wl * tr.u_f[:v] * ci, V_diff[:v]) * np.sum(wl * cf * tr.u_i[:v])
                if not (A[t, p] and job.L_max >= 1 and v < N - 10 and tr.excitation):
                    continue
                wave = np.array([pa["k_i"][p], pa["l_i"][p], pa["d_i"][p], pa["e_i"][p], pa["s_i"][p],
                                 pa["k_f"][p], pa["l_f"][p], pa["d_f"][p], pa["e_f"][p], pa["s_f"][p]])
                if legacy:  # analytical tail from r_m with the moments of r[:n1]
                    m = np.zeros(nl)
                    rp = np.ones(v)
                    base = wl * tr.u_f[:v] * tr.u_i[:v]
                    for L in range(1, nl):
                        rp = rp * r[:v]
                        m[L] = np.dot(base, rp)
                    self.tails[t, p] = _lib.outer_tails(wave, float(r[v - 1]), float(r[-1]), job.L_max, m, 1, max_seg,
                                                        max_dphi)
                else:
                    self.tails[t, p] = _lib.outer_tails(wave, float(r[v - 1]), float(r[-1]), job.L_max, mom_full, 0,
                                                        max_seg, max_dphi)

    def launch(self) -> None:
        lib, job, g = self.lib, self.job, self.job.grid
        st = _stream()
        if self.n_sets:
            _lib.check(lib.dwba_build_nodesets(_ptr(self.recs_d), self.n_sets, g.N, _ptr(self.ccx), _ptr(self.ccw),
                                               job.CC_nodes, _ptr(self.ns_status), st), "dwba_build_nodesets")
            _lib.check(lib.dwba_cupy_exchange_ops(_ptr(self.crec_d), self.n_sets, self.max_n1, job.L_max, _ptr(self.ccx),
                                                  _ptr(self.ccw), job.CC_nodes, st), "dwba_cupy_exchange_ops")
        for s0 in range(0, self.n_folds, 65535):
            n = min(65535, self.n_folds - s0)
            _lib.check(lib.dwba_fold(_ptr(self.folds_d) + s0 * _lib.FOLD_DTYPE.itemsize, n, g.N, st), "dwba_fold")
        self.form_launch.launch(lib, job.L_max, self.ds, float(g.r[0]), float(g.r[-1]))
        if self.n_cforms:
            _lib.check(lib.dwba_cupy_exchange_forms(_ptr(self.cforms_d), self.n_cforms, job.L_max, float(g.r[0]),
                                                    float(g.r[-1]), st), "dwba_cupy_exchange_forms")

    def collect(self):
        """(I_dir, I_exc) as (T, P, L_max+1) float64 arrays."""
        res = self.out.cpu().numpy()
        if self.n_sets and int(self.ns_status.item()) != 0:
            raise _lib.DWBAError(_lib.DWBA_ERR_RANGE, "dwba_build_nodesets")
        T, P, nl = self.T, self.P, self.nl
        I_dir = res[0::2].reshape(T, P, nl).copy() + self.tails
        I_exc = res[1::2].reshape(T, P, nl).copy()
        I_dir[:, :, 0] += self.corr_dir
        I_exc[:, :, 0] += self.corr_ex
        return I_dir, I_exc
