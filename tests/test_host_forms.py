"""Host logic of the exact engine's form launches, checked on the CPU.

A prepared job is built on the CPU device (descriptors only, no kernel runs), its operand rows are
filled with random values, and the launch sequence of the exact FP64 engine is emulated from the
descriptors (multipole potentials, dot forms in padded runs, the remaining semiseparable forms and
their scatter into the result rows). Every result row must equal the bilinear form a^T K_L b that
the job's form descriptor names, evaluated by the oracle's semiseparable restatement. This pins the
pointer and row bookkeeping of dwba_multipole_potentials / dwba_dot_forms without a GPU.
"""
import ctypes

import numpy as np
import torch

import bench
from dwba_b200 import _lib
from oracle.folded import semiseparable_eval


def _view(ptr, n):
    return np.ctypeslib.as_array((ctypes.c_double * int(n)).from_address(int(ptr)))


def _potential_model(r, b, n_cols, L_max):
    """phi_L = K_L b (dense restatement of K_L on the grid, diagonal clamp included)."""
    bb = np.zeros(len(r))
    bb[:n_cols] = b[:n_cols]
    rl = np.minimum(r[:, None], r[None, :])
    rg = np.maximum(r[:, None], r[None, :])
    lr = np.log(np.minimum(rl / rg, 1.0 - 1e-12) + 1e-300)
    return np.stack([(1.0 / rg) * np.exp(L * lr) @ bb for L in range(L_max + 1)])


def _job(engine):
    from dwba_b200.dwba_matrix_elements import GPUCache, _make_job
    from dwba_b200.engine import DeviceGrid, PreparedJob
    from dwba_b200.plan import GridInfo
    g, z, bounds, pairs = bench.make_workload(N=301, n_cont=9, n_bound=3, seed_shift=5)
    r = g.r
    # two low-k pairs (k_i + k_f <= 0.5): the standard Simpson branch, whose direct forms keep a
    # truncated b and stay semiseparable forms
    for l1, l2 in ((0, 1), (2, 3)):
        w = [bench._Wave(l, 0.2, 0.3, np.sin(0.2 * r + 0.3) * (1 - np.exp(-(r * 0.2 / (l + 1)) ** (l + 1))))
             for l in (l1, l2)]
        pairs.append(tuple(w))

    class Cache:  # the host side of GPUCache, on the CPU device
        info = GridInfo(g.r, g.w_simpson, g.w_trapz)
        dg = DeviceGrid(info, torch.device("cpu"))
    job = _make_job(g, z, z, [b[0] for b in bounds], [b[1] for b in bounds], pairs, 5, z, {}, Cache)
    return PreparedJob(job, Cache.dg, engine), r


def _emulate(fl, L_max, r):
    nl = L_max + 1
    for p in fl.pots_host:
        phi = _potential_model(r, _view(p["b"], p["n_cols"]), int(p["n_cols"]), L_max)
        dst = _view(p["phi"], nl * int(p["stride"])).reshape(nl, int(p["stride"]))
        dst[:, :p["n_rows"]] = phi[:, :p["n_rows"]]
    runs = fl.dots_host.reshape(-1, _lib.DOT_RUN)
    for run in runs:
        assert run[0]["n_rows"] > 0 or np.all(run["n_rows"] == 0)  # a run starts with a real form
        for d in run:
            if d["n_rows"] == 0:
                assert d["out"] == 0
                continue
            assert d["phi"] == run[0]["phi"] and d["stride"] == run[0]["stride"]
            n = int(d["n_rows"])
            phi = _view(d["phi"], nl * int(d["stride"])).reshape(nl, int(d["stride"]))
            _view(d["out"], nl)[:] = phi[:, :n] @ _view(d["a"], n)
    if fl.n_ss:
        rows = fl.ss_rows_d.numpy()
        out = fl.out.numpy()
        for f, row in zip(fl.ss_forms_host, rows):
            a = np.zeros(len(r))
            b = np.zeros(len(r))
            a[:f["n_rows"]] = _view(f["a"], f["n_rows"])
            b[:f["n_cols"]] = _view(f["b"], f["n_cols"])
            out[row] = semiseparable_eval(r, a, b, L_max)


def _check(pj, out_rows_of_form, out, r):
    L_max = pj.job.L_max
    fh = pj.forms_host
    for k, f in enumerate(fh):
        a = np.zeros(len(r))
        b = np.zeros(len(r))
        a[:f["n_rows"]] = _view(f["a"], f["n_rows"])
        b[:f["n_cols"]] = _view(f["b"], f["n_cols"])
        want = semiseparable_eval(r, a, b, L_max)
        scale = semiseparable_eval(r, np.abs(a), np.abs(b), L_max)
        got = out[out_rows_of_form(k)]
        assert np.all(np.abs(got - want) <= 1e-13 * scale + 1e-300), (k, got, want)


def test_semisep_engine_form_launch():
    pj, r = _job("semisep")
    rng = np.random.default_rng(3)
    pj.ops.copy_(torch.from_numpy(rng.normal(size=tuple(pj.ops.shape))))
    pj.out.fill_(np.nan)
    dp = pj.direct_plan
    assert len(dp.dot_fo) > 0 and np.all(dp.dot_fo % 2 == 0)
    assert np.any(dp.ss_fo % 2 == 0)  # the standard-branch direct forms stay semiseparable
    assert np.count_nonzero(dp.pot_b) == pj.T
    assert len(dp.dot_fo) + len(dp.ss_fo) == pj.n_forms
    _emulate(pj.form_launch, pj.job.L_max, r)
    _check(pj, lambda k: k, pj.out.numpy(), r)


def test_tensor_core_engine_direct_launch():
    """The direct forms of the split-BF16 engines take the same exact path into out_dir."""
    pj, r = _job("tc_bf16x3")
    rng = np.random.default_rng(4)
    pj.ops.copy_(torch.from_numpy(rng.normal(size=tuple(pj.ops.shape))))
    pj.out_dir.fill_(np.nan)
    dp = pj.direct_plan
    assert np.all(dp.ss_fo % 2 == 0) and len(dp.dot_fo) + len(dp.ss_fo) == pj.T * pj.P
    _emulate(pj.form_launch, pj.job.L_max, r)
    out = pj.out_dir.numpy()
    L_max = pj.job.L_max
    for k in range(0, pj.n_forms, 2):
        f = pj.forms_host[k]
        a = np.zeros(len(r))
        b = np.zeros(len(r))
        a[:f["n_rows"]] = _view(f["a"], f["n_rows"])
        b[:f["n_cols"]] = _view(f["b"], f["n_cols"])
        want = semiseparable_eval(r, a, b, L_max)
        scale = semiseparable_eval(r, np.abs(a), np.abs(b), L_max)
        assert np.all(np.abs(out[k // 2] - want) <= 1e-13 * scale + 1e-300), k


class _EmulatedLib:
    """The two semiseparable entry points of the guard, evaluated from their descriptors on the CPU."""

    def __init__(self, r):
        self.r = r

    def _run(self, forms_ptr, n, L_max, out_ptr, absolute):
        nl = L_max + 1
        f = np.ctypeslib.as_array((ctypes.c_uint8 * (n * _lib.FORM_DTYPE.itemsize)).from_address(forms_ptr))
        f = f.view(_lib.FORM_DTYPE)
        out = _view(out_ptr, n * nl).reshape(n, nl)
        for k, d in enumerate(f):
            a = np.zeros(len(self.r))
            b = np.zeros(len(self.r))
            if d["n_rows"]:
                a[:d["n_rows"]] = _view(d["a"], d["n_rows"])
            if d["n_cols"]:
                b[:d["n_cols"]] = _view(d["b"], d["n_cols"])
            if absolute:
                a, b = np.abs(a), np.abs(b)
            out[k] = semiseparable_eval(self.r, a, b, L_max)
        return 0

    def dwba_bilinear_semisep_abs_fp64(self, forms, n, L_max, ds, r0, r1, out, st):
        return self._run(forms, n, L_max, out, True)

    def dwba_bilinear_semisep_fp64(self, forms, n, L_max, ds, r0, r1, out, st):
        return self._run(forms, n, L_max, out, False)


def test_tensor_core_guard_routes_the_dominant_forms(monkeypatch):
    """The guard recomputes exactly the exchange forms whose |I_L| exceeds theta times the largest
    |I_L| of their transition at some L, and leaves the others as the tensor cores gave them."""
    from dwba_b200 import engine
    monkeypatch.setattr(engine, "_stream", lambda: 0)  # no CUDA stream on the CPU
    pj, r = _job("tc_bf16x3")
    rng = np.random.default_rng(6)
    pj.ops.copy_(torch.from_numpy(rng.normal(size=tuple(pj.ops.shape))))
    g = pj.tc_guard
    n, nl = pj.T * pj.P, pj.nl
    # stand-in tensor-core results: the exact values with a relative error of 1e-3
    lib = _EmulatedLib(r)
    exact = torch.zeros((n, nl), dtype=torch.float64)
    lib.dwba_bilinear_semisep_fp64(g.forms_d.data_ptr(), n, pj.job.L_max, None, 0, 0, exact.data_ptr(), None)
    out = exact * (1.0 + 1e-3)
    before = out.clone()
    g.theta = 0.3
    g.launch(lib, pj.job.L_max, pj.ds, float(r[0]), float(r[-1]), out)
    t_of = torch.from_numpy(np.repeat(np.arange(pj.T), pj.P))
    gmax = torch.stack([before[t_of == t].abs().max(0).values for t in range(pj.T)])
    want = (before.abs() > 0.3 * gmax[t_of]).any(1)
    assert torch.equal(g.flag, want) and 0 < int(want.sum()) < n
    assert torch.equal(out[want], exact[want]) and torch.equal(out[~want], before[~want])
    assert torch.equal(g.forms_d, pj.forms_ex_d)  # the descriptors themselves are untouched
    # every transition keeps its largest form at each L exactly
    for t in range(pj.T):
        rows = torch.nonzero(t_of == t).ravel()
        top = rows[before[rows].abs().argmax(0)]
        assert bool(g.flag[top].all())


def test_fused_node_sets_carry_their_pairs_folds():
    """A batch whose pairs each have their own node set (different energies): with fusing, every set
    is applied to its pair's multi-folds in the node-set launch and no multi-fold is left for the fold
    launch; the fused fold descriptors are those the unfused job launches (same functions, outputs,
    bands and sizes), in the order of the fused sets, and the sets get no operator memory."""
    from dwba_b200.dwba_matrix_elements import _make_job
    from dwba_b200.engine import FUSE_MIN_SETS, DeviceGrid, PreparedJob
    from dwba_b200.plan import GridInfo
    g, z, bounds, pairs = bench.make_workload(N=1201, n_cont=FUSE_MIN_SETS + 6, n_bound=3, seed_shift=9)

    class Cache:
        info = GridInfo(g.r, g.w_simpson, g.w_trapz)
        dg = DeviceGrid(info, torch.device("cpu"))
    job = _make_job(g, z, z, [b[0] for b in bounds], [b[1] for b in bounds], pairs, 4, z, {}, Cache)
    fu = PreparedJob(job, Cache.dg, "semisep", rebuild_nodesets=True)
    un = PreparedJob(job, Cache.dg, "semisep", plans=fu.plans, rebuild_nodesets=True, fuse_folds=False)
    ns = fu.nodesets
    assert ns.n_fused == len(fu.plans.nodesets) >= FUSE_MIN_SETS and ns.n == 0
    assert len(fu.multi_host) == 0 and len(un.multi_host) == 2 * ns.n_fused
    assert un.nodesets.n_fused == 0 and un.nodesets.n == ns.n_fused

    def rel(m, job_):  # pointers as offsets into the job's function and operand matrices
        F, O = job_.F.data_ptr(), job_.ops.data_ptr()
        key = []
        for fld in ("g",):
            key.append(int(m[fld]) - F)
        key += [int(x) - F for x in m["f"][:m["n_f"]]]
        key += [int(x) - O for x in m["out"][:m["n_f"]]]
        return tuple(key) + tuple(int(m[k]) for k in ("n_f", "half_band", "n_out", "n_src", "n_clear"))
    want = {}
    for q in range(len(un.multi_host) // 2):
        mT, mB = un.multi_host[2 * q], un.multi_host[2 * q + 1]
        k = int(np.nonzero(un.nodesets.ta_all == mT["op"])[0][0])
        assert un.nodesets.bx_all[k] == mB["op"]
        want[k] = (rel(mT, un), rel(mB, un))
    got = {int(k): (rel(ns.fused_folds[2 * q], fu), rel(ns.fused_folds[2 * q + 1], fu))
           for q, k in enumerate(ns.fused_idx)}
    assert got == want
    assert np.all(ns.ta_all == 0) and np.all(ns.bx_all == 0)
    # a job with fewer single-pair sets than the threshold stores its operators
    small = _make_job(g, z, z, [b[0] for b in bounds], [b[1] for b in bounds], pairs[:8], 4, z, {}, Cache)
    assert PreparedJob(small, Cache.dg, "semisep", rebuild_nodesets=True).nodesets.n_fused == 0


def test_fused_sets_grouped_by_the_part_of_the_wave_upload_they_read():
    """With the waves uploaded in parts (WaveMatrix.chunks), the fused node sets are reordered so that
    each launch group reads only waves of its part: the groups tile the sets in ascending part order,
    every set's pair has its waves in the group's part (or the last group waits for everything), and
    the records and fold descriptors are permuted together (each set keeps its own folds)."""
    from dwba_b200.dwba_matrix_elements import _make_job
    from dwba_b200.engine import FUSE_MIN_SETS, DeviceGrid, PreparedJob
    from dwba_b200.plan import GridInfo
    g, z, bounds, pairs = bench.make_workload(N=801, n_cont=FUSE_MIN_SETS + 10, n_bound=2, seed_shift=13)

    class Cache:
        info = GridInfo(g.r, g.w_simpson, g.w_trapz)
        dg = DeviceGrid(info, torch.device("cpu"))
    job = _make_job(g, z, z, [b[0] for b in bounds], [b[1] for b in bounds], pairs, 4, z, {}, Cache)
    ref = PreparedJob(job, Cache.dg, "semisep", rebuild_nodesets=True)
    waves = job._waves
    waves.chunks = [(0, 37, None), (37, 90, None), (90, 120, None)]  # rows beyond 120: the whole upload
    got = PreparedJob(job, Cache.dg, "semisep", plans=ref.plans, rebuild_nodesets=True)
    ns, ns0 = got.nodesets, ref.nodesets
    groups = ns.fused_groups
    assert len(groups) > 1 and groups[0][1] == 0 and groups[-1][2] == ns.n_fused
    assert all(a[2] == b[1] and a[0] < b[0] for a, b in zip(groups[:-1], groups[1:]))
    wi, wf = job._wave_idx
    set_pair = {}
    for (t, p), k in np.ndenumerate(ref.plans.ns_index):
        if k >= 0:
            set_pair[int(k)] = p
    for k_part, a, b in groups:
        for j in range(a, b):
            p = set_pair[int(ns.fused_idx[j])]
            assert waves.chunk_of(np.array([max(wi[p], wf[p])]))[0] == k_part
    # records and folds follow the same permutation of the sets
    by_set0 = {int(k): (bytes(ns0.fused_recs[q].tobytes()),) for q, k in enumerate(ns0.fused_idx)}
    by_set = {int(k): (bytes(ns.fused_recs[q].tobytes()),) for q, k in enumerate(ns.fused_idx)}
    assert sorted(by_set) == sorted(by_set0)
    def rel(m, job_):  # fold pointers as offsets into the job's function and operand matrices
        F, O = job_.F.data_ptr(), job_.ops.data_ptr()
        return ((int(m["g"]) - F,) + tuple(int(x) - F for x in m["f"][:m["n_f"]]) +
                tuple(int(x) - O for x in m["out"][:m["n_f"]]) +
                tuple(int(m[f]) for f in ("n_f", "half_band", "n_out", "n_src", "n_clear")))
    for k in by_set0:  # the same record and the same folds (relative to each job's buffers)
        assert by_set[k][0] == by_set0[k][0]
        q0, q = list(ns0.fused_idx).index(k), list(ns.fused_idx).index(k)
        for h in (0, 1):
            assert rel(ns.fused_folds[2 * q + h], got) == rel(ns0.fused_folds[2 * q0 + h], ref)
    assert list(ns.fused_idx) != list(ns0.fused_idx)  # the order did change
