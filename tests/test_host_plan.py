"""Host planning (product code) plus a NumPy model of the kernels' index arithmetic, against the goldens.

Runs without a GPU: it checks the integration limit, branch and node-set choice, the
C++ outer tails and L=0 corrections, and the banded fold design of nodes.cu/fold.cu.
"""
import numpy as np
import pytest

import golden_cases as gc
import kernel_model as km
from oracle.folded import folded_eval
from dwba_b200 import _lib
from dwba_b200 import dwba_matrix_elements as dme
from dwba_b200.engine import plan_job
from dwba_b200.plan import GridInfo, cc_reference

UNIT = np.load(gc.GOLDEN_DIR + "/unit_quadrature.npz")


class _Cache:
    def __init__(self, grid):
        self.info = GridInfo(grid.r, grid.w_simpson, grid.w_trapz)


def _model_eval(call):
    grid, V, Ui, bi, bf, ci, cf, L_max = call["args"]
    kw = dict(call["kwargs"])
    Uf = kw.pop("U_f_array")
    job = dme._make_job(grid, V, Ui, bi, bf, [(ci, cf)], L_max, Uf, kw, _Cache(grid))
    job.tails_on_device = False  # every tail through the native host path here
    pp = plan_job(job).pair(0, 0)
    g, N, r = job.grid, job.grid.N, job.grid.r
    (wi, wf), = job.pairs
    tr = job.transitions[0]
    n1 = pp.n1
    if pp.osc and pp.nodeset is not None:
        ns = pp.nodeset
        ta, bx = km.bands(r, n1, ns.n_breaks, ns.breaks, job.CC_nodes, ns.log1, ns.log2)
        a_dir = km.fold(ta, 1, wf.chi_of_r, wi.chi_of_r, n1, n1, N)
        a_ex = km.fold(ta, 1, tr.u_f, wi.chi_of_r, n1, n1, N)
        b_ex = km.fold(bx, 2, wf.chi_of_r, tr.u_i, min(N, n1 + 2), N, N)
        b_dir = g.w * tr.u_f * tr.u_i
    else:
        wl = g.w.copy()
        wl[n1:] = 0
        a_dir, a_ex = wl * wf.chi_of_r * wi.chi_of_r, wl * tr.u_f * wi.chi_of_r
        b_ex, b_dir = wl * wf.chi_of_r * tr.u_i, wl * tr.u_f * tr.u_i
    Id, Ie = folded_eval(r, a_dir, b_dir, L_max), folded_eval(r, a_ex, b_ex, L_max)
    Sd = folded_eval(r, np.abs(a_dir), np.abs(b_dir), L_max)
    Se = folded_eval(r, np.abs(a_ex), np.abs(b_ex), L_max)
    if pp.tail is not None:
        Id += pp.tail
        Sd += np.abs(pp.tail)
    Id[0] += pp.corr_dir
    Ie[0] += pp.corr_ex
    Sd[0] += abs(pp.corr_dir)
    Se[0] += abs(pp.corr_ex)
    return Id, Ie, Sd, Se, pp


@pytest.mark.parametrize("call", gc.all_calls(), ids=[c["label"] for c in gc.all_calls()])
def test_plan_and_kernel_model(call):
    Id, Ie, Sd, Se, _ = _model_eval(call)
    assert np.all(np.abs(Id - call["ref_dir"]) <= 1e-12 * np.abs(call["ref_dir"]) + 1e-14 * Sd)
    assert np.all(np.abs(Ie - call["ref_exc"]) <= 1e-12 * np.abs(call["ref_exc"]) + 1e-14 * Se)


def test_coulomb_breaks_bit_exact():
    r = np.load(gc.GOLDEN_DIR + "/case_h_1s2p_50eV.npz")["r"]
    for i in range(5):
        n, k, dphi, eta, d = UNIT[f"phase_params_{i}"]
        if abs(eta) < 1e-10:
            continue
        rr = r[: int(n)]
        br = _lib.phase_breaks_coulomb(rr[0], rr[-1], k, d, eta)
        np.testing.assert_array_equal(br, UNIT[f"phase_nodes_{i}"])


def test_tail_device_routing():
    """Pairs reach the device tail kernel unless a phase branch has ~zero mid-interval frequency."""
    w = np.array([1.2, 2, 0.3, 0.0, 0.0, 0.9, 3, 0.1, 0.0, 0.0])
    assert _lib.tail_on_device(w, 50.0, 200.0)
    same = np.array([1.0, 0, 0.3, 0.0, 0.0, 1.0, 0, 0.1, 0.0, 0.0])  # k_i = k_f, l = 0: Phi' of the minus branch = 0
    assert not _lib.tail_on_device(same, 50.0, 200.0)


def test_outer_tails_native():
    for row in UNIT["tails"]:
        rm, rmax, ki, kf, li, lf, di, df, ei, ef, si, sf, L, mom, t_out, t_inf, t_rm, _ = row
        L = int(L)
        moments = np.zeros(L + 1)
        moments[L] = mom
        wave = [ki, li, di, ei, si, kf, lf, df, ef, sf]
        adv = _lib.outer_tails(wave, rm, rmax, L, moments, 0, 4096, np.pi / 2)[L]
        leg = _lib.outer_tails(wave, rm, rmax, L, moments, 1, 4096, np.pi / 2)[L]
        assert abs(adv - (t_out + t_inf)) <= 1e-12 * abs(t_out + t_inf) + 1e-16
        assert abs(leg - t_rm) <= 1e-14 * abs(t_rm) + 1e-18


def test_cc_tables_match_reference():
    for n in (2, 3, 5, 7, 9):
        x, w = cc_reference(n)
        np.testing.assert_array_equal(x, UNIT[f"cc_x_{n}"])
        np.testing.assert_array_equal(w, UNIT[f"cc_w_{n}"])


def test_vectorised_planner_matches_scalar_idx_limit():
    """The vectorised planner against the scalar restatement of dwba_matrix_elements.py:909-1022."""
    from dwba_b200.plan import idx_limit
    for name in gc.case_names():
        common, calls = gc.load_case(name)
        grid = common["grid"]
        pairs = [(a, b) for a in common["waves_i"].values() for b in common["waves_f"].values()]
        job = dme._make_job(grid, common["V_core"], common["U_i"], common["bound_i"], common["bound_f"], pairs, 4,
                            common["U_f"], {}, _Cache(grid))
        jp = plan_job(job)
        tr = job.transitions[0]
        for p_i, (ci, cf) in enumerate(job.pairs):
            pp = jp.pair(0, p_i)
            n1 = idx_limit(job.grid, job.U_i, job.U_f, tr.u_i, tr.u_f, ci.k_au, cf.k_au, ci.l, cf.l, ci.idx_match,
                           cf.idx_match)
            assert pp.n1 == n1, (name, ci.l, cf.l)


def test_invalid_arguments_raise_value_error():
    with pytest.raises(ValueError):
        _lib.check(_lib.DWBA_ERR_INVALID_ARG, "x")
    with pytest.raises(_lib.DWBAError):
        _lib.check(_lib.DWBA_ERR_CUDA, "x")


def test_node_set_plans_equal_single_key_planning():
    """plan_job's node sets (linspace counts for all keys at once, Coulomb sets one by one) equal
    plan_nodeset for each key, on the golden calls and on synthetic batch waves."""
    import bench
    from dwba_b200.plan import plan_nodeset
    jobs = []
    for call in gc.all_calls():
        grid, V, Ui, bi, bf, ci, cf, L_max = call["args"]
        kw = dict(call["kwargs"])
        Uf = kw.pop("U_f_array")
        jobs.append(dme._make_job(grid, V, Ui, bi, bf, [(ci, cf)], L_max, Uf, kw, _Cache(grid)))
    g, z, bounds, pairs = bench.make_workload(N=4001, n_cont=64, n_bound=2)
    jobs.append(dme._make_job(g, z, z, [b[0] for b in bounds], [b[1] for b in bounds], pairs, 4, z, {}, _Cache(g)))
    n = 0
    for job in jobs:
        for ns in plan_job(job).nodesets:
            ref = plan_nodeset(job.grid, ns.key)
            assert ref is not None and ref.n_breaks == ns.n_breaks
            assert (ref.log1, ref.log2) == (ns.log1, ns.log2)
            assert (ref.breaks is None) == (ns.breaks is None)
            if ref.breaks is not None:
                assert np.array_equal(ref.breaks, ns.breaks)
            n += 1
    assert n >= 64
