"""The decomposition the ``semantics="cupy"`` mode evaluates on the GPU, checked in NumPy.

dwba_b200/cupy_mode.py evaluates the reference's CuPy quadrature (``radial_ME_all_L_gpu``,
``dwba_matrix_elements.py:1563-2549``) without its n1 x N_cc kernel matrix:
* the outer CC sums are folds a = M rho1 with the tridiagonal M_ij = sum_x W lambda_i(x) lambda_j(x)
  of the linear hats on r[:n1] (the node-set operator built with linear interpolation);
* direct: I_L = a . phi_L[:n1] with phi_L = K_L (w u_f u_i) on the full grid (int_r2);
* exchange: the kernel at a node x in (r_j, r_{j+1}] factorises per grid row, so
      inner_i = r_i^-(L+1) sum_{j<i} (alpha_j rho_j + beta_j rho_{j+1})
              + r_i^L      sum_{j>=i} (gamma_j rho_j + delta_j rho_{j+1})
  with per-interval coefficients (cupy_nodes.cu) and I_L = a . inner;
* the standard branch is w-weighted bilinear forms on r[:n1]; L=0 corrections ungated; tails added.
This model restates that decomposition step by step (the same per-interval sums the kernels form)
and must reproduce the reference's recorded CuPy-path outputs (tests/golden/cupy_semantics.npz)
and the oracle's dense restatement (oracle/cupy_path.py).
"""
import numpy as np
import pytest

import golden_cases as gc
from oracle.cupy_path import filon_params_cupy, radial_me_all_L_cupy, select_idx_limit_cupy
from oracle.radial_me import _is_excitation
from oracle.tails import analytical_multipole_tail, outer_integral_1d

CUPY = np.load(gc.GOLDEN_DIR + "/cupy_semantics.npz")
CALLS = [c for c in gc.all_calls() if not c["label"].startswith("large_grid")]


def _kernel(rows, cols, L):
    inv = 1.0 / np.maximum(rows[:, None], cols[None, :])
    return inv * (np.minimum(rows[:, None], cols[None, :]) * inv) ** L


def _hat_fold(r1, prm, f):
    """a = M f: a_i = sum_x W lambda_i(x) (f interpolated linearly at x)."""
    X, W, iL, iR, wL, wR = (prm[k] for k in ("X", "W", "iL", "iR", "wL", "wR"))
    fx = np.interp(X, r1, f)
    a = np.zeros(len(r1))
    np.add.at(a, iL, W * wL * fx)
    np.add.at(a, iR, W * wR * fx)
    return a


def _exchange_coefficients(r1, prm, L_max):
    """(alpha, beta, gamma, delta)[L, j] per grid interval j: the sums cupy_ops_kernel forms."""
    X, W, iL, iR, wL, wR = (prm[k] for k in ("X", "W", "iL", "iR", "wL", "wR"))
    n1 = len(r1)
    G = np.exp(wL * np.log(r1[iL]) + wR * np.log(r1[iR]))
    h = wL / r1[iL] + wR / r1[iR]
    t = (X - r1[iL]) / (r1[iR] - r1[iL])
    co = np.zeros((4, L_max + 1, n1))
    for L in range(L_max + 1):
        for q, v in enumerate((W * G ** L * (1 - t), W * G ** L * t, W * h * G ** -L * (1 - t), W * h * G ** -L * t)):
            np.add.at(co[q, L], iL, v)
    return co


def _exchange_inner(r1, co, rho2, L):
    """inner_i by the exclusive prefix of A and the inclusive suffix of B (cupy_forms_kernel)."""
    rho_next = np.append(rho2[1:], 0.0)
    A = co[0, L] * rho2 + co[1, L] * rho_next
    B = co[2, L] * rho2 + co[3, L] * rho_next
    pre = np.concatenate([[0.0], np.cumsum(A)[:-1]])
    suf = np.cumsum(B[::-1])[::-1]
    return r1 ** (-(L + 1)) * pre + r1 ** L * suf


def model(grid, V_core, U_i, bound_i, bound_f, cont_i, cont_f, L_max, use_oscillatory_quadrature=True,
          oscillatory_method="advanced", CC_nodes=5, phase_increment=1.5708, min_grid_fraction=0.10, k_threshold=0.5,
          U_f_array=None):
    r, w = np.asarray(grid.r, float), np.asarray(grid.w_simpson, float)
    N = len(r)
    exc = _is_excitation(bound_f)
    u_i, u_f = np.asarray(bound_i.u_of_r)[:N], np.asarray(bound_f.u_of_r)[:N]
    n1 = select_idx_limit_cupy(r, np.asarray(grid.w_trapz, float), U_i, U_f_array, u_i, u_f, cont_i.k_au,
                               cont_f.k_au, cont_i.l, cont_f.l, cont_i.idx_match, cont_f.idx_match, min_grid_fraction,
                               exc)
    r1, w1 = r[:n1], w[:n1]
    ci, cf = np.asarray(cont_i.chi_of_r)[:n1], np.asarray(cont_f.chi_of_r)[:n1]
    ui, uf = u_i[:n1], u_f[:n1]
    k_total = cont_i.k_au + cont_f.k_au
    osc = use_oscillatory_quadrature and k_total > k_threshold
    prm = filon_params_cupy(r1, k_total, phase_increment, CC_nodes) if osc else None
    d, e = np.zeros(L_max + 1), np.zeros(L_max + 1)
    if prm is not None:
        a_dir, a_ex = _hat_fold(r1, prm, cf * ci), _hat_fold(r1, prm, uf * ci)
        co = _exchange_coefficients(r1, prm, L_max)
        b_full = w * u_f * u_i
        wave = (cont_i.k_au, cont_i.l, cont_i.phase_shift, cont_i.eta, cont_i.sigma_l,
                cont_f.k_au, cont_f.l, cont_f.phase_shift, cont_f.eta, cont_f.sigma_l)
        for L in range(L_max + 1):
            d[L] = a_dir @ (_kernel(r1, r, L) @ b_full)
            e[L] = a_ex @ _exchange_inner(r1, co, cf * ui, L)
            if L >= 1 and n1 < N - 10 and exc:
                k_i, l_i, d_i, e_i, s_i, k_f, l_f, d_f, e_f, s_f = wave
                if oscillatory_method == "legacy":
                    mom = float(np.dot(w1 * uf * ui, r1 ** L))
                    if abs(mom) > 1e-12:
                        d[L] += analytical_multipole_tail(r1[-1], k_i, k_f, d_i, d_f, l_i, l_f, L, mom, e_i, e_f,
                                                          s_i, s_f)
                else:
                    mom = float(np.dot(b_full, r ** L))
                    if abs(mom) > 1e-12:
                        env = (lambda m, LL: (lambda x: m / (x ** (LL + 1)) if x > 1e-6 else 0.0))(mom, L)
                        d[L] += outer_integral_1d(env, k_i, l_i, d_i, e_i, s_i, k_f, l_f, d_f, e_f, s_f, r1[-1], r[-1],
                                                  delta_phi=np.pi / 4)
                        d[L] += analytical_multipole_tail(r[-1], k_i, k_f, d_i, d_f, l_i, l_f, L, mom, e_i, e_f,
                                                          s_i, s_f)
    else:
        for L in range(L_max + 1):
            K = _kernel(r1, r1, L)
            d[L] = (w1 * cf * ci) @ K @ (w1 * uf * ui)
            e[L] = (w1 * uf * ci) @ K @ (w1 * cf * ui)
    vd = (np.asarray(V_core) - np.asarray(U_i))[:n1]
    d[0] += np.dot(w1 * cf * ci, vd) * np.sum(w1 * uf * ui)
    e[0] += np.dot(w1 * uf * ci, vd) * np.sum(w1 * cf * ui)
    return d, e, prm is not None


@pytest.mark.parametrize("call", CALLS, ids=[c["label"] for c in CALLS])
def test_decomposition_reproduces_the_cupy_path(call):
    name, idx = call["label"].rstrip("]").split("[")
    d, e, filon = model(*call["args"], **call["kwargs"])
    od, oe = radial_me_all_L_cupy(*call["args"], **call["kwargs"])
    L = call["L_max"]
    for got, dense, key in ((d, od, f"{name}_{idx}_dir"), (e, oe, f"{name}_{idx}_exc")):
        ref = CUPY[key]
        dense = np.array([dense[l] for l in range(L + 1)])
        tol = 1e-11 * np.abs(ref) + 1e-13 * np.max(np.abs(ref))
        assert np.all(np.abs(got - ref) <= tol), (key, got, ref)
        assert np.all(np.abs(got - dense) <= tol), (key, got, dense)


def test_the_cases_cover_both_branches():
    kinds = {model(*c["args"], **c["kwargs"])[2] for c in CALLS}
    assert kinds == {True, False}


def test_semantics_is_validated_before_any_device_work():
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_gpu
    c = CALLS[0]
    with pytest.raises(ValueError, match="semantics"):
        radial_ME_all_L_gpu(*c["args"], **c["kwargs"], semantics="gpu")


@pytest.mark.parametrize("name", sorted({c["label"].split("[")[0] for c in CALLS}))
def test_host_plan_follows_the_cupy_rules(name):
    """CupyPreparedJob's host plan (built with CPU tensors, no launch): per pair the integration limit,
    the branch (phase split or standard) and the number of phase intervals of the CuPy path, the L=0
    corrections without the overlap gate and the tails of the phase-split entries."""
    from types import SimpleNamespace
    from dwba_b200 import _lib
    from dwba_b200.cupy_mode import CupyPreparedJob
    from dwba_b200.dwba_matrix_elements import _make_job
    from dwba_b200.engine import DeviceGrid
    from dwba_b200.plan import GridInfo
    calls = [c for c in CALLS if c["label"].split("[")[0] == name]
    c0 = calls[0]
    grid, V, U, bi, bf, _, _, _ = c0["args"]
    L = max(c["L_max"] for c in calls)
    kw = {k: v for k, v in c0["kwargs"].items() if k != "U_f_array"}
    calls = [c for c in calls if {k: v for k, v in c["kwargs"].items() if k != "U_f_array"} == kw]
    info = GridInfo(grid.r, grid.w_simpson, grid.w_trapz)
    cache = SimpleNamespace(info=info, dg=DeviceGrid(info, "cpu"))
    pairs = [(c["args"][5], c["args"][6]) for c in calls]
    job = _make_job(grid, V, U, bi, bf, pairs, L, c0["kwargs"]["U_f_array"], kw, cache)
    pj = CupyPreparedJob(job, cache.dg)
    r = np.asarray(grid.r)
    recs = np.frombuffer(pj.recs_d.numpy().tobytes(), dtype=_lib.NODESET_DTYPE) if pj.n_sets else None
    for p, c in enumerate(calls):
        ci, cf = c["args"][5], c["args"][6]
        n1 = select_idx_limit_cupy(r, np.asarray(grid.w_trapz), U, c0["kwargs"]["U_f_array"], bi.u_of_r, bf.u_of_r,
                                   ci.k_au, cf.k_au, ci.l, cf.l, ci.idx_match, cf.idx_match,
                                   kw.get("min_grid_fraction", 0.10), _is_excitation(bf))
        assert pj.n1[0, p] == n1, (c["label"], pj.n1[0, p], n1)
        k_total = ci.k_au + cf.k_au
        osc = kw.get("use_oscillatory_quadrature", True) and k_total > kw.get("k_threshold", 0.5)
        prm = filon_params_cupy(r[:n1], k_total, kw.get("phase_increment", 1.5708), kw.get("CC_nodes", 5)) if osc \
            else None
        assert bool(pj.A[0, p]) == (prm is not None), c["label"]
        if prm is not None:
            rec = recs[pj.set_of[0, p]]
            assert rec["n1"] == n1 and rec["log1"] == 0 and rec["log2"] == 0 and rec["breaks"] == 0
            assert rec["n_breaks"] == len(prm["W"]) // kw.get("CC_nodes", 5) + 1
        d, e, _ = model(*c["args"], **c["kwargs"])
        w1 = np.asarray(grid.w_simpson)[:n1]
        vd = (np.asarray(V) - np.asarray(U))[:n1]
        cd = np.dot(w1 * cf.chi_of_r[:n1] * ci.chi_of_r[:n1], vd) * np.sum(w1 * bf.u_of_r[:n1] * bi.u_of_r[:n1])
        assert pj.corr_dir[0, p] == pytest.approx(cd, rel=1e-12, abs=1e-300)
    assert pj.n_cforms == int(pj.A.sum())
    assert pj.form_launch.n_dots >= int(pj.A.sum())
    assert pj.form_launch.n_ss == 2 * int((~pj.A).sum())
