"""The oracle's O(N L) semiseparable evaluation against its dense restatement of the reference's
kernel (K_L = (1/r_>) exp(L log(min(r_</r_>, 1-1e-12) + 1e-300)), dwba_matrix_elements.py:1057-1116)
at the full sizes of the measured workloads, where (r_max/r_min)^(L+1) reaches 1e68 to 1e80. The
GPU parity tests at those sizes (tests/test_gpu_fullsize.py) use the semiseparable evaluation as
their checker; this pins it to the dense form there."""
import numpy as np

import bench
from oracle.folded import fold_pair, folded_eval, semiseparable_eval


def _pair(r, l1, k1, l2, k2, seed):
    rng = np.random.default_rng(seed)
    out = []
    for l, k in ((l1, k1), (l2, k2)):
        d = float(rng.uniform(0.0, np.pi))
        out.append(bench._Wave(l, k, d, np.sin(k * r - 0.5 * l * np.pi + d) *
                               (1.0 - np.exp(-(r / ((l + 1) / k)) ** (l + 1)))))
    return out


def _agree(r, a, b, L_max, tol):
    s = semiseparable_eval(r, a, b, L_max)
    d = folded_eval(r, a, b, L_max)
    scale = semiseparable_eval(r, np.abs(a), np.abs(b), L_max)
    assert np.all(np.abs(s - d) <= 1e-13 * np.abs(d) + tol * scale), (s, d, np.abs(s - d) / scale)


def test_kernel_batch_size_exchange_form():
    """N = 15000 on [1e-5, 400], L = 0..8, l = 63 against l = 0 (exchange form of the widest node set)."""
    g, zeros, bounds, _ = bench.make_workload(15000, n_cont=1)
    ci, cf = _pair(g.r, 0, 8.0, 63, 7.5, 3)
    fp = fold_pair(g, zeros, zeros, bounds[0][0], bounds[0][1], ci, cf, 8, U_f_array=zeros)
    assert fp["n1"] == 15000
    _agree(g.r, fp["a_ex"], fp["b_ex"], 8, 1e-15)


def test_ionization_size_direct_form():
    """N = 8000 on [1e-5, 200], L = 0..10, an ejected Coulomb wave as the final state (direct form,
    full-grid inner integral)."""
    pts = bench.make_ionization_points(select=(0,))
    pt = pts[0]
    ci, cf = pt["pairs"][-1]
    fp = fold_pair(pt["grid"], pt["V_core_array"], pt["U_i_array"], pt["bound_i"][-1], pt["bound_f"][-1], ci, cf, 10,
                   U_f_array=pt["U_f_array"])
    _agree(pt["grid"].r, fp["a_dir"], fp["b_dir"], 10, 1e-15)
