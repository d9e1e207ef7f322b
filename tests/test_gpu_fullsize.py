"""GPU parity at the full sizes of the measured workloads.

The CUDA engines (through the public batched and sweep entry points and the C ABI behind them)
against the oracle's folded FP64 operands (``oracle/folded.py``: ``fold_pair`` restates the
reference's quadrature, ``semiseparable_eval`` the bilinear forms, pinned against the dense
restatement at these sizes in ``tests/test_oracle_fullsize.py``), with the same gate as the goldens:

    |dI| <= 1e-12 |I| + c S_L,   S_L = |a|^T K_L |b| + |c_L| + |t_L|   (c = 1e-14 dense, 3e-14 semisep)

plus, on the direct integrals with outer tails, the round-off of the tails (Levin segments agree
only to round-off times the condition number of their collocation systems).

The checker interpolates onto the CC nodes with the kernel's tap arithmetic (kernel_model.py):
on log grids the kernel forms log x - log r_j from the series of log(1 + (x - r_j)/r_j), where the
reference subtracts two rounded logarithms, an error of about eps |log x| / (log r_{j+1} - log r_j)
per tap (1e-12 at N = 15000 on [1e-5, 400]) that moves direct integrals there by up to 3e-14 S_L.
tests/test_oracle_fullsize.py shows that the two tap arithmetics differ by no more than the
first-order bound of that rounding; here the engines are held to the gate above against the same
taps.

Workloads and sizes (seeded synthetic inputs with the shapes of each study):
* kernel batch: N = 15000 on [1e-5, 400], L = 0..8, the four bound pairs of the benchmark and
  16 continuum pairs spanning l = 0..63, k = 0.5..8 (the extremes included);
* ragged sweep: the lowest-energy point (45 eV, N = 2000) and the highest (1000 eV, N = 15000)
  of both transitions, Coulomb-like waves, n1 < N, outer tails on the device;
* ionization: N = 8000, L = 10, ejected Coulomb waves at 0.5 and 99 eV;
* differentiation sizes: N = 6000, L = 4, V_core != U_i (live L=0 correction).
Reference path these follow: dwba_matrix_elements.py:780-1300.
"""
import numpy as np
import pytest

import bench
from golden_cases import fullsize_batch_inputs, levin_condition
from kernel_model import engine_interp_op
from oracle.folded import fold_pair, semiseparable_eval

pytestmark = pytest.mark.gpu

REL = 1e-12
ABS = {"dense": 1e-14, "semisep": 3e-14}
TC_SCALE = 5e-6  # split-BF16 exchange forms: FP32 accumulation, checked against the scale S_L


def _oracle(grid, V, Ui, bi, bf, ci, cf, L_max, Uf):
    """(direct, exchange, S_direct, S_exchange, tail tolerance, folded operands) of one (transition, pair)."""
    fp = fold_pair(grid, V, Ui, bi, bf, ci, cf, L_max, U_f_array=Uf, interp_op=engine_interp_op)
    r = np.asarray(grid.r)

    def ev(a, b):
        return semiseparable_eval(r, a, b, L_max)
    tail = fp["tail"]
    d = ev(fp["a_dir"], fp["b_dir"]) + tail
    e = ev(fp["a_ex"], fp["b_ex"])
    d[0] += fp["corr_dir"]
    e[0] += fp["corr_ex"]
    sd = ev(np.abs(fp["a_dir"]), np.abs(fp["b_dir"])) + np.abs(tail)
    se = ev(np.abs(fp["a_ex"]), np.abs(fp["b_ex"]))
    sd[0] += abs(fp["corr_dir"])
    se[0] += abs(fp["corr_ex"])
    tt = np.zeros(L_max + 1)
    if np.any(tail):
        n1 = fp["n1"]
        r_m, r_max = r[n1 - 1], r[-1]
        w = [ci.k_au, ci.l, ci.phase_shift, ci.eta, ci.sigma_l, cf.k_au, cf.l, cf.phase_shift, cf.eta, cf.sigma_l]
        cond = levin_condition(w, r_m, r_max)
        L = np.arange(L_max + 1)
        mom = np.array([np.sum(grid.w_simpson * r ** l * bf.u_of_r * bi.u_of_r) for l in L])
        tt = 1e-13 * np.abs(tail) + (1e-14 + 1e-16 * cond) * np.abs(mom) / r_m ** (L + 1) * (r_max - r_m)
    return d, e, sd, se, tt, fp


def _check(gd, ge, ref, abs_scale, what, tc=False):
    d, e, sd, se, tt = ref[:5]
    bad_d = np.abs(gd - d) > REL * np.abs(d) + abs_scale * sd + tt
    assert not bad_d.any(), (what, "direct", gd, d, np.abs(gd - d) / sd)
    tol_e = TC_SCALE * se if tc else REL * np.abs(e) + abs_scale * se
    bad_e = np.abs(ge - e) > tol_e
    assert not bad_e.any(), (what, "exchange", ge, e, np.abs(ge - e) / se)


# ----------------------------------------------------------------------------- kernel batch
@pytest.fixture(scope="module")
def batch_case():
    g, zeros, bounds, pairs = fullsize_batch_inputs()
    refs = [[_oracle(g, zeros, zeros, bi, bf, ci, cf, 8, zeros) for ci, cf in pairs] for bi, bf in bounds]
    return g, zeros, bounds, pairs, refs


@pytest.mark.parametrize("engine", ["dense", "semisep", "tc_bf16x3"])
def test_kernel_batch_full_size(batch_case, engine):
    """N = 15000 to r = 400, L = 0..8 ((r_max/r_min)^(L+1) ~ 3e68): 4 transitions x 16 pairs in one call."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch
    g, zeros, bounds, pairs, refs = batch_case
    I_d, I_e = radial_ME_all_L_batch(g, zeros, zeros, [b[0] for b in bounds], [b[1] for b in bounds], pairs, 8,
                                     U_f_array=zeros, engine=engine, as_arrays=True)
    tc = engine.startswith("tc_")
    for t in range(len(bounds)):
        for p in range(len(pairs)):
            _check(I_d[t, p], I_e[t, p], refs[t][p], ABS.get(engine, ABS["semisep"]), (engine, t, p), tc=tc)


# ----------------------------------------------------------------------------- ragged sweep
def _pick(pairs, n):
    """The first and last pairs, the pairs with the largest l, and evenly spaced others."""
    idx = {0, len(pairs) - 1, int(np.argmax([a.l + b.l for a, b in pairs])),
           int(np.argmax([a.l - b.l for a, b in pairs])), int(np.argmax([b.l - a.l for a, b in pairs]))}
    for q in np.linspace(0, len(pairs) - 1, n).astype(int):
        if len(idx) >= n:
            break
        idx.add(int(q))
    return [pairs[i] for i in sorted(idx)]


@pytest.fixture(scope="module")
def sweep_case():
    pts = bench.make_ragged_points(64, select=(0, 63))
    for pt in pts:
        pt["pairs"] = _pick(pt["pairs"], 6)
    refs = [[_oracle(pt["grid"], pt["V_core_array"], pt["U_i_array"], pt["bound_i"], pt["bound_f"], ci, cf, 6,
                     pt["U_f_array"]) for ci, cf in pt["pairs"]] for pt in pts]
    return pts, refs


@pytest.mark.parametrize("engine", ["dense", "semisep"])
def test_ragged_sweep_extreme_points(sweep_case, engine):
    """The 45 eV (N = 2000) and 1000 eV (N = 15000) points of both transitions in one graph-replayed
    sweep, n1 < N and outer tails on the device; each point's batch call gives the same values."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch, radial_ME_all_L_sweep
    pts, refs = sweep_case
    keys = ("grid", "V_core_array", "U_i_array", "bound_i", "bound_f", "pairs", "U_f_array")
    res = radial_ME_all_L_sweep([{k: pt[k] for k in keys} for pt in pts], 6, engine=engine, graph=True, replays=1)
    assert len({len(pt["grid"].r) for pt in pts}) == 2
    for k, (pt, rr) in enumerate(zip(pts, res)):
        assert any(np.any(ref[0] != 0) for ref in refs[k])
        for p, ref in enumerate(refs[k]):
            gd = np.array([rr[p].I_L_direct[L] for L in range(7)])
            ge = np.array([rr[p].I_L_exchange[L] for L in range(7)])
            _check(gd, ge, ref, ABS[engine], (engine, k, p))
        bd, be = radial_ME_all_L_batch(pt["grid"], pt["V_core_array"], pt["U_i_array"], pt["bound_i"],
                                       pt["bound_f"], pt["pairs"], 6, U_f_array=pt["U_f_array"], engine=engine,
                                       as_arrays=True)
        for p, ref in enumerate(refs[k]):
            _check(bd[p], be[p], ref, ABS[engine], (engine, "batch", k, p))
    # the outer tails took part at both grid sizes
    assert all(any(np.any(ref[5]["tail"] != 0) for ref in refs[k]) for k in range(len(pts)))


# ----------------------------------------------------------------------------- ionization
@pytest.fixture(scope="module")
def ionization_case():
    pts = bench.make_ionization_points(select=(0, 39))
    out = []
    for pt in pts:
        sel_t = sorted({0, len(pt["l_ej"]) // 2, len(pt["l_ej"]) - 1})
        bi = [pt["bound_i"][t] for t in sel_t]
        bf = [pt["bound_f"][t] for t in sel_t]
        pairs = _pick(pt["pairs"], 6)
        refs = [[_oracle(pt["grid"], pt["V_core_array"], pt["U_i_array"], b_i, b_f, ci, cf, 10, pt["U_f_array"])
                 for ci, cf in pairs] for b_i, b_f in zip(bi, bf)]
        out.append((pt, bi, bf, pairs, refs))
    return out


@pytest.mark.parametrize("engine", ["dense", "semisep"])
def test_ionization_full_size(ionization_case, engine):
    """N = 8000 on [1e-5, 200], L = 0..10 ((r_max/r_min)^(L+1) ~ 2e80), ejected Coulomb waves at the
    lowest (0.5 eV, eta = -5.2) and highest (99 eV) ejected energies as the final states."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch
    for pt, bi, bf, pairs, refs in ionization_case:
        I_d, I_e = radial_ME_all_L_batch(pt["grid"], pt["V_core_array"], pt["U_i_array"], bi, bf, pairs, 10,
                                         U_f_array=pt["U_f_array"], engine=engine, as_arrays=True)
        for t in range(len(bi)):
            for p in range(len(pairs)):
                _check(I_d[t, p], I_e[t, p], refs[t][p], ABS[engine], (engine, pt["E_ej"], t, p))


# ----------------------------------------------------------------------------- differentiation sizes
@pytest.mark.parametrize("engine", ["dense", "semisep"])
def test_differentiation_sizes(engine):
    """N = 6000, L = 0..4, V_core != U_i: the L=0 corrections are live in both integrals."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch
    g, V, U, bi, bf, pairs, _ = bench.make_gradient_inputs()
    pairs = _pick(pairs, 8)
    I_d, I_e = radial_ME_all_L_batch(g, V, U, bi, bf, pairs, 4, U_f_array=U, engine=engine, as_arrays=True)
    live = 0
    for p, (ci, cf) in enumerate(pairs):
        ref = _oracle(g, V, U, bi, bf, ci, cf, 4, U)
        live += int(ref[5]["corr_dir"] != 0.0 and ref[5]["corr_ex"] != 0.0)
        _check(I_d[p], I_e[p], ref, ABS[engine], (engine, p))
    assert live == len(pairs)
