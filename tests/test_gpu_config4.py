"""Differentiation study at the config-4 sizes, end to end from the potential parameters.

Na-like 3s -> 3p in the parametric SAE core potential
    V(r) = -[1 + 10 e^{-a1 r} + a2 r e^{-a3 r} + a4 e^{-a5 r}] / r
(the reference's form, potential_core.py:143-200, with Zc = 1 and its a1 = 10), parameters seeded
within +-10 % of (a1..a5) = (3.0, 2.0, 1.5, 1.0, 0.8); N = 6000 on [1e-5, 200], E = 20 eV,
l_i, l_f <= 25, L <= 4 (338 pairs). The inputs of the integrals come from dwba_b200/sae.py's
solvers; dTCS/d(a_k) is the CUDA backward of the integrals (and of the torch DCS/TCS) contracted
with the central-difference tangents of the solvers (h = 1e-6 relative), and is checked against
central differences of the TCS itself; the FP32-accumulated tensor-core backward is compared with
the exact FP64 one; and a fit recovers perturbed parameters from a DCS target.
"""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu

P_REF = np.array([3.0, 2.0, 1.5, 1.0, 0.8])


def _setup(backward="fp64", l_max=25, n_theta=181):
    from dwba_b200 import sae
    from dwba_b200.autograd import RadialIntegrals
    from dwba_b200.coupling import CouplingTables
    from dwba_b200.fit import CouplingCrossSection
    g = bench.make_grid(6000, 1e-5, 200.0)
    p = np.random.default_rng(2).uniform(0.9, 1.1, 5) * P_REF
    prob = sae.SAEProblem(g, sae.Transition(E_eV=20.0, l_max=l_max, L_max=4), p,
                          full_params=lambda q: np.concatenate([[10.0], q]))
    x0 = prob.inputs(p)
    bi, bf, pairs = prob.wave_objects(x0)
    model = RadialIntegrals(g, bi, bf, pairs, 4, U_f_array=x0.U_f, engine="semisep", backward=backward)
    tab = CouplingTables(np.linspace(0.0, np.pi, n_theta), prob.pairs_l, 4, prob.k_i, prob.k_f, 0, 1)
    return prob, p, model, CouplingCrossSection(tab), x0


def test_tcs_gradient_in_the_potential_parameters():
    from dwba_b200 import sae
    from dwba_b200.autograd import RadialIntegrals
    prob, p, model, xs, x0 = _setup()
    assert len(prob.pairs_l) == 338
    v, g, fd = sae.value_and_grad(prob, model, xs.tcs, p, with_fd=True)
    assert v > 0
    assert np.all(np.abs(g - fd) <= 1e-5 * np.abs(fd) + 1e-8 * np.max(np.abs(fd))), (g, fd)
    # the same gradient with the K_L products of the backward on the tensor cores (FP32 accumulation)
    bi, bf, pairs = prob.wave_objects(x0)
    model_tc = RadialIntegrals(prob.grid, bi, bf, pairs, 4, U_f_array=x0.U_f, engine="semisep",
                               backward="tc_bf16x3", gpu_cache=model.cache)
    v2, g2 = sae.value_and_grad(prob, model_tc, xs.tcs, p)
    assert v2 == v
    assert np.all(np.abs(g2 - g) <= 1e-3 * np.max(np.abs(g))), (g2, g)


def test_fit_recovers_potential_parameters_from_a_dcs():
    """A DCS at 37 angles computed at the seeded parameters is the target; the fit starts 3 % away
    in every parameter and recovers them."""
    import torch
    from dwba_b200 import sae
    prob, p_true, model, xs, _ = _setup(l_max=12, n_theta=37)
    with torch.no_grad():
        target = xs.dcs(model(**prob.torch_inputs(prob.inputs(p_true))))

    def objective(I):
        return ((xs.dcs(I) / target - 1.0) ** 2).sum()
    p0 = p_true * np.array([1.03, 0.97, 1.03, 0.97, 1.03])
    p_fit, hist = sae.fit_parameters(prob, model, objective, p0, max_iter=80)
    assert hist[-1] < 1e-10 * hist[0], hist[-5:]
    assert np.allclose(p_fit, p_true, rtol=1e-3), (p_fit, p_true)
