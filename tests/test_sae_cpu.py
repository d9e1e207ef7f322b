"""The SAE parameter model (dwba_b200/sae.py) and the torch cross sections on the CPU.

* the solvers: hydrogen bound states, free continuum waves (Riccati-Bessel normalisation), and
  smooth dependence of the outputs on the potential parameters (central differences at two steps
  agree);
* CouplingCrossSection (torch) equals CouplingTables.dcs / .tcs (the reference's coupling algebra);
* value_and_grad: the chain of a torch model's gradient with the solver tangents equals the central
  differences of the objective (a toy bilinear model stands in for the CUDA integrals here).
"""
import numpy as np
import torch

import bench
from dwba_b200 import sae
from dwba_b200.coupling import CouplingTables
from dwba_b200.fit import CouplingCrossSection

GRID = bench.make_grid(6000, 1e-5, 200.0)


def test_hydrogen_bound_states_and_free_waves():
    r = GRID.r
    V = -1.0 / r
    for l, n, E_exact in ((0, 1, -0.5), (0, 2, -0.125), (1, 1, -0.125), (1, 2, -1.0 / 18.0)):
        E, u = sae.bound_state(r, GRID.w_trapz, V, l, n)
        assert abs(E - E_exact) < 1e-4 * abs(E_exact), (l, n, E)
        assert abs(np.sum(GRID.w_trapz * u * u) - 1.0) < 1e-12
    E, u = sae.bound_state(r, GRID.w_trapz, V, 0, 1)
    assert np.max(np.abs(u - 2.0 * r * np.exp(-r))) < 1e-3
    from scipy.special import spherical_jn
    chi, d = sae.continuum_waves(r, np.zeros_like(r), [0, 3, 25], 1.2)
    for j, l in enumerate((0, 3, 25)):
        ref = 1.2 * r * spherical_jn(l, 1.2 * r)
        assert abs(d[j]) < 0.05 and np.max(np.abs(chi[j] - ref)) < 0.05  # Numerov phase error of the grid


def _problem():
    p = np.random.default_rng(2).uniform(0.9, 1.1, 5) * np.array([3.0, 2.0, 1.5, 1.0, 0.8])
    t = sae.Transition(l_max=6)
    return sae.SAEProblem(GRID, t, p, full_params=lambda q: np.concatenate([[10.0], q])), p


def test_solver_outputs_are_smooth_in_the_parameters():
    prob, p = _problem()
    for k in (0, 3):
        d = {}
        for h in (1e-6, 1e-5):
            e = np.zeros(5)
            e[k] = h * p[k]
            xp, xm = prob.inputs(p + e), prob.inputs(p - e)
            d[h] = [(getattr(xp, n) - getattr(xm, n)) / (2 * h * p[k]) for n in ("u_i", "u_f", "U_i", "chi_i", "chi_f")]
        for a, b in zip(d[1e-6], d[1e-5]):
            assert np.max(np.abs(a - b)) <= 1e-4 * np.max(np.abs(b)) + 1e-9, k


def test_torch_cross_section_equals_coupling_tables():
    rng = np.random.default_rng(8)
    chans = [(a, b) for a in range(5) for b in range(5) if (a + b) % 2 == 1]
    theta = np.linspace(0, np.pi, 37)
    tab = CouplingTables(theta, chans, 4, 1.2, 1.1, 0, 1)
    I = rng.normal(size=(len(chans), 2, 5))
    xs = CouplingCrossSection(tab, device="cpu")
    dcs = xs.dcs(torch.as_tensor(I)).numpy()
    ref = tab.dcs(I[:, 0], I[:, 1])
    assert np.allclose(dcs, ref, rtol=1e-12, atol=1e-14 * ref.max())
    assert abs(float(xs.tcs(torch.as_tensor(I))) - tab.tcs(I[:, 0], I[:, 1])) <= 1e-12 * tab.tcs(I[:, 0], I[:, 1])


class _ToyModel:
    """A bilinear stand-in for the integrals: I[p, 0, L] = sum w r^L chi_i chi_f u_i u_f, I[p, 1, L] with
    the exchange pairing and (V - U_i) -- smooth and differentiable like the real forms."""

    def __init__(self, L_max):
        self.r = torch.as_tensor(GRID.r)
        self.w = torch.as_tensor(GRID.w_simpson)
        self.L = L_max

    def __call__(self, V_core, U_i, u_i, u_f, chi_i, chi_f):
        rl = torch.stack([(self.r / 50.0) ** L for L in range(self.L + 1)])
        d = torch.einsum("n,ln,pn,pn,n,n->pl", self.w, rl, chi_i, chi_f, u_i, u_f)
        e = torch.einsum("n,ln,pn,n->pl", self.w, rl, chi_i, u_f) * torch.einsum("n,pn,n->p", self.w, chi_f, u_i)[:, None] \
            + torch.einsum("n,pn,n->p", self.w, chi_f * chi_i, (V_core - U_i))[:, None]
        return torch.stack([d, e], dim=1)


def test_chain_gradient_equals_central_differences_cpu():
    prob, p = _problem()
    tab = CouplingTables(np.linspace(0, np.pi, 19), prob.pairs_l, 4, prob.k_i, prob.k_f, 0, 1)
    xs = CouplingCrossSection(tab, device="cpu")
    model = _ToyModel(4)
    orig = prob.torch_inputs
    prob.torch_inputs = lambda x, device="cpu": orig(x, device="cpu")
    v, g, fd = sae.value_and_grad(prob, model, xs.tcs, p, with_fd=True)
    assert v > 0 and np.all(np.isfinite(g))
    assert np.all(np.abs(g - fd) <= 1e-6 * np.abs(fd) + 1e-9 * np.max(np.abs(fd))), (g, fd)
