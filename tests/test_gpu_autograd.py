"""Backward kernels and the differentiable path.

* dwba_bilinear_semisep_backward_fp64 and dwba_fold_adjoint against the oracle's dense gradients;
* ``RadialIntegrals`` forward against the reference's golden I_L;
* its gradients against central finite differences (h = 1e-6, relative perturbations) of the
  forward, along random directions, for every differentiable input;
* the fit mode recovering known parameters from a DCS.
"""
import json
import os

import numpy as np
import pytest
import torch

import golden_cases as gc
from dwba_b200 import _lib
from oracle.backward import fold_adjoint, form_grads

pytestmark = pytest.mark.gpu


def _t(x):
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device="cuda")


def _stream():
    return torch.cuda.current_stream().cuda_stream


def test_form_backward_matches_oracle():
    rng = np.random.default_rng(11)
    N, L_max = 1500, 9  # two multipole chunks of the kernel
    r = np.exp(np.linspace(np.log(1e-4), np.log(120.0), N))
    forms = [(N, N), (900, N), (N, 1100), (700, 700)]
    a = [rng.normal(size=N) * np.exp(-r / 30) for _ in forms]
    b = [rng.normal(size=N) * np.exp(-r / 15) for _ in forms]
    g = rng.normal(size=(len(forms), L_max + 1))
    rd = _t(r)
    A = [_t(x) for x in a]
    B = [_t(x) for x in b]
    GA = torch.zeros((len(forms), N), dtype=torch.float64, device="cuda")
    GB = torch.zeros_like(GA)
    desc = np.zeros(len(forms), dtype=_lib.FORM_GRAD_DTYPE)
    for f, (nr, nc) in enumerate(forms):
        desc[f] = (rd.data_ptr(), A[f].data_ptr(), B[f].data_ptr(), GA[f].data_ptr(), GB[f].data_ptr(), nr, nc)
    desc_d = torch.from_numpy(desc.view(np.uint8).copy()).cuda()
    from dwba_b200.plan import diag_scale
    ds = diag_scale(L_max)
    gd = _t(g)
    _lib.check(_lib.load().dwba_bilinear_semisep_backward_fp64(desc_d.data_ptr(), len(forms), L_max, ds.ctypes.data,
                                                               gd.data_ptr(), float(r[0]), float(r[-1]), _stream()),
               "backward")
    GA_h, GB_h = GA.cpu().numpy(), GB.cpu().numpy()
    for f, (nr, nc) in enumerate(forms):
        aa = a[f].copy()
        aa[nr:] = 0
        bb = b[f].copy()
        bb[nc:] = 0
        ga, gb = form_grads(r, aa, bb, g[f])
        assert np.allclose(GA_h[f, :nr], ga[:nr], rtol=1e-11, atol=1e-13 * np.max(np.abs(ga)))
        assert np.allclose(GB_h[f, :nc], gb[:nc], rtol=1e-11, atol=1e-13 * np.max(np.abs(gb)))
        assert np.all(GA_h[f, nr:] == 0) and np.all(GB_h[f, nc:] == 0)


def test_fold_adjoint_matches_oracle():
    rng = np.random.default_rng(12)
    N = 777
    cases = [(0, 700, N), (1, 500, 500), (2, 760, N), (2, 300, 302)]
    ops = [_t(rng.normal(size=N * (2 * H + 1))) for H, _, _ in cases]
    ys = [_t(rng.normal(size=N)) for _ in cases]
    Z = torch.full((len(cases), N), np.nan, dtype=torch.float64, device="cuda")
    adj = np.zeros(len(cases), dtype=_lib.FOLD_ADJ_DTYPE)
    for k, (H, n_out, n_src) in enumerate(cases):
        adj[k] = (ops[k].data_ptr(), ys[k].data_ptr(), Z[k].data_ptr(), H, n_out, n_src, 0)
    adj_d = torch.from_numpy(adj.view(np.uint8).copy()).cuda()
    _lib.check(_lib.load().dwba_fold_adjoint(adj_d.data_ptr(), len(cases), N, _stream()), "fold adjoint")
    Zh = Z.cpu().numpy()
    for k, (H, n_out, n_src) in enumerate(cases):
        want = fold_adjoint(ops[k].cpu().numpy(), H, ys[k].cpu().numpy(), n_out, n_src)
        assert np.allclose(Zh[k, :n_src], want, rtol=1e-14, atol=1e-14)


def _setup(call):
    from dwba_b200.autograd import RadialIntegrals
    grid, V, Ui, bi, bf, ci, cf, L_max = call["args"]
    kw = dict(call["kwargs"])
    Uf = kw.pop("U_f_array")
    model = RadialIntegrals(grid, bi, bf, [(ci, cf)], L_max, U_f_array=Uf, engine="semisep", **kw)
    N = len(grid.r)
    x = dict(V_core=_t(V[:N]), U_i=_t(Ui[:N]), u_i=_t(bi.u_of_r[:N]), u_f=_t(bf.u_of_r[:N]),
             chi_i=_t(ci.chi_of_r[None, :N]), chi_f=_t(cf.chi_of_r[None, :N]))
    return model, x


CALLS = gc.all_calls()


@pytest.mark.parametrize("call", CALLS, ids=[c["label"] for c in CALLS])
def test_forward_matches_reference(call):
    model, x = _setup(call)
    I = model(**x).cpu().numpy()[0]
    for kind, ref in ((0, call["ref_dir"]), (1, call["ref_exc"])):
        scale = np.max(np.abs(ref))
        assert np.all(np.abs(I[kind] - ref) <= 1e-11 * np.abs(ref) + 1e-13 * scale), (kind, I[kind], ref)


GRAD_CALLS = [c for c in CALLS if c["L_max"] >= 2][:8]


@pytest.mark.parametrize("call", GRAD_CALLS, ids=[c["label"] for c in GRAD_CALLS])
def test_gradients_match_central_differences(call):
    model, x = _setup(call)
    rng = np.random.default_rng(21)
    L = call["L_max"]
    c = _t(rng.normal(size=(1, 2, L + 1)))
    xs = {k: v.clone().requires_grad_(True) for k, v in x.items()}
    loss = (model(**xs) * c).sum()
    loss.backward()
    h = 1e-6
    for name in x:
        v = _t(rng.normal(size=tuple(x[name].shape))) * x[name].abs()  # relative perturbation

        def f(s):
            y = dict(x)
            y[name] = x[name] + s * v
            with torch.no_grad():
                return float((model(**y) * c).sum())
        fd = (f(h) - f(-h)) / (2 * h)
        an = float((xs[name].grad * v).sum())
        scale = float((xs[name].grad.abs() * v.abs()).sum()) + 1e-300
        assert abs(fd - an) <= 1e-6 * scale + 1e-9 * abs(float(loss)), (name, fd, an, scale)


def test_fit_to_cross_section_recovers_parameters():
    """Fit mode: two model parameters (a change of the final bound orbital's shape and a short-range
    term of V_core) recovered from a DCS at 19 angles on 16 config-1 pairs (synthetic amplitude basis)."""
    from dwba_b200.autograd import RadialIntegrals
    from dwba_b200.fit import CrossSection, fit_to_cross_section
    z = np.load(os.path.join(gc.GOLDEN_DIR, "config1.npz"))
    meta = json.loads(bytes(z["meta_json"]).decode())
    grid = gc.Grid(r=z["r"], dr=z["dr"], w_trapz=z["w_trapz"], w_simpson=z["w_simpson"])
    bi = gc.BoundOrbital(l=0, energy_au=-0.5, u_of_r=z["u_i"], n_index=1)
    bf = gc.BoundOrbital(l=1, energy_au=-0.125, u_of_r=z["u_f"], n_index=1)
    pairs = [(gc._wave(meta["waves_i"][str(li)], z["chi_i"][li]), gc._wave(meta["waves_f"][str(lf)], z["chi_f"][lf]))
             for li, lf in meta["pairs"][:16]]
    model = RadialIntegrals(grid, bi, bf, pairs, 4, U_f_array=z["U_f"], engine="semisep")
    r = _t(z["r"])
    base = dict(V_core=_t(z["V_core"]), U_i=_t(z["U_i"]), u_i=_t(z["u_i"]), u_f=_t(z["u_f"]),
                chi_i=_t(np.stack([p[0].chi_of_r for p in pairs])), chi_f=_t(np.stack([p[1].chi_of_r for p in pairs])))

    def build(beta):
        x = dict(base)
        x["u_f"] = base["u_f"] * (1.0 + beta[0] * r * torch.exp(-r / 2.0))
        x["V_core"] = base["V_core"] + beta[1] * torch.exp(-r) / r
        return x
    rng = np.random.default_rng(31)
    shape = (3, 2, 16, 5, 19)
    F = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    G = 0.3 * (rng.normal(size=shape) + 1j * rng.normal(size=shape))
    xs = CrossSection(np.linspace(0, np.pi, 19), F, G, meta["k_i"], meta["k_f"])
    beta_true = torch.tensor([0.2, 0.5], dtype=torch.float64, device="cuda")
    with torch.no_grad():
        target = xs.dcs(model(**build(beta_true)))
    beta, hist = fit_to_cross_section(model, build, lambda I: ((xs.dcs(I) / target - 1.0) ** 2).sum(), [0.0, 0.0],
                                      max_iter=100, tol=1e-24)
    assert hist[-1] < 1e-14 * hist[0], hist[-5:]
    assert torch.allclose(beta, beta_true, rtol=1e-6, atol=1e-8), beta


def test_gradients_config4_sizes():
    """Config-4 sizes (N = 6000, L = 0..4) with the synthetic batch's waves and a live
    L=0 correction (V_core != U_i): gradients of a random functional against central differences."""
    import bench
    from dwba_b200.autograd import RadialIntegrals
    g, z, bounds, pairs = bench.make_workload(N=6000, n_cont=4, n_bound=1, seed_shift=44)
    bi, bf = bounds[0]
    r = np.asarray(g.r)
    V = -1.0 / r
    U = V + 0.3 * np.exp(-r)  # V_core - U_i != 0: the L=0 correction takes part
    model = RadialIntegrals(g, bi, bf, pairs, 4, U_f_array=U, engine="semisep")
    x = dict(V_core=_t(V), U_i=_t(U), u_i=_t(bi.u_of_r), u_f=_t(bf.u_of_r),
             chi_i=_t(np.stack([p[0].chi_of_r for p in pairs])), chi_f=_t(np.stack([p[1].chi_of_r for p in pairs])))
    rng = np.random.default_rng(45)
    c = _t(rng.normal(size=(len(pairs), 2, 5)))
    xs = {k: v.clone().requires_grad_(True) for k, v in x.items()}
    loss = (model(**xs) * c).sum()
    loss.backward()
    for name in x:
        v = _t(rng.normal(size=tuple(x[name].shape))) * x[name].abs()

        def f(s):
            y = dict(x)
            y[name] = x[name] + s * v
            with torch.no_grad():
                return float((model(**y) * c).sum())
        fd = (f(1e-6) - f(-1e-6)) / 2e-6
        an = float((xs[name].grad * v).sum())
        scale = float((xs[name].grad.abs() * v.abs()).sum()) + 1e-300
        assert abs(fd - an) <= 1e-6 * scale + 1e-9 * abs(float(loss)), (name, fd, an, scale)


@pytest.mark.parametrize("nt", [2, 3])
def test_tensor_core_backward_matches_fp64_backward(nt):
    """dwba_bilinear_tc_bf16_backward against dwba_bilinear_semisep_backward_fp64 on the same forms
    (N = 3001, ragged row/column lengths, L = 0..6): the split-BF16 gradients agree with the exact
    ones to the accuracy of FP32-accumulated products (measured: about 1e-5 relative to each gradient
    vector's size for both splits; the three-term split is no better because the FP32 accumulation
    of these oscillating sums, not the bf16 split, sets the error)."""
    import torch
    from dwba_b200 import _lib
    from dwba_b200.engine import diag_scale
    lib = _lib.load()
    dev = torch.device("cuda")
    rng = np.random.default_rng(31 + nt)
    N, nf, L_max = 3001, 300, 6
    r = 1e-5 * (200.0 / 1e-5) ** np.linspace(0.0, 1.0, N)
    k = rng.uniform(0.5, 4.0, (nf, 2))
    A = np.sin(k[:, :1] * r) * r * np.exp(-rng.uniform(0.2, 1.0, (nf, 1)) * r)
    B = np.cos(k[:, 1:] * r) * r * r * np.exp(-rng.uniform(0.2, 1.0, (nf, 1)) * r)
    n_rows = rng.integers(N // 2, N + 1, nf).astype(np.int32)
    n_cols = rng.integers(N // 2, N + 1, nf).astype(np.int32)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)  # noqa: E731
    rd, Ad, Bd = t(r), t(A), t(B)
    G = t(rng.normal(size=(nf, L_max + 1)))
    out = {}
    for kind in ("fp64", "tc"):
        GA = torch.zeros((nf, N), dtype=torch.float64, device=dev)
        GB = torch.zeros((nf, N), dtype=torch.float64, device=dev)
        desc = np.zeros(nf, dtype=_lib.FORM_GRAD_DTYPE)
        row = np.uint64(8 * N)
        idx = np.arange(nf, dtype=np.uint64)
        desc["r"] = rd.data_ptr()
        desc["a"], desc["b"] = np.uint64(Ad.data_ptr()) + row * idx, np.uint64(Bd.data_ptr()) + row * idx
        desc["ga"], desc["gb"] = np.uint64(GA.data_ptr()) + row * idx, np.uint64(GB.data_ptr()) + row * idx
        desc["n_rows"], desc["n_cols"] = n_rows, n_cols
        desc_d = torch.from_numpy(desc.view(np.uint8).copy()).to(dev)
        ds = diag_scale(L_max)
        st = torch.cuda.current_stream().cuda_stream
        if kind == "fp64":
            rc = lib.dwba_bilinear_semisep_backward_fp64(desc_d.data_ptr(), nf, L_max, ds.ctypes.data, G.data_ptr(),
                                                         float(r[0]), float(r[-1]), st)
        else:
            nb = int(lib.dwba_tc_backward_workspace_bytes(nf, N, L_max, nt))
            ws = torch.empty(nb, dtype=torch.uint8, device=dev)
            status = torch.zeros(1, dtype=torch.int32, device=dev)
            rc = lib.dwba_bilinear_tc_bf16_backward(desc_d.data_ptr(), nf, rd.data_ptr(), N, L_max, nt, ds.ctypes.data,
                                                    G.data_ptr(), ws.data_ptr(), nb, status.data_ptr(), st)
            torch.cuda.synchronize()
            assert int(status.item()) == 0
        assert rc == 0
        out[kind] = (GA.cpu().numpy(), GB.cpu().numpy())
    for q in range(2):
        ref, got = out["fp64"][q], out["tc"][q]
        lens = n_rows if q == 0 else n_cols
        for f in range(nf):
            assert np.all(got[f, lens[f]:] == 0.0)
        rel = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        print(f"nt={nt} {'ga' if q == 0 else 'gb'}: max rel {rel.max():.2e}, median {np.median(rel):.2e}")
        assert rel.max() < 1e-4
