"""Tensor-core (split-BF16) engine against the exact FP64 semiseparable engine on the same forms.

The split-BF16 engines trade precision for tensor throughput; the gates are |dI| <= tol * S_L
with S_L = |a|^T K_L |b| (cancellation-aware scale): tol = 3e-6 for 2 terms (hi/lo, three
products) and 1.5e-6 for 3 terms (hi/mid/lo, six products). The three-term split removes the
representation error of the operands (~1e-8 S_L at N = 500); at N ~ 10^4 both are limited by the
FP32 accumulation of ~N/16 tensor-core steps per output (~5e-7 S_L measured at N = 15000).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"tc_bf16x3": 3e-6, "tc_bf16x6": 1.5e-6}


def _job(N, n_pairs, L_max, seed):
    import bench
    from dwba_b200.dwba_matrix_elements import GPUCache, _make_job
    g, z, bounds, pairs = bench.make_workload(N=N, n_cont=n_pairs, n_bound=2, seed_shift=seed)
    cache = GPUCache.from_grid(g)
    job = _make_job(g, z, z, [b[0] for b in bounds], [b[1] for b in bounds], pairs, L_max, z, {}, cache)
    return job, cache


def _run(job, cache, engine):
    import torch
    from dwba_b200.engine import PreparedJob
    pj = PreparedJob(job, cache.dg, engine)
    pj.launch()
    d, e = pj.collect()
    torch.cuda.synchronize()
    return d, e, pj


def _scale(job, cache, pj):
    """S_L = |a|^T K_L |b| per exchange form, from the exact engine on |a|, |b|."""
    import torch
    from dwba_b200 import _lib
    from dwba_b200.engine import _ptr, _stream
    forms = pj.forms_host[1::2].copy()
    ops_abs = pj.ops.abs()
    base, base_abs = pj.ops.data_ptr(), ops_abs.data_ptr()
    forms["a"] = forms["a"] - base + base_abs
    forms["b"] = forms["b"] - base + base_abs
    n = len(forms)
    fd = torch.from_numpy(forms.view(np.uint8).copy()).cuda()
    out = torch.empty((n, job.L_max + 1), dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().dwba_bilinear_semisep_fp64(_ptr(fd), n, job.L_max, pj.ds.ctypes.data,
                                                      float(job.grid.r[0]), float(job.grid.r[-1]), _ptr(out),
                                                      _stream()), "semisep")
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(len(job.transitions), len(job.pairs), job.L_max + 1)


@pytest.mark.parametrize("engine", ["tc_bf16x3", "tc_bf16x6"])
@pytest.mark.parametrize("N,n_pairs,L_max", [(500, 8, 2), (4001, 40, 8)])
def test_tc_engine_vs_exact(engine, N, n_pairs, L_max):
    job, cache = _job(N, n_pairs, L_max, seed=7)
    d_ref, e_ref, pj_ref = _run(job, cache, "semisep")
    d, e, pj = _run(job, cache, engine)
    np.testing.assert_array_equal(d, d_ref)  # direct forms use the exact engine in both
    S = _scale(job, cache, pj_ref)
    err = np.abs(e - e_ref) / S
    assert np.isfinite(e).all()
    assert err.max() <= TOL[engine], (engine, err.max())
