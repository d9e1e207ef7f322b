"""The oracle's backward of the folded form against central finite differences of the oracle's
forward (h = 1e-6), and the semiseparable split the CUDA backward uses against the dense one."""
import numpy as np

from oracle.backward import fold_adjoint, form_grads, kernel_dense
from oracle.folded import folded_eval


def _case(n=300, seed=3):
    rng = np.random.default_rng(seed)
    r = np.exp(np.linspace(np.log(1e-3), np.log(60.0), n))
    a = rng.normal(size=n) * np.exp(-r / 20)
    b = rng.normal(size=n) * np.exp(-r / 10)
    return r, a, b


def test_form_grads_match_central_differences():
    r, a, b = _case()
    L_max = 5
    g = np.random.default_rng(4).normal(size=L_max + 1)
    ga, gb = form_grads(r, a, b, g)
    h = 1e-6
    rng = np.random.default_rng(5)
    for _ in range(3):
        va, vb = rng.normal(size=len(r)), rng.normal(size=len(r))
        f = lambda s: g @ folded_eval(r, a + s * va, b + s * vb, L_max)  # noqa: E731
        fd = (f(h) - f(-h)) / (2 * h)
        an = ga @ va + gb @ vb
        assert abs(fd - an) <= 1e-7 * (abs(an) + np.abs(ga) @ np.abs(va) + np.abs(gb) @ np.abs(vb))


def test_semiseparable_backward_equals_dense():
    """(K_g y)_p = sum_L g_L [r_p^-(L+1) sum_{q<p} y_q r_q^L + r_p^L sum_{q>p} y_q r_q^-(L+1) + d_L y_p / r_p]."""
    r, a, b = _case(n=400, seed=8)
    g = np.array([0.3, -1.2, 0.7, 0.05, -0.4])
    ga, gb = form_grads(r, a, b, g)
    for y, want in ((b, ga), (a, gb)):
        u = np.zeros_like(r)
        for L, gl in enumerate(g):
            p, q = r ** L, r ** (-(L + 1))
            pre = np.cumsum(y * p) - y * p
            suf = np.cumsum((y * q)[::-1])[::-1] - y * q
            u += gl * (q * pre + p * suf + np.exp(L * np.log(1 - 1e-12)) * y / r)
        assert np.allclose(u, want, rtol=1e-12, atol=1e-12 * np.max(np.abs(want)))


def test_kernel_dense_is_symmetric():
    r, _, _ = _case(n=50)
    for L in (0, 1, 4):
        K = kernel_dense(r, L)
        assert np.array_equal(K, K.T)


def test_fold_adjoint_is_transpose():
    rng = np.random.default_rng(9)
    for H in (0, 1, 2):
        n_out, n_src = 37, 41
        op = rng.normal(size=(n_out, 2 * H + 1))
        A = np.zeros((n_out, n_src))
        for i in range(n_out):
            for d in range(-H, H + 1):
                if 0 <= i + d < n_src:
                    A[i, i + d] = op[i, d + H]
        y = rng.normal(size=n_out)
        assert np.allclose(fold_adjoint(op.ravel(), H, y, n_out, n_src), A.T @ y, rtol=0, atol=1e-14)
