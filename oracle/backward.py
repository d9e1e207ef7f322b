"""Gradients of the folded form -- oracle only (test infrastructure; never on the product path).

The reference computes no gradients; this module states the backward of the folded evaluation
in ``oracle/folded.py`` (I_L = a^T K_L b + c_L + t_L) in plain NumPy, as the checker for the
CUDA backward kernels:

* bilinear part: dLoss/da = K_g b, dLoss/db = K_g a with K_g = sum_L g_L K_L (K_L symmetric),
  K_L generated densely with the reference formula (dwba_matrix_elements.py:1057-1080);
* banded folds a = Op (f * g): dLoss/d(f * g) = Op^T y (row i of Op holds columns i-H..i+H).
"""
from __future__ import annotations

import numpy as np


def kernel_dense(r, L):
    """K_L[i, j] = (1/r_>) exp(L log(min(r_</r_>, 1-1e-12) + 1e-300)) (reference formula)."""
    r = np.asarray(r, dtype=float)
    rl = np.minimum(r[:, None], r[None, :])
    rg = np.maximum(r[:, None], r[None, :])
    inv = 1.0 / rg
    if L == 0:
        return inv
    return inv * np.exp(L * np.log(np.minimum(rl / rg, 1.0 - 1e-12) + 1e-300))


def form_grads(r, a, b, g):
    """(K_g b, K_g a) for upstream gradients g[L], L = 0..len(g)-1."""
    Kg = sum(float(gl) * kernel_dense(r, L) for L, gl in enumerate(g))
    return Kg @ b, Kg @ a


def fold_adjoint(op, half_band, y, n_out, n_src):
    """z = Op^T y for a banded fold operator stored row-major with 2H+1 taps per row."""
    W = 2 * half_band + 1
    op = np.asarray(op, dtype=float).reshape(-1, W)
    z = np.zeros(n_src)
    for i in range(n_out):
        for d in range(-half_band, half_band + 1):
            k = i + d
            if 0 <= k < n_src:
                z[k] += op[i, d + half_band] * y[i]
    return z
