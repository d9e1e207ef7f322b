"""dwba_multipole_potentials through the C ABI at the chunk boundaries of its kernel.

The kernel splits each potential into chunks of 1024 rows; CTAs stride over the chunks, sum the
prefix and suffix series of the columns outside their chunk, and scan inside it. The row and column
counts here put the chunk ends on, just before and just after every boundary (1, 1023, 1024, 1025,
2049 rows), with n_rows < n_cols, n_rows > n_cols, a stride above n_rows, L_max = 0, 8 and 14 (two
launches of up to 12 multipoles), and enough potentials in one call that CTAs loop over several
chunks. Checked against a dense long-double restatement of
    phi_L(p) = sum_{q<n_cols} K_L(r_p, r_q) b_q,  K_L = (1/r_>) min(r_</r_>, 1-1e-12)^L
(the inner integral int_r2 of the reference's Filon direct term, oscillatory_integrals.py:2571), with
|dphi| <= 1e-14 sum_q |K_L(r_p, r_q) b_q| per row.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dense(r, b, n_rows, n_cols, L_max):
    rl = np.longdouble
    rr = r.astype(rl)
    lo = np.minimum(rr[:n_rows, None], rr[None, :n_cols])
    hi = np.maximum(rr[:n_rows, None], rr[None, :n_cols])
    ratio = np.minimum(lo / hi, rl(1.0) - rl(1e-12))
    bb = b[:n_cols].astype(rl)
    out, scale = [], []
    for L in range(L_max + 1):
        K = ratio ** L / hi
        out.append((K @ bb).astype(float))
        scale.append((np.abs(K) @ np.abs(bb)).astype(float))
    return np.array(out), np.array(scale)


@pytest.mark.parametrize("L_max", [0, 8, 14])
def test_potentials_at_chunk_boundaries(L_max):
    import torch
    from dwba_b200 import _lib
    from dwba_b200.engine import _ptr, _stream
    lib = _lib.load()
    rng = np.random.default_rng(17 + L_max)
    N = 2600
    r = np.geomspace(1e-3, 40.0, N) if L_max < 14 else np.geomspace(1e-2, 20.0, N)
    shapes = [(1, 1), (1, 900), (1023, 1023), (1024, 1024), (1025, 1025), (1024, 600), (700, 2049),
              (2049, 2049), (2049, 1500), (2600, 2600), (1025, 2600)]
    shapes = shapes * 30  # 330 potentials: several chunks per CTA
    dev = torch.device("cuda", 0)
    r_d = torch.tensor(r, device=dev)
    nl = L_max + 1
    bs = [rng.normal(size=N) * np.exp(-r / rng.uniform(1.0, 10.0)) for _ in shapes]
    b_d = torch.tensor(np.array(bs), device=dev)
    strides = [n_rows + (7 if i % 3 == 0 else 0) for i, (n_rows, _) in enumerate(shapes)]
    offs = np.concatenate([[0], np.cumsum([nl * s for s in strides])[:-1]]).astype(np.int64)
    phi = torch.full((int(offs[-1]) + nl * strides[-1],), np.nan, dtype=torch.float64, device=dev)
    rec = np.zeros(len(shapes), dtype=_lib.POTENTIAL_DTYPE)
    rec["r"] = _ptr(r_d)
    rec["b"] = _ptr(b_d) + 8 * N * np.arange(len(shapes), dtype=np.uint64)
    rec["phi"] = _ptr(phi) + 8 * offs.astype(np.uint64)
    rec["n_rows"] = [s[0] for s in shapes]
    rec["n_cols"] = [s[1] for s in shapes]
    rec["stride"] = strides
    rec_d = torch.from_numpy(rec.view(np.uint8).copy()).to(dev)
    ds = np.array([(1.0 - 1e-12) ** L for L in range(nl)])
    _lib.check(lib.dwba_multipole_potentials(_ptr(rec_d), len(shapes), L_max, ds.ctypes.data, float(r[0]),
                                             float(r[-1]), _stream()), "dwba_multipole_potentials")
    got = phi.cpu().numpy()
    checked = {}
    for i, (n_rows, n_cols) in enumerate(shapes):
        m = got[offs[i]: offs[i] + nl * strides[i]].reshape(nl, strides[i])
        assert np.all(np.isnan(m[:, n_rows:])), (i, "rows beyond n_rows were written")
        key = (i % 11, n_rows, n_cols)
        if i >= 22 and key in checked:
            continue  # the later copies differ only in b: check a few of them in full
        ref, scale = _dense(r, bs[i], n_rows, n_cols, L_max)
        err = np.abs(m[:, :n_rows] - ref)
        assert np.all(err <= 1e-14 * scale), (i, n_rows, n_cols, float(np.max(err / scale)))
        checked[key] = True
