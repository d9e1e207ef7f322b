"""``semantics="cupy"``: the GPU engine against the reference's recorded CuPy-path outputs.

tests/golden/cupy_semantics.npz holds what the reference's ``radial_ME_all_L_gpu``
(``dwba_matrix_elements.py:1563-2549``) returns on the inputs of the golden cases (recorded on the
CPU through a NumPy stand-in for CuPy by tests/golden/make_cupy_golden.py). The CuPy mode
(dwba_b200/cupy_mode.py: node sets with linear interpolation, folds, multipole potentials and dot
forms, the CuPy exchange kernels of cupy_nodes.cu, semiseparable forms for the standard branch)
must reproduce them in FP64, per call and batched.
"""
import json
from collections import defaultdict

import numpy as np
import pytest

import golden_cases as gc

pytestmark = pytest.mark.gpu

CUPY = np.load(gc.GOLDEN_DIR + "/cupy_semantics.npz")
CALLS = [c for c in gc.all_calls() if not c["label"].startswith("large_grid")]
REL, ABS = 1e-10, 1e-12


def _key(call):
    name, idx = call["label"].rstrip("]").split("[")
    return f"{name}_{idx}"


def _close(got, ref):
    return np.all(np.abs(got - ref) <= REL * np.abs(ref) + ABS * np.max(np.abs(ref)))


@pytest.mark.parametrize("call", CALLS, ids=[c["label"] for c in CALLS])
def test_single_call_matches_reference_cupy_path(call):
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_gpu
    res = radial_ME_all_L_gpu(*call["args"], **call["kwargs"], semantics="cupy")
    L = call["L_max"]
    d = np.array([res.I_L_direct[l] for l in range(L + 1)])
    e = np.array([res.I_L_exchange[l] for l in range(L + 1)])
    k = _key(call)
    assert _close(d, CUPY[k + "_dir"]), (k, d, CUPY[k + "_dir"])
    assert _close(e, CUPY[k + "_exc"]), (k, e, CUPY[k + "_exc"])


def test_batched_calls_match_reference_cupy_path():
    """Every case's calls with equal L_max and options in one batched call per group."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_batch
    groups = defaultdict(list)
    for c in CALLS:
        groups[(c["label"].split("[")[0], c["L_max"], json.dumps(
            {k: v for k, v in c["kwargs"].items() if k != "U_f_array"}, sort_keys=True))].append(c)
    assert len(groups) >= 4
    for calls in groups.values():
        grid, V, U, bi, bf, _, _, L = calls[0]["args"]
        kw = dict(calls[0]["kwargs"])
        pairs = [(c["args"][5], c["args"][6]) for c in calls]
        d, e = radial_ME_all_L_batch(grid, V, U, bi, bf, pairs, L, **kw, semantics="cupy", as_arrays=True)
        for p, c in enumerate(calls):
            k = _key(c)
            assert _close(d[p], CUPY[k + "_dir"]), (k, d[p], CUPY[k + "_dir"])
            assert _close(e[p], CUPY[k + "_exc"]), (k, e[p], CUPY[k + "_exc"])


def test_the_two_semantics_differ_where_the_reference_paths_do():
    """The CPU-path semantics (default) give the CPU goldens, the CuPy semantics the CuPy goldens, and
    the two differ by more than round-off on the phase-split cases."""
    from dwba_b200.dwba_matrix_elements import radial_ME_all_L_gpu
    differ = 0
    for c in CALLS:
        L = c["L_max"]
        cpu = radial_ME_all_L_gpu(*c["args"], **c["kwargs"])
        d = np.array([cpu.I_L_direct[l] for l in range(L + 1)])
        differ += int(not _close(d, CUPY[_key(c) + "_dir"]))
    assert differ >= 3
