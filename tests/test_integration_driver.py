"""The drop-in recipe of INTEGRATION.md under the reference's own driver (CPU test).

The recipe (the code block of INTEGRATION.md section 1, read from that file) is appended to the
reference's ``dwba_matrix_elements`` module, and the reference's ``driver.compute_total_excitation_cs``
(``driver.py:646``) runs an H 1s->2p excitation in a child process:

* without a usable GPU (this host): ``HAS_CUPY`` is true (the engine library loads) but
  ``check_cupy_runtime()`` is false, so the driver's selection (``driver.py:856-862``) takes its CPU
  branch and the reference's own ``radial_ME_all_L`` runs in the driver's worker pool
  (``driver.py:1184``, ``:420``); the engine is never called;
* the GPU branch, exercised on the CPU: with ``check_cupy_runtime`` answering true, the driver
  creates its ``GPUCache`` through the engine's class and calls the engine's ``radial_ME_all_L_gpu``
  with its own arguments (``driver.py:1016-1029``); a recorder in its place checks that those
  arguments bind to the engine's signature and evaluates the pair with the reference's CPU
  function, so the cross section equals the CPU branch's.

The reference is imported from the directory named by ``DWBA_REFERENCE_PATH``; the test is
skipped when it is not set (the reference tree is not part of this repository).
"""
import json
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("DWBA_REFERENCE_PATH")

pytestmark = pytest.mark.skipif(not REF or not os.path.exists(os.path.join(REF or "", "driver.py")),
                                reason="DWBA_REFERENCE_PATH (the reference source tree) is not set")

CHILD = r'''
import json, logging, os, sys
import numpy as np
import scipy.special as ss
if not hasattr(ss, "sph_harm"):  # removed in SciPy 1.18; the reference's coupling module imports it
    ss.sph_harm = lambda m, n, phi, theta: ss.sph_harm_y(n, m, theta, phi)
root, ref, mode, log_path = sys.argv[1:5]
sys.path.insert(0, root)
sys.path.insert(0, ref)
logging.disable(logging.WARNING)
import dwba_matrix_elements as dme
cpu_fn = dme.radial_ME_all_L
exec(compile(sys.stdin.read(), "INTEGRATION.md", "exec"), dme.__dict__)   # the recipe
import dwba_b200.dwba_matrix_elements as eng
assert dme.radial_ME_all_L is cpu_fn
assert dme.radial_ME_all_L_gpu is eng.radial_ME_all_L_gpu and dme.GPUCache is eng.GPUCache
assert dme.check_cupy_runtime is eng.check_cupy_runtime and dme.HAS_CUPY is eng.HAS_CUPY

def record(*what):
    with open(log_path, "a") as fh:
        fh.write(json.dumps(what) + "\n")

def cpu_recorded(*a, **k):
    record("cpu")
    return cpu_fn(*a, **k)
dme.radial_ME_all_L = cpu_recorded
runtime = dme.check_cupy_runtime()
if mode == "gpu_branch":
    import inspect
    sig = inspect.signature(eng.radial_ME_all_L_gpu)

    def gpu_recorded(*a, **k):
        sig.bind(*a, **k)  # TypeError if the driver's arguments do not fit the engine's signature
        record("gpu", sorted(k), type(k.get("gpu_cache")).__name__)
        keep = ("use_oscillatory_quadrature", "oscillatory_method", "CC_nodes", "phase_increment",
                "min_grid_fraction", "k_threshold", "U_f_array")
        return cpu_fn(*a, **{n: k[n] for n in keep if n in k})

    class GPUCache(eng.GPUCache):
        def __init__(self, grid, max_chi_cached=20, device=None):  # no device here: record only
            self.grid, self.max_chi_cached = grid, max_chi_cached
            record("cache", int(max_chi_cached))

        def clear(self):
            record("clear")
    dme.radial_ME_all_L_gpu, dme.GPUCache = gpu_recorded, GPUCache
    dme.check_cupy_runtime = lambda: True
import driver  # binds the names with its own import lines
from potential_core import CorePotentialParams
chan = driver.ExcitationChannelSpec(l_i=0, l_f=1, n_index_i=1, n_index_f=1, N_equiv=1, L_max_integrals=2,
                                    L_target_i=0, L_target_f=1, L_max_projectile=6)
core = CorePotentialParams(Zc=1.0, a1=0.0, a2=0.0, a3=0.0, a4=0.0, a5=0.0, a6=0.0)
res = driver.compute_total_excitation_cs(20.0, chan, core, r_max=60.0, n_points=500, n_theta=19)
print(json.dumps({"runtime": bool(runtime), "has_cupy": bool(dme.HAS_CUPY), "tcs": float(res.sigma_total_au)}))
'''


def _recipe() -> str:
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```python\n(.*?)```", text, flags=re.S)
    recipe = [b for b in blocks if "try:" in b and "radial_ME_all_L_gpu, HAS_CUPY, check_cupy_runtime" in b]
    assert len(recipe) == 1, "INTEGRATION.md must hold exactly one drop-in recipe block"
    return recipe[0]


def _run(mode, tmp_path):
    log = tmp_path / f"{mode}.log"
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", ""))
    p = subprocess.run([sys.executable, "-c", CHILD, ROOT, REF, mode, str(log)], input=_recipe(), text=True,
                       capture_output=True, timeout=900, env=env)
    assert p.returncode == 0, p.stderr[-4000:]
    out = json.loads(p.stdout.strip().splitlines()[-1])
    calls = [json.loads(line) for line in log.read_text().splitlines()] if log.exists() else []
    return out, calls


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="needs a host without a usable GPU")
def test_driver_with_recipe_cpu_and_gpu_branches(tmp_path):
    cpu, cpu_calls = _run("cpu", tmp_path)
    assert cpu["has_cupy"] and not cpu["runtime"]            # library present, no usable GPU
    assert cpu_calls and all(c[0] == "cpu" for c in cpu_calls)  # CPU branch: the reference's own path
    gpu, gpu_calls = _run("gpu_branch", tmp_path)
    kinds = [c[0] for c in gpu_calls]
    assert "cpu" not in kinds and kinds.count("gpu") >= len(cpu_calls) // 2
    assert kinds[0] == "cache" and "clear" in kinds             # GPUCache.from_grid per energy, then clear()
    kw = next(c for c in gpu_calls if c[0] == "gpu")
    assert {"gpu_cache", "gpu_block_size", "gpu_memory_mode", "U_f_array"} <= set(kw[1]) and kw[2] == "GPUCache"
    assert gpu["tcs"] > 0 and abs(gpu["tcs"] - cpu["tcs"]) <= 1e-10 * cpu["tcs"]
