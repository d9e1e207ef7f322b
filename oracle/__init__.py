"""CPU oracle for the DWBA radial matrix-element hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy, the algorithm of the reference implementation
(StaryPasterz/DWBA ``dwba_matrix_elements.radial_ME_all_L`` and the quadrature
in ``oscillatory_integrals.py``). Every function cites the reference file:line
it follows. It is the checker against which the CUDA engine in ``dwba_b200`` is
validated, and the CPU baseline that ``bench.py --impl reference`` times.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline
and reference arms) may import this package. The product package
``dwba_b200`` never imports it.

Parity pin: the restatement is checked against golden vectors produced by the
reference itself (``tests/golden/make_golden.py``, which imports the reference
source tree and records inputs and outputs of ``radial_ME_all_L``).
"""
from .quadrature import (  # noqa: F401
    cc_reference,
    check_phase_sampling,
    adaptive_phase_increment,
    generate_phase_nodes,
    is_log_spaced_grid,
    interp_on_radial_grid,
)
from .radial_me import radial_me_all_L, select_idx_limit  # noqa: F401
from .tails import outer_integral_1d, analytical_multipole_tail  # noqa: F401
from .folded import fold_pair, folded_eval, semiseparable_eval  # noqa: F401
