"""B200-native engine for the DWBA radial matrix elements (direct and exchange I_L).

``dwba_b200.dwba_matrix_elements`` is the drop-in for the reference module of the
same name; ``libdwba_b200.so`` (C ABI in ``include/dwba_b200.h``) holds the
sm_100a kernels.
"""
from . import _lib  # noqa: F401

__all__ = ["dwba_matrix_elements"]
