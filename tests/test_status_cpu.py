"""Host-side failure handling (CPU): status flags and NaN propagation in the oracle."""
from __future__ import annotations

import warnings

import numpy as np
import pytest

from oracle import tet4
from psierra_b200.assembler import raise_if_wait_gave_up


def test_wait_flag_is_raised_and_other_flags_are_not():
    for flags in (0, 2, 4, 6):  # PCG status bits, not a wait
        raise_if_wait_gave_up(flags)
    for flags in (1, 3, 5, 7):
        with pytest.raises(RuntimeError, match="bounded wait"):
            raise_if_wait_gave_up(flags)


def test_reference_element_propagates_nan_without_raising():
    # element/tet4_total_lagrangian.py:110-112 tests only J <= 0.0, which is false for NaN
    X = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    u = np.zeros((4, 3))
    u[2, 1] = np.nan
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        k, f = tet4.force_and_tangent(X, u, 1e3, 5e3)
    assert np.isnan(f).all() and np.isnan(k).all()
