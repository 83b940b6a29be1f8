"""Paganin oracle and the library's filter table against the reference's own
Paganin (processing/paganin.py run on NumPy arrays by
tests/golden/make_golden_paganin.py).  No GPU needed."""
import os

import numpy as np
import pytest

from oracle.paganin import paganin_filter, retrieve

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "paganin.npz"))


@pytest.mark.parametrize("L", [0.02, 0.1, 1.0])
def test_oracle_and_table_vs_reference(L):
    from model_mosaic_b200.processing.paganin import paganin_table
    f = paganin_filter(64, 32, 4.13e-11, 1.4e-6, L, 1e-3)
    assert np.array_equal(f, GOLD[f"filt_L{L}"])
    assert np.array_equal(paganin_table(64, 32, 4.13e-11, 1.4e-6, L, 1e-3), GOLD[f"filt_L{L}"])
    g = GOLD[f"phase_L{L}"]
    assert np.linalg.norm(retrieve(GOLD["intensity"], f) - g) / np.linalg.norm(g) < 1e-6
