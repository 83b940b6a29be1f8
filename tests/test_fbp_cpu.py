"""FBP filter weights and oracle against the reference's own FBPFilter
(processing/fbp_filter.py run on NumPy arrays by tests/golden/make_golden_fbp.py).
Runs without a GPU: the weights are host arithmetic."""
import os

import numpy as np
import pytest

from oracle.fbp import FILTERS, calc_filter, filter_rows

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fbp_filter.npz"))


@pytest.mark.parametrize("n", [16, 64, 100])
def test_oracle_weights_bit_identical(n):
    for name in FILTERS:
        assert np.array_equal(calc_filter(n, name), GOLD[f"w_{name}_n{n}"]), name


@pytest.mark.parametrize("n,name", [(64, "ramp"), (64, "shepp"), (100, "hann")])
def test_oracle_filter_matches_reference(n, name):
    s, g = GOLD[f"sino_{name}_n{n}"], GOLD[f"filt_{name}_n{n}"]
    r = filter_rows(s, GOLD[f"w_{name}_n{n}"])
    assert np.linalg.norm(r - g) / np.linalg.norm(g) < 2e-7      # golden is float32


@pytest.mark.parametrize("n", [16, 64, 100])
def test_library_weights_match_reference(n):
    from model_mosaic_b200.processing.fbp_filter import filter_weights
    for name in FILTERS:
        assert np.array_equal(filter_weights(n, name), GOLD[f"w_{name}_n{n}"]), name


def test_library_weights_reject_unknown_names():
    from model_mosaic_b200.processing.fbp_filter import filter_weights
    with pytest.raises(ValueError, match="unknown FBP filter"):
        filter_weights(64, "triangle")
    with pytest.raises(ValueError):
        filter_weights(4, "ramp")                                   # too short for the 12-point quadrature
