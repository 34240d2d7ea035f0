"""Pins the oracle's metric restatement (mesh/metric.py:31-70) to the
reference's Fortran golden data: test3, two blocks of 51 x 51 x 11 nodes,
Jacobian compared with atol 1e-13 as in the reference's
tests/validation/test_m11_metric_match.py:23-36."""
from pathlib import Path

import numpy as np

from oracle.ref import NP

GOLDEN = Path(__file__).parent / "golden" / "test3_metric.npz"


def test_oracle_metric_matches_fortran_jac():
    data = np.load(GOLDEN)
    for b in (1, 2):
        jac, kxyz, vol = NP.compute_metrics(data[f"xyz{b}"], ghost=0)
        ref = data[f"jac{b}"]
        assert jac.shape == ref.shape == (51, 51, 11)
        diff = np.abs(jac - ref)
        assert diff.max() <= 1e-13, f"block {b}: max abs diff {diff.max():.3e}"
        assert (diff / np.abs(ref)).max() <= 1e-14
        np.testing.assert_array_equal(vol, np.abs(jac))
