"""The oracle's restatement of the reference's volume projection (emdata::project3d) against
projections made by the reference's own code (tests/golden/project_*.npz, from
tests/golden/make_project_golden.py): bit-identical."""
import os

import numpy as np
import pytest

import oracle
from fixture_data import PROJECTION_CASES, bump_volume

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(PROJECTION_CASES))
def test_oracle_projection_equals_reference(name):
    size, blobs, seed, ri, angles = PROJECTION_CASES[name]
    gold = np.load(os.path.join(GOLDEN, f"project_{name}.npz"))
    vol = bump_volume(size, blobs, seed)
    assert float(vol.astype(np.float64).sum()) == float(gold["volume_sum"])  # inputs reproduced exactly
    got = oracle.project3d(vol, angles, ri)
    ref = gold["projections"]
    assert np.abs(ref).max() > 0
    assert got.tobytes() == ref.tobytes(), float(np.abs(got - ref).max())
