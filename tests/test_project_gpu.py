"""Template generation on the device (gisspa_project / gisspa_set_templates_from_volume)
against the reference's own projections and the oracle: bit-identical."""
import os

import numpy as np
import pytest

import gisspa
import oracle
from fixture_data import PROJECTION_CASES, bump_volume
from parity import small_case

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def searcher():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    return gisspa.Searcher(cfg)


@pytest.mark.parametrize("name", sorted(PROJECTION_CASES))
def test_projection_equals_reference(searcher, name):
    size, blobs, seed, ri, angles = PROJECTION_CASES[name]
    ref = np.load(os.path.join(GOLDEN, f"project_{name}.npz"))["projections"]
    got = searcher.project(bump_volume(size, blobs, seed), angles, ri)
    assert got.tobytes() == ref.tobytes(), float(np.abs(got - ref).max())


@pytest.mark.parametrize("ri", [0, 25])
def test_projection_equals_oracle_at_any_angle(searcher, ri):
    vol = bump_volume(64, 60, 11)
    rng = np.random.default_rng(4)
    angles = rng.uniform(0.0, 2 * np.pi, (12, 3)).astype(np.float32)
    got = searcher.project(vol, angles, ri)
    ref = oracle.project3d(vol, angles, ri)
    assert np.abs(ref).max() > 0
    assert got.tobytes() == ref.tobytes(), float(np.abs(got - ref).max())


def test_templates_from_volume_search_like_uploaded_templates():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    vol = bump_volume(64, 60, 12)
    angles = np.array([[0.3, 0.2, 0.1], [1.1, 2.0, 0.5], [2.2, 4.1, 1.7], [0.9, 5.5, 3.3]], np.float32)
    a = gisspa.Searcher(cfg)
    a.set_templates_from_volume(vol, angles)
    b = gisspa.Searcher(cfg)
    b.set_templates(a.project(vol, angles))
    pa, pb = a.search(img, ctf), b.search(img, ctf)
    assert len(pa) > 0 and pa.tobytes() == pb.tobytes()
