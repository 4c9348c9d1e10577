"""The CPU restatement (oracle/cast_oracle.c) pinned against the reference's own answers.

tests/golden/cast_reference.npz holds the compiled reference's closest-hit ids, hit
distances and occlusion bits (Builder_SAH(16,64,4) + Tree::intersect / intersect_p) for
seeded inputs.  The restatement must agree on every ray except disagreements explained by
rounding at a triangle edge or an equal-t tie (the reference's rcpss reciprocal and its
last-tested tie rule), and its hit distances must be within 2 ulp where the ids agree.
"""

import hashlib
import json
import pathlib

import numpy as np
import pytest

import oracle
import sprout_b200 as sb
from cases import MISS, classify_mismatches, edge_rays

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "cast_reference.npz"
CASES = {"sphere32": (32, 65536, 7, True), "sphere128": (128, 16384, 9, True),
         "bench512": (512, 16384, 1, False)}


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def golden():
    data = np.load(GOLDEN)
    meta = json.loads(bytes(data["meta"]).decode())
    return data, meta


def _inputs(name):
    n, count, seed, with_edges = CASES[name]
    pos, idx = sb.sphere_mesh(n, 0.1, 1)
    rays = sb.random_rays(count, seed=seed)
    if with_edges:
        rays = np.concatenate([rays, edge_rays(pos, idx)])
    return pos, idx, rays


@pytest.mark.parametrize("name", list(CASES))
def test_inputs_regenerate_bit_identical(golden, name):
    _, meta = golden
    pos, idx, rays = _inputs(name)
    assert _digest(pos, idx) == meta["cases"][name]["mesh_sha256"]
    assert _digest(rays) == meta["cases"][name]["rays_sha256"]


@pytest.mark.parametrize("name", list(CASES))
def test_restatement_matches_reference(golden, name):
    data, _ = golden
    pos, idx, rays = _inputs(name)
    ref_ids = data[f"{name}_ids"]
    ref_t = data[f"{name}_t"]
    ref_occ = data[f"{name}_occ"]
    got = oracle.restated_cast(pos, idx, rays)

    explained, unexplained = classify_mismatches(pos, idx, rays, ref_ids, ref_t, got["ids"], got["t"],
                                                 oracle.triangle_test)
    assert unexplained == [], f"unexplained id mismatches at rays {unexplained[:10]}"
    # Random rays rarely pass within rounding distance of an edge; the hand-made edge rays
    # (after the first `count`) aim at shared edges and vertices on purpose.
    count = CASES[name][1]
    random_explained = [i for i in explained if i < count]
    assert len(random_explained) <= max(2, 1e-4 * count)

    same = ref_ids == got["ids"]
    ulps = np.abs(ref_t[same].view(np.int32).astype(np.int64) - got["t"][same].view(np.int32))
    assert ulps.max() <= 2

    occ_diff = np.nonzero(ref_occ != got["occluded"])[0]
    assert np.count_nonzero(occ_diff < count) <= max(2, 1e-4 * count)
    # every occlusion disagreement is also an edge case of the closest-hit query
    assert set(occ_diff.tolist()) <= set(explained)


def test_brute_force_equals_bvh_oracle():
    pos, idx = sb.sphere_mesh(16, 0.1, 1)
    rays = np.concatenate([sb.random_rays(20000, seed=11), edge_rays(pos, idx)])
    a = oracle.restated_cast(pos, idx, rays, brute=True)
    b = oracle.restated_cast(pos, idx, rays)
    assert np.array_equal(a["ids"], b["ids"])
    assert np.array_equal(a["t"].view(np.uint32), b["t"].view(np.uint32))
    assert np.array_equal(a["uv"].view(np.uint32), b["uv"].view(np.uint32))
    assert np.array_equal(a["occluded"], b["occluded"])


def test_any_hit_agrees_with_closest_hit():
    pos, idx = sb.sphere_mesh(32, 0.1, 1)
    rays = np.concatenate([sb.random_rays(50000, seed=5), edge_rays(pos, idx)])
    r = oracle.restated_cast(pos, idx, rays)
    assert np.array_equal(r["occluded"] == 1, r["ids"] != MISS)


def test_duplicate_triangles_tie_to_smaller_index():
    pos = np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], np.float32)
    idx = np.array([[0, 1, 2], [0, 1, 2], [0, 1, 2]], np.uint32)
    rays = np.array([[0, 0, -1, 0, 0, 0, 1, 10]], np.float32)
    r = oracle.restated_cast(pos, idx, rays)
    assert r["ids"][0] == 0 and r["t"][0] == 1.0


def test_tree_independence_on_degenerate_mesh():
    """Zero-area and sliver triangles: the hit definition (test passes and the hit point lies
    within the triangle's bounds widened by the hit margin) keeps brute force and any
    conservative tree in agreement, bit for bit."""
    rng = np.random.default_rng(4)
    pos = rng.normal(size=(3000, 3)).astype(np.float32)
    pos[:500] = pos[0]
    pos[500:1000, 2] = 0.25
    idx = rng.integers(0, 3000, size=(5000, 3)).astype(np.uint32)
    idx[:200] = [0, 1, 2]
    with np.errstate(invalid="ignore"):
        rays = np.concatenate([sb.random_rays(20000, seed=2, extent=3.0), edge_rays(pos, idx[200:])])
    a = oracle.restated_cast(pos, idx, rays, brute=True)
    b = oracle.restated_cast(pos, idx, rays)
    assert np.array_equal(a["ids"], b["ids"])
    assert np.array_equal(a["t"].view(np.uint32), b["t"].view(np.uint32))
    assert np.array_equal(a["occluded"], b["occluded"])


@pytest.mark.parametrize("n", [1, 7, 64, 512])
def test_synthesis_restatement_matches_the_product(n):
    """The bench's reference arm makes the benchmark mesh and rays with the oracle's C
    restatement (so that it loads no product code); both must be the product's bit for bit."""
    want_pos, want_idx = sb.sphere_mesh(n, 0.1, 1)
    pos, idx = oracle.synth_sphere_mesh(n, 0.1, 1)
    assert np.array_equal(idx, want_idx)
    assert np.array_equal(pos.view(np.uint32), want_pos.view(np.uint32))


@pytest.mark.parametrize("first,count,seed,extent", [(0, 200000, 1, 2.0), ((1 << 24) - 5000, 10000, 1, 2.0),
                                                     (12345, 3000, 9, 3.0)])
def test_ray_synthesis_restatement_matches_the_product(first, count, seed, extent):
    want = sb.random_rays(count, seed=seed, first=first, extent=extent)
    got = oracle.synth_rays(count, seed=seed, first=first, extent=extent)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
