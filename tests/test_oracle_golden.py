"""Pin the CPU oracle to the reference's own known-answer tests.

Each test restates one of cenote's CPU-side tests against the oracle:
  alias table          crates/cenote/src/lights.rs:320-475
  environment tables   crates/cenote/src/environment.rs:258-324
  colour matrix        crates/cenote/src/color.rs:39-59
  sampler strata       crates/cenote/src/wavefront.rs:1041-1135 (run here on the CPU restatement)
Values and tolerances are the reference's.
"""
import math

import numpy as np
import pytest

import oracle
from cenote_b200 import scenes

KIND_TRIANGLE, KIND_DISTANT, KIND_POINT = 0, 1, 2
LIGHT_NONE = 0xFFFFFFFF
X, Y, Z, ZERO = np.array([1, 0, 0.]), np.array([0, 1, 0.]), np.array([0, 0, 1.]), np.zeros(3)


def luminance(c):
    c = np.asarray(c, np.float32)
    return float(np.float32(np.float32(c[0] * np.float32(0.2722287)) + np.float32(c[1] * np.float32(0.6740818)))
                 + np.float32(c[2] * np.float32(0.0536895)))


def power(rec):
    luma = luminance(rec["emission"])
    if rec["kind"] == KIND_TRIANGLE:
        e1, e2 = rec["edge1"].astype(np.float64), rec["edge2"].astype(np.float64)
        return math.pi * luma * np.linalg.norm(np.cross(e1, e2)) / 2.0
    if rec["kind"] == KIND_DISTANT:
        return luma
    return 4.0 * math.pi * luma


def selection_probability(records, index):
    """The exact probability the kernel's alias walk assigns light `index` (lights.rs:298-313)."""
    mass = 0.0
    for slot, r in enumerate(records):
        t = float(r["alias_threshold"])
        mass += (t if slot == index else 0.0) + ((1.0 - t) if r["alias_index"] == index else 0.0)
    return mass / len(records)


def tri(c, e, inst, prim):
    return (np.asarray(c, np.float32), np.asarray(e, np.float32), inst, prim)


def test_selection_matches_power_share():  # lights.rs:320-360
    tris = [
        tri([ZERO, X, Z], [4, 4, 4], 0, 0),
        tri([ZERO, [1.0, 0.5, 0.0], Z * 2.0], [1, 1, 1], 0, 1),
        tri([Y, Y + X * 3.0, Y + Z], [2.0, 0.5, 3.0], 3, 0),
    ]
    deltas = [(KIND_DISTANT, -Y, [2, 2, 2]), (KIND_POINT, Y * 5.0, [0.25, 0.25, 0.25])]
    recs, total = oracle.build_lights(tris, deltas)
    assert len(recs) == 5
    for i, r in enumerate(recs):
        want = power(r) / total
        got = selection_probability(recs, i)
        assert abs(got - want) < 1e-6, (i, got, want)


def test_pdf_folds_selection_per_kind():  # lights.rs:365-387
    tris = [tri([ZERO, X * 2.0, Z], [1, 1, 1], 0, 0), tri([ZERO, X * 6.0, Z], [1, 1, 1], 7, 0)]
    recs, _ = oracle.build_lights(tris)
    assert abs(recs[0]["pdf"] - 0.25) < 1e-6
    assert abs(recs[1]["pdf"] - 0.25) < 1e-6
    assert recs[1]["instance"] == 7
    recs, _ = oracle.build_lights(tris[:1], [(KIND_POINT, Y, [0.25] * 3)])
    assert abs(recs[1]["pdf"] - 0.5) < 1e-6, recs[1]["pdf"]
    assert recs[1]["instance"] == LIGHT_NONE


def test_triangle_records_keep_input_order():  # lights.rs:392-418
    tris = [tri([ZERO, X, Z], [1, 1, 1], 2, 0), tri([ZERO, X, Z], [1, 1, 1], 2, 1), tri([ZERO, X, Z], [1, 1, 1], 5, 0)]
    recs, _ = oracle.build_lights(tris, [(KIND_DISTANT, -Y, [1, 1, 1])])
    ids = [(int(r["kind"]), int(r["instance"]), int(r["primitive"])) for r in recs]
    assert ids == [(KIND_TRIANGLE, 2, 0), (KIND_TRIANGLE, 2, 1), (KIND_TRIANGLE, 5, 0), (KIND_DISTANT, LIGHT_NONE, 0)]


def test_single_light_never_aliases():  # lights.rs:422-437
    recs, _ = oracle.build_lights([tri([ZERO, X * 2.0, Z * 2.0], [1, 1, 1], 0, 0)])
    assert len(recs) == 1
    assert abs(recs[0]["alias_threshold"] - 1.0) < 1e-7
    assert abs(recs[0]["pdf"] - 0.5) < 1e-6


def test_degenerate_triangles_hold_their_slot_unsampled():  # lights.rs:443-457
    tris = [tri([ZERO, X, X * 2.0], [1, 1, 1], 0, 0), tri([ZERO, X, Z], [1, 1, 1], 0, 1)]
    recs, _ = oracle.build_lights(tris)
    assert len(recs) == 2
    assert recs[0]["pdf"] == 0.0
    assert abs(selection_probability(recs, 0)) < 1e-12
    assert abs(selection_probability(recs, 1) - 1.0) < 1e-9


def test_a_powerless_list_builds_finite():  # lights.rs:463-475
    recs, total = oracle.build_lights([tri([ZERO, X, X * 2.0], [1, 1, 1], 0, 0)])
    assert recs[0]["pdf"] == 0.0
    assert abs(recs[0]["alias_threshold"] - 1.0) < 1e-7
    assert abs(total) < 1e-12


def _image(w, h, lum_at):
    t = np.zeros((h, w, 4), np.float32)
    for r in range(h):
        for c in range(w):
            t[r, c, :3] = lum_at(c, r)
            t[r, c, 3] = 1.0
    return t


def test_env_tables_are_normalized_distributions():  # environment.rs:258-274
    tex = _image(8, 4, lambda c, r: (1 + c + r * 8) * 0.1)
    m, cond, pdfs, _ = oracle.env_tables(8, 4, tex)
    assert m[0] == 0.0 and m[-1] == 1.0
    assert np.all(np.diff(m) >= 0)
    for row in range(4):
        cdf = cond[row * 9:(row + 1) * 9]
        assert cdf[0] == 0.0 and cdf[8] == 1.0
        assert np.all(np.diff(cdf) >= 0)
    assert abs(pdfs.astype(np.float64).mean() - 1.0) < 1e-6


def test_env_support_covers_the_bilinear_footprint():  # environment.rs:281-295
    tex = _image(8, 4, lambda c, r: float(c == 0 and r == 0))
    _, _, pdfs, _ = oracle.env_tables(8, 4, tex)
    for row in range(4):
        for col in range(8):
            inside = row <= 1 and col in (7, 0, 1)
            assert (pdfs[row * 8 + col] > 0.0) == inside, (col, row)


def test_black_environment_has_no_mass():  # environment.rs:300-308
    m, _, pdfs, power_ = oracle.env_tables(1, 1, np.array([[[0, 0, 0, 1]]], np.float32))
    assert power_ == 0.0
    assert np.all(pdfs == 0.0)
    assert m[-1] == 1.0


@pytest.mark.parametrize("w,h", [(1, 1), (8, 4), (13, 7)])
def test_constant_environment_power_is_exact(w, h):  # environment.rs:313-324
    tex = _image(w, h, lambda c, r: 0.5)
    _, _, _, power_ = oracle.env_tables(w, h, tex)
    want = 4.0 * math.pi * luminance([0.5, 0.5, 0.5])
    assert abs(power_ - want) < 1e-9


def test_white_maps_to_white():  # color.rs:39-43
    assert np.allclose(scenes.acescg((1, 1, 1)), 1.0, atol=1e-6)


def test_primaries_match_published_values():  # color.rs:47-59
    cases = [((1, 0, 0), (0.613097, 0.070194, 0.020616)), ((0, 1, 0), (0.339523, 0.916354, 0.109570)),
             ((0, 0, 1), (0.047379, 0.013452, 0.869815))]
    for rgb, want in cases:
        assert np.allclose(scenes.acescg(rgb), want, atol=1e-5)


@pytest.mark.parametrize("pixel,dim", [(0, 0), (7, 0), (123456, 3)])
def test_sampler_is_stratified(pixel, dim):  # wavefront.rs:1041-1126
    pts, vals = oracle.sampler(pixel, dim, 64)
    assert np.all((pts >= 0) & (pts < 1)) and np.all((vals >= 0) & (vals < 1))
    cells = np.zeros(64, int)
    xb, yb, vb = np.zeros(64, int), np.zeros(64, int), np.zeros(64, int)
    for (x, y), v in zip(pts, vals):
        cells[int(y * 8) * 8 + int(x * 8)] += 1
        xb[int(x * 64)] += 1
        yb[int(y * 64)] += 1
        vb[int(v * 64)] += 1
    for bins in (cells, xb, yb, vb):
        assert np.all(bins == 1)


def test_sampler_decorrelates_keys():  # wavefront.rs:1128-1135
    a = oracle.sampler(0, 0, 64)
    assert not np.array_equal(a[0], oracle.sampler(1, 0, 64)[0])
    assert not np.array_equal(a[0], oracle.sampler(0, 1, 64)[0])


def test_sampler_matches_committed_vectors():
    """The oracle's sampler against tests/golden/sampler.npz (made by
    tests/golden/make_golden.py from this restatement, kept to catch drift)."""
    g = np.load(pytest.importorskip("pathlib").Path(__file__).parent / "golden" / "sampler.npz")
    for k, (pixel, dim) in enumerate(g["keys"]):
        pts, vals = oracle.sampler(int(pixel), int(dim), g["points"].shape[1])
        assert np.array_equal(pts, g["points"][k])
        assert np.array_equal(vals, g["values"][k])
