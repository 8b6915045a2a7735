"""Denoiser guides (albedo, normal, depth) and the multi-layer EXR.

The guides follow shade_surface.slang:322-340, 488-503 and
shade_miss.slang:52-66: camera rays are fully open, the first hit records
camera-plane depth (+inf on a miss), a surface records its clamped albedo
estimate and shading normal with the fraction the sampled lobe's roughness
ramp gives, near-specular scatters pass the rest on tinted, and the
environment records white albedo. The film adds each buffer with its own
guard (accumulate.slang:38-67). CPU tests pin the oracle's guides on scenes
whose answer is known; GPU tests hold the CUDA path to the oracle.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from cenote_b200 import scenes
from cenote_b200.exr import read_exr, write_aov_exr


def wall_scene(mat, size=24, dist=3.0):
    """A 40×40 quad facing the camera at `dist`, nothing else (black sky)."""
    quad = scenes.quad([(-20, -20, 0), (20, -20, 0), (20, 20, 0), (-20, 20, 0)])
    obj = scenes.Object(quad, scenes.rows(np.eye(4)), mat)
    cam = scenes.Camera((0.0, 0.0, dist), (0.0, 0.0, 0.0), vfov_degrees=40.0)
    env = scenes.Environment.constant((0.0, 0.0, 0.0))
    return scenes.SceneSpec("wall", [obj], cam, env, size, size, 4, 4)


def guides(spec, spp=4, max_bounces=4):
    g = oracle.OracleScene(spec).render_guides(spec.width, spec.height, 0, spp, max_bounces)
    return {k: v / spp for k, v in g.items()}


def test_oracle_guides_on_a_matte_wall():
    base = scenes.acescg((0.6, 0.3, 0.1))
    g = guides(wall_scene(scenes.matte(base)))
    # A rough diffuse surface records everything at the first hit.
    assert np.allclose(g["albedo"][..., :3], base, atol=1e-6)
    assert np.allclose(g["normal"][..., :3], (0.0, 0.0, 1.0), atol=1e-6)
    # Camera-plane z: the same distance across the image, not the ray length.
    assert np.allclose(g["depth"], 3.0, rtol=1e-5)
    assert (g["albedo"][..., 3] == 0).all() and (g["normal"][..., 3] == 0).all()


def test_oracle_guides_on_a_miss():
    spec = wall_scene(scenes.matte(scenes.acescg((0.5, 0.5, 0.5))))
    spec.camera = scenes.Camera((0.0, 0.0, 3.0), (0.0, 0.0, 6.0))  # looking away
    g = guides(spec)
    assert np.isinf(g["depth"]).all() and (g["depth"] > 0).all()
    assert np.allclose(g["albedo"][..., :3], 1.0)
    assert (g["normal"] == 0).all()


def test_oracle_guides_pass_through_a_mirror():
    # A smooth metal records only sqrt(alpha)/0.15 of the guides itself (its
    # roughness floor): the tinted rest reaches the sky (white albedo), so
    # albedo ~ the mirror's tint and the normal is +z times that fraction.
    tint = scenes.acescg((0.9, 0.6, 0.3))
    g = guides(wall_scene(scenes.metal(tint, 0.0)))
    assert np.allclose(g["albedo"][..., :3], tint, atol=1e-3)
    rec = g["normal"][..., 2]
    assert np.abs(g["normal"][..., :2]).max() < 1e-6
    assert 0.0 < rec.min() and rec.max() < 0.5 and np.ptp(rec) < 1e-5


def test_oracle_guides_leave_beauty_untouched():
    spec = scenes.cornell(24, 24, 4, 6)
    s = oracle.OracleScene(spec)
    assert np.array_equal(s.render_sum(24, 24, 0, 4, 6), s.render_guides(24, 24, 0, 4, 6)["beauty"])


def test_aov_exr_layers(tmp_path):
    rng = np.random.default_rng(3)
    b, a, n = (rng.random((3, 5, 4), dtype=np.float32) for _ in range(3))
    d = rng.random((3, 5), dtype=np.float32)
    d[1, 2] = np.inf
    write_aov_exr(tmp_path / "x.exr", b, a, n, d)
    r = read_exr(tmp_path / "x.exr")
    assert sorted(r) == ["A", "B", "G", "R", "Z", "albedo.B", "albedo.G", "albedo.R", "normal.X", "normal.Y",
                         "normal.Z"]
    assert np.array_equal(r["Z"], d)
    assert np.allclose(r["G"], b[..., 1].astype(np.float16)) and np.allclose(r["normal.Y"], n[..., 1], atol=1e-3)


# ---- the CUDA path against the oracle ------------------------------------------------


def gpu_guides(ctx, spec, spp, max_bounces):
    from cenote_b200 import Film, Renderer, Scene

    scene = Scene(ctx, spec)
    r = Renderer(ctx, max_bounces)
    f = Film(ctx, spec.width, spec.height)
    r.accumulate(scene, f, spp)
    return f.all_averages()


def assert_guides_match(got, ref):
    for k in ("albedo", "normal"):
        err = np.abs(got[k] - ref[k])
        # Rare pixels may take a different path after an FP32 rounding fork.
        bad = (err > 1e-4 + 1e-4 * np.abs(ref[k])).any(-1)
        assert bad.mean() <= 0.002, (k, bad.mean(), err.max())
    fin = np.isfinite(ref["depth"])
    assert np.array_equal(fin, np.isfinite(got["depth"]))
    assert np.allclose(got["depth"][fin], ref["depth"][fin], rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_gpu_guides_match_oracle_cornell(ctx):
    spec = scenes.cornell(48, 48, 16, 8)
    assert_guides_match(gpu_guides(ctx, spec, 16, 8), guides(spec, 16, 8))


@pytest.mark.gpu
def test_gpu_guides_match_oracle_chart(ctx):
    spec = scenes.chart(64, 36, 8, 6, env_size=(128, 64))
    assert_guides_match(gpu_guides(ctx, spec, 8, 6), guides(spec, 8, 6))


@pytest.mark.gpu
def test_gpu_guides_known_answers(ctx):
    base = scenes.acescg((0.6, 0.3, 0.1))
    g = gpu_guides(ctx, wall_scene(scenes.matte(base)), 4, 4)
    assert np.allclose(g["albedo"][..., :3], base, atol=1e-6)
    assert np.allclose(g["depth"], 3.0, rtol=1e-5)
    tint = scenes.acescg((0.9, 0.6, 0.3))
    g = gpu_guides(ctx, wall_scene(scenes.metal(tint, 0.0)), 4, 4)
    assert np.allclose(g["albedo"][..., :3], tint, atol=1e-3)


@pytest.mark.gpu
def test_gpu_guides_reset_and_one_sample(ctx):
    from cenote_b200 import Film, Renderer, Scene

    spec = scenes.cornell(32, 32, 4, 6)
    scene, r = Scene(ctx, spec), Renderer(ctx, 6)
    f = Film(ctx, 32, 32)
    r.accumulate(scene, f, 3)
    first = f.all_averages()
    f.reset()
    r.accumulate(scene, f, 3)
    again = f.all_averages()
    for k in first:
        assert np.array_equal(first[k], again[k]), k
    assert math.isclose(float(np.nanmean(np.where(np.isfinite(again["depth"]), again["depth"], np.nan))),
                        float(np.nanmean(np.where(np.isfinite(first["depth"]), first["depth"], np.nan))))
