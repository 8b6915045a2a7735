"""Guided path sampling with the learned guide (cenote_renderer_set_guide).

The guide only proposes directions: every guided vertex weighs its sample by
the one-sample-MIS pdf alpha q + (1 - alpha) p_bsdf, and next-event MIS uses
the same pdf, so the estimator stays unbiased whatever the network outputs.
The tests check exactly that (furnaces and agreement with plain sampling under
an untrained, randomly initialised guide), determinism with a frozen guide,
and what online training gains on a box lit only by a bounce off its ceiling,
where next-event estimation cannot reach the light from most surfaces.
"""
from __future__ import annotations

import numpy as np
import pytest

from cenote_b200 import Film, Guide, Renderer, Scene, scenes
from cenote_b200.metrics import rel_mse

pytestmark = pytest.mark.gpu
WHITE = (1.0, 1.0, 1.0)


def render(ctx, spec, spp, guide=None, fraction=0.5, steps=0, lr=1e-2, spw=0, bounces=8, scene=None, film=None):
    r = Renderer(ctx, bounces, samples_per_wave=spw)
    if guide is not None:
        r.set_guide(guide, fraction, steps, lr)
    s = scene or Scene(ctx, spec)
    f = film or Film(ctx, spec.width, spec.height)
    r.accumulate(s, f, spp)
    return f.averages()


@pytest.mark.parametrize("mat, expect", [(scenes.matte(WHITE, 1.0), 0.5), (scenes.metal(WHITE, 0.5), None)])
def test_guided_furnace_is_unbiased(ctx, mat, expect):
    spec = scenes.furnace(mat)
    plain = render(ctx, spec, 256)
    g = Guide(ctx, seed=5)
    guided = render(ctx, spec, 256, guide=g)
    m_g, m_p = guided[..., 0].mean(), plain[..., 0].mean()
    if expect is not None:
        assert abs(m_g - expect) < 0.006, m_g
    assert abs(m_g - m_p) < 0.01 * max(m_p, 0.1), (m_g, m_p)


def test_guided_agrees_with_plain_sampling(ctx):
    spec = scenes.cornell(32, 32, 8, 8)
    plain = render(ctx, spec, 2048)
    g = Guide(ctx, seed=6)
    guided = render(ctx, spec, 2048, guide=g, steps=2, spw=16)
    assert abs(guided[..., :3].mean() / plain[..., :3].mean() - 1.0) < 0.01
    assert rel_mse(guided[..., :3], plain[..., :3]) < 0.01


def test_frozen_guide_is_deterministic(ctx):
    spec = scenes.cornell(24, 24, 4, 6)
    g = Guide(ctx, seed=7)
    a = render(ctx, spec, 8, guide=g, bounces=6)
    b = render(ctx, spec, 8, guide=g, bounces=6)
    assert np.array_equal(a, b)


def test_trained_guide_lowers_error_at_equal_samples(ctx):
    size, spp = 48, 32
    spec = scenes.ceiling_box(size, size, 16, 8)
    scene = Scene(ctx, spec)
    r = Renderer(ctx, 8)
    f = Film(ctx, size, size)
    r.accumulate_range(scene, f, 1 << 24, 8192)  # shares no samples with the renders it judges
    ref = f.averages()[..., :3]
    plain = render(ctx, spec, spp, scene=scene)[..., :3]
    g = Guide(ctx, seed=8)
    # Train online over 1,024 samples per pixel, then render with the trained
    # guide (still training) at the same sample count as the plain render.
    render(ctx, spec, 1024, guide=g, steps=4, lr=5e-3, spw=16, scene=scene)
    guided = render(ctx, spec, spp, guide=g, steps=4, lr=5e-3, spw=8, scene=scene)[..., :3]
    e_plain, e_guided = rel_mse(plain, ref), rel_mse(guided, ref)
    print(f"relMSE plain {e_plain:.4f} guided {e_guided:.4f}")
    assert e_guided < 0.9 * e_plain, (e_plain, e_guided)
