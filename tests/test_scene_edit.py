"""cenote_scene_add_delta_light: editing a built scene's light list.

The reference builds its light list once from the triangle lights and the
delta lights, in that order (crates/cenote/src/lights.rs:175-275), and picks
between the environment and the lights by their powers
(crates/cenote/src/scene/mod.rs:665-671). Appending a light must leave the
scene exactly as if it had been created with the light last among its deltas.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from cenote_b200 import scenes

pytestmark = pytest.mark.gpu

SUN = scenes.DeltaLight(1, (0.3, -0.9, 0.3160696), (2.0, 1.8, 1.5))
BULB = scenes.DeltaLight(2, (0.1, 1.2, 0.4), (3.0, 2.5, 2.0))


def spec_with(deltas):
    spec = scenes.cornell(48, 48, 4, 6)
    return dataclasses.replace(spec, delta_lights=list(spec.delta_lights) + list(deltas))


def render(ctx, scene, spec, spp=4):
    from cenote_b200 import Film, Renderer

    f = Film(ctx, spec.width, spec.height)
    Renderer(ctx, 6).accumulate(scene, f, spp)
    return f.averages()


@pytest.mark.parametrize("first, added", [([], [BULB]), ([SUN], [BULB]), ([], [SUN, BULB])])
def test_added_lights_match_a_scene_built_with_them(ctx, first, added):
    from cenote_b200 import Scene

    edited = Scene(ctx, spec_with(first))
    for light in added:
        edited.add_delta_light(light)
    built_spec = spec_with(first + added)
    built = Scene(ctx, built_spec)
    assert edited.light_records().tobytes() == built.light_records().tobytes()
    assert np.array_equal(render(ctx, edited, built_spec), render(ctx, built, built_spec))


def test_a_light_added_to_an_environment_lit_scene_takes_its_share(ctx):
    from cenote_b200 import Scene

    spec = scenes.furnace(scenes.matte((0.5, 0.5, 0.5), 1.0))
    s = Scene(ctx, spec)
    assert len(s.light_records()) == 0
    before = render(ctx, s, spec, 16)
    s.add_delta_light(scenes.DeltaLight(2, (0.0, 0.5, -0.5), (1.0, 1.0, 1.0)))
    recs = s.light_records()
    assert len(recs) == 1 and recs["pdf"][0] == np.float32(1.0)
    ref = Scene(ctx, dataclasses.replace(spec, delta_lights=[scenes.DeltaLight(2, (0.0, 0.5, -0.5), (1.0, 1.0, 1.0))]))
    assert np.array_equal(render(ctx, s, spec, 16), render(ctx, ref, spec, 16))
    assert not np.array_equal(before, render(ctx, s, spec, 16))


def test_an_invalid_light_is_refused(ctx):
    from cenote_b200 import CenoteError, Scene

    s = Scene(ctx, spec_with([]))
    n = len(s.light_records())
    with pytest.raises(CenoteError):
        s.add_delta_light(scenes.DeltaLight(7, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)))
    with pytest.raises(CenoteError):
        s.add_delta_light(scenes.DeltaLight(2, (float("nan"), 0.0, 0.0), (1.0, 1.0, 1.0)))
    assert len(s.light_records()) == n
