"""The launch knobs: material sort before shading, wave size, refill threshold,
and the autotuner that picks them per scene.

Every knob only reorders or regroups work: each path's arithmetic and random
numbers are keyed by its pixel and sample, never by its queue slot, and
equal-distance hits resolve by (instance, primitive) whatever the traversal
order, so every setting must give the same film bit for bit, and the same ray
counts.
"""
from __future__ import annotations

import numpy as np
import pytest

from cenote_b200 import SORT_ALL, SORT_NONE, SORT_SECONDARY, scenes

pytestmark = pytest.mark.gpu


def run(ctx, spec, mode, spp, bounces, spw=0):
    from cenote_b200 import Film, Renderer, Scene

    r = Renderer(ctx, bounces, samples_per_wave=spw, material_sort=mode)
    f = Film(ctx, spec.width, spec.height)
    r.accumulate(Scene(ctx, spec), f, spp)
    st = r.stats()
    return f.all_averages(), (st["extension_rays"], st["shadow_rays"], st["overflow"])


@pytest.mark.parametrize("name", ["cornell", "chart", "textured"])
def test_every_sort_mode_gives_the_same_film(ctx, name):
    spec = {"cornell": lambda: scenes.cornell(64, 64, 8, 8), "chart": lambda: scenes.chart(96, 54, 4, 8),
            "textured": lambda: scenes.textured(64, 48, 4, 6)}[name]()
    base, counts = run(ctx, spec, SORT_NONE, spec.spp, spec.max_bounces)
    assert counts[2] == 0
    for mode in (SORT_ALL, SORT_SECONDARY):
        got, c = run(ctx, spec, mode, spec.spp, spec.max_bounces, spw=2)
        assert c == counts
        for k in base:
            assert np.array_equal(got[k], base[k], equal_nan=True), (mode, k)


def test_split_shading_of_a_mixed_scene_matches(ctx):
    """A sorted bounce of a scene mixing layered and layer-free materials
    shades its layer-free range without the coat, fuzz and transmission
    lobes: the film agrees with unsorted shading (every path through the
    full kernel) but for the compiler's fused multiply-adds, and the ray
    counts agree exactly."""
    import dataclasses

    spec = scenes.cornell(64, 64, 8, 8)
    objs = list(spec.objects)
    k = max(range(len(objs)), key=lambda i: objs[i].mesh.triangle_count)  # a box
    objs[k] = dataclasses.replace(objs[k], material=scenes.glass(0.2, 1.5))
    spec = dataclasses.replace(spec, objects=objs)
    base, counts = run(ctx, spec, SORT_NONE, spec.spp, spec.max_bounces)
    got, c = run(ctx, spec, SORT_ALL, spec.spp, spec.max_bounces)
    assert c == counts and counts[2] == 0
    # An ulp can flip a Russian-roulette draw that sits on its threshold, so
    # a rare pixel may differ by a path; nearly all agree to ulps.
    for key in base:
        a, b = base[key], got[key]
        fin = np.isfinite(a)
        assert np.array_equal(fin, np.isfinite(b))
        close = np.abs(a[fin] - b[fin]) <= 1e-5 * np.abs(a[fin]) + 1e-30
        assert close.mean() >= 0.995, (key, close.mean())


def test_sorted_render_once_matches(ctx):
    from cenote_b200 import Renderer, Scene

    spec = scenes.cornell(40, 30, 1, 8)
    scene = Scene(ctx, spec)
    a = Renderer(ctx, 8).render(scene, 40, 30, 3)
    b = Renderer(ctx, 8, material_sort=SORT_ALL).render(scene, 40, 30, 3)
    assert np.array_equal(a, b)


def test_unknown_mode_is_refused(ctx):
    from cenote_b200 import CenoteError, Renderer

    with pytest.raises(CenoteError):
        Renderer(ctx, 4).set_material_sort(3)


def test_tuning_knobs_leave_the_film_unchanged(ctx):
    from cenote_b200 import Film, Renderer, Scene

    spec = scenes.chart(96, 54, 4, 8)
    scene = Scene(ctx, spec)
    films = []
    for knobs in [(SORT_NONE, 0, 0, 0, 0, 0), (SORT_ALL, 1, 4, 80, 1, 1), (SORT_SECONDARY, 4, 16, 320, 0, 0),
                  (SORT_ALL, 2, 32, 1, 1, 0), (SORT_NONE, 3, 8, 7, 0, 1), (SORT_ALL, 0, 8, 0, 0, 1)]:
        r = Renderer(ctx, 8)
        r.set_tuning(*knobs)
        f = Film(ctx, spec.width, spec.height)
        r.accumulate(scene, f, 4)
        films.append(f.averages())
    for f in films[1:]:
        assert np.array_equal(f, films[0])


def test_autotune_picks_a_valid_setting_and_keeps_it(ctx):
    from cenote_b200 import Film, Renderer, Scene

    spec = scenes.cornell(128, 96, 8, 8)
    scene = Scene(ctx, spec)
    r = Renderer(ctx, 8)
    t = r.autotune(scene, spec.width, spec.height)
    assert t["material_sort"] in (SORT_NONE, SORT_ALL, SORT_SECONDARY)
    assert t["refill_idle"] in (0, 4, 8, 16) and t["top_nodes"] in (0, 80, 320) and t["ms_per_sample"] > 0
    kept = r.tuning()
    knobs = ("material_sort", "samples_per_wave", "refill_idle", "top_nodes", "l2_window", "per_lane_triangles")
    assert {k: kept[k] for k in knobs} == {k: t[k] for k in knobs}
    f, g = Film(ctx, spec.width, spec.height), Film(ctx, spec.width, spec.height)
    r.accumulate(scene, f, 8)
    Renderer(ctx, 8).accumulate(scene, g, 8)
    assert np.array_equal(f.averages(), g.averages())


def test_bad_tuning_is_refused(ctx):
    from cenote_b200 import CenoteError, Renderer

    r = Renderer(ctx, 4)
    with pytest.raises(CenoteError):
        r.set_tuning(SORT_ALL, 0, 33)
    with pytest.raises(CenoteError):
        r.set_tuning(SORT_ALL, 0, 8, 321)
    with pytest.raises(CenoteError):
        r.set_tuning(SORT_ALL, 0, 8, 0, 2)
    with pytest.raises(CenoteError):
        r.set_tuning(SORT_ALL, 0, 8, 0, 0, 2)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["chart", "textured"])
def test_traversal_block_size_and_stack_depth_are_bitwise_invisible(ctx, name):
    """The traversal's launch variants (128 or 256 threads per block, 16 or
    32 stack entries per lane) walk the same tree to the same hits: films
    are bitwise equal whichever the tuning picks, per-lane and queued
    triangle tests alike."""
    from cenote_b200 import Film, Renderer, Scene, scenes

    spec = scenes.chart(96, 64, env_size=(256, 128)) if name == "chart" else scenes.textured(80, 45, 4, 5, size=32)
    s = Scene(ctx, spec)
    films = []
    for per_lane in (0, 1):
        for block, stack in ((128, 32), (128, 16), (256, 32), (256, 16)):
            r = Renderer(ctx, spec.max_bounces)
            r.set_tuning(1, 0, 0, 0, 0, per_lane, block, stack)
            t = r.tuning()
            assert (t["block_size"], t["stack_depth"]) == (block, stack)
            f = Film(ctx, spec.width, spec.height)
            r.accumulate(s, f, 4)
            films.append(f.sums())
    for other in films[1:]:
        assert np.array_equal(films[0], other)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["chart", "textured"])
def test_sort_by_location_is_bitwise_invisible(ctx, name):
    """The material sort's key (instance, or the Morton cell of the hit's
    location) only reorders how a bounce is shaded and the next one is
    walked: films are bitwise equal, per-lane and queued triangle tests
    alike, sorting every bounce or from the first bounce on."""
    from cenote_b200 import Film, Renderer, Scene, scenes

    spec = scenes.chart(96, 64, env_size=(256, 128)) if name == "chart" else scenes.textured(80, 45, 4, 5, size=32)
    s = Scene(ctx, spec)
    films = []
    for sort in (1, 2):
        for per_lane in (0, 1):
            for location in (0, 1):
                r = Renderer(ctx, spec.max_bounces)
                r.set_tuning(sort, 0, 0, 0, 0, per_lane, 0, 0, location)
                assert r.tuning()["sort_by_location"] == location
                f = Film(ctx, spec.width, spec.height)
                r.accumulate(s, f, 4)
                films.append(f.sums())
    for other in films[1:]:
        assert np.array_equal(films[0], other)
