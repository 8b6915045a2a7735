"""The GPU BVH builds (binned SAH, and PLOC over Morton order; both collapsed
on the device).

Closest hits do not depend on the tree (equal distances resolve by the
(instance, primitive) key), so a scene built on the GPU must render bit for
bit what the host-built scene renders, with the same ray counts, and its
prep must report a build time.
"""
from __future__ import annotations

import numpy as np
import pytest

from cenote_b200 import BVH_AUTO, BVH_GPU_PLOC, BVH_GPU_SAH, BVH_HOST_SAH, scenes

pytestmark = pytest.mark.gpu


def render_with(builder, spec, spp, bounces):
    from cenote_b200 import Context, Film, Renderer, Scene

    ctx = Context(0)
    ctx.set_bvh_builder(builder)
    scene = Scene(ctx, spec)
    r = Renderer(ctx, bounces)
    f = Film(ctx, spec.width, spec.height)
    r.accumulate(scene, f, spp)
    st = r.stats()
    assert scene.bvh_builder() == (BVH_HOST_SAH if builder == BVH_AUTO else builder)
    out = f.all_averages(), (st["extension_rays"], st["shadow_rays"], st["overflow"]), scene.prep_times_ms()
    return out


SPECS = {
    "cornell": lambda: scenes.cornell(64, 64, 4, 8),
    "chart": lambda: scenes.chart(96, 54, 4, 8),
    "textured": lambda: scenes.textured(64, 48, 4, 6),
    "one_triangle": lambda: scenes.furnace(scenes.matte((0.5, 0.5, 0.5), 1.0)),
}


GPU_BUILDERS = {"sah": BVH_GPU_SAH, "ploc": BVH_GPU_PLOC}


@pytest.mark.parametrize("builder", sorted(GPU_BUILDERS))
@pytest.mark.parametrize("name", sorted(SPECS))
def test_gpu_built_scene_renders_like_the_host_built_one(name, builder):
    spec = SPECS[name]()
    host, c_host, _ = render_with(BVH_HOST_SAH, spec, spec.spp, spec.max_bounces)
    gpu, c_gpu, prep = render_with(GPU_BUILDERS[builder], spec, spec.spp, spec.max_bounces)
    assert c_gpu == c_host and c_gpu[2] == 0
    for k in host:
        assert np.array_equal(gpu[k], host[k], equal_nan=True), k
    assert prep[0] > 0.0


@pytest.mark.parametrize("builder", sorted(GPU_BUILDERS))
def test_gpu_build_of_a_large_mesh_matches(builder):
    """The large scene's shape at a quarter of its terrain (0.5 M triangles,
    instanced glass, coat and fuzz, 1,024 emitters): many PLOC rounds, SAH
    levels of chunked (multi-CTA) and one-warp tasks, and collapse levels."""
    spec = scenes.large(160, 90, 2, 6, grid=512, instances=120, emitters=1024, texture_size=128, textures=16)
    host, c_host, p_host = render_with(BVH_HOST_SAH, spec, 2, 6)
    gpu, c_gpu, p_gpu = render_with(GPU_BUILDERS[builder], spec, 2, 6)
    assert c_gpu == c_host and c_gpu[2] == 0
    assert np.array_equal(gpu["beauty"], host["beauty"], equal_nan=True)
    print(f"BVH build ms: host {p_host[0]:.1f}, GPU {builder} {p_gpu[0]:.1f}")


def test_auto_builder_keeps_small_scenes_on_the_host():
    """BVH_AUTO (the default) builds on the host below 2^20 triangles."""
    spec = SPECS["chart"]()
    auto, c_auto, _ = render_with(BVH_AUTO, spec, spec.spp, spec.max_bounces)
    host, c_host, _ = render_with(BVH_HOST_SAH, spec, spec.spp, spec.max_bounces)
    assert c_auto == c_host
    for k in host:
        assert np.array_equal(auto[k], host[k], equal_nan=True), k


def test_unknown_builder_is_refused():
    from cenote_b200 import CenoteError, Context

    with pytest.raises(CenoteError):
        Context(0).set_bvh_builder(4)


def test_auto_builder_builds_large_scenes_on_the_gpu():
    """BVH_AUTO (the default) builds a scene of at least 2^20 triangles with
    the GPU binned-SAH builder: the large scene's 3.08 M triangles."""
    from cenote_b200 import Context, Scene

    ctx = Context(0)
    scene = Scene(ctx, scenes.large(64, 36, 1, 2, texture_size=64, textures=8))
    assert scene.bvh_builder() == BVH_GPU_SAH
    assert scene.prep_times_ms()[0] > 0.0
