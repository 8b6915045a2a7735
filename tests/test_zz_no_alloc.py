"""The allocation-free environment-table entry point (cenote_env_tables_static).

Some callers cannot allocate device memory: a host that gives this library a
fixed arena and accounts for every byte of HBM, code that must not stall the
device on cudaMalloc/cudaFree in the middle of an interactive loop, or a
binding that only holds memory another runtime owns. For them the library
builds the environment's sampling tables into caller-owned device buffers with
its scratch in a static device array. This file checks, through the C ABI,
that the tables are the same bits the allocating build (cenote_scene_create,
read back with cenote_scene_env_tables) produces, over consecutive calls that
reuse the shared scratch, and that inputs past the array's size are refused.

It is collected last so that a failure here leaves the rest of a `-x` run
already done; it passes alone in a fresh process too.
"""
import numpy as np
import pytest

from cenote_b200 import CenoteError, Scene, env_tables_static, scenes

pytestmark = pytest.mark.gpu


def sun_sky(width, height, elevation):
    return scenes.sky_hdri(width, height, sun_elevation_deg=elevation, sun_sigma_deg=2.0, sun_peak=800.0)


def allocating_build(ctx, env):
    spec = scenes.furnace(scenes.matte((0.5, 0.5, 0.5)))
    spec.environment = env
    m, c, p, power, _ = Scene(ctx, spec).env_tables()
    return m, c, p, power


def test_static_build_matches_the_allocating_build(ctx):
    torch = pytest.importorskip("torch")
    envs = [sun_sky(512, 256, 35.0), sun_sky(256, 128, 60.0), sun_sky(512, 256, 35.0)]
    free_after = []
    for k, env in enumerate(envs):
        w, h = env.width, env.height
        want = allocating_build(ctx, env)
        tex = torch.from_numpy(np.ascontiguousarray(env.texels, np.float32)).cuda()
        marginal = torch.full((h + 1,), -1.0, dtype=torch.float32, device="cuda")
        conditional = torch.full((h * (w + 1),), -1.0, dtype=torch.float32, device="cuda")
        pdfs = torch.full((h * w,), -1.0, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        power = env_tables_static(ctx, tex.data_ptr(), w, h, marginal.data_ptr(), conditional.data_ptr(),
                                  pdfs.data_ptr())
        free_after.append(torch.cuda.mem_get_info()[0])
        got = [marginal.cpu().numpy(), conditional.cpu().numpy(), pdfs.cpu().numpy()]
        for a, b in zip(got, want[:3]):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k
        assert power == want[3], k
        if k > 0:  # past the first call's one-time set-up, device memory stays put
            assert free_after[-1] == free_before, (k, free_before, free_after[-1])


def test_static_build_refuses_inputs_past_its_scratch(ctx):
    torch = pytest.importorskip("torch")
    w, h = 1024, 512  # 524,288 texels: twice the static scratch's limit
    tex = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    out = torch.zeros((h * (w + 1),), dtype=torch.float32, device="cuda")
    with pytest.raises(CenoteError) as e:
        env_tables_static(ctx, tex.data_ptr(), w, h, out.data_ptr(), out.data_ptr(), out.data_ptr())
    assert e.value.code == -1
    assert "262144 texels" in str(e.value)
