"""The wavefront engine on the device: the reference's estimator tests
(crates/cenote/src/render/tests.rs, crates/cenote/src/wavefront.rs tests)
re-run through the C ABI, plus image parity against the CPU oracle."""
import math

import numpy as np
import pytest

import oracle
from cenote_b200 import LIGHT_SAMPLING_BSDF, LIGHT_SAMPLING_MIS, LIGHT_SAMPLING_NEE, Film, Renderer, Scene, scenes

pytestmark = pytest.mark.gpu
WHITE = (1.0, 1.0, 1.0)


def bsdf_only_sum(ctx, spec, size, samples, max_bounces=8):
    r = Renderer(ctx, max_bounces, LIGHT_SAMPLING_BSDF)
    s = Scene(ctx, spec)
    return sum(r.render(s, size, size, k) for k in range(samples))


def accumulate_mean(ctx, spec, size, samples, max_bounces=8, light_sampling=LIGHT_SAMPLING_MIS):
    r = Renderer(ctx, max_bounces, light_sampling)
    s = Scene(ctx, spec)
    f = Film(ctx, size, size)
    r.accumulate(s, f, samples)
    return f.sums()


def test_lambert_furnace_is_exact_per_sample(ctx):  # render/tests.rs:185-214
    spec = scenes.furnace(scenes.matte(WHITE, 0.0))
    total = bsdf_only_sum(ctx, spec, 32, 4)
    assert np.all(np.abs(total[..., :3] / 4.0 - 0.5) < 1e-3)


def test_rough_furnace_mean(ctx):  # render/tests.rs:205-213
    s = accumulate_mean(ctx, scenes.furnace(scenes.matte(WHITE, 1.0)), 32, 64)
    mean = s[..., 0].sum() / (32 * 32 * 64)
    assert abs(mean - 0.5) < 0.005


def test_ray_offsets_hold_at_scene_scale(ctx):  # render/tests.rs:226-249
    spec = scenes.furnace(scenes.matte((0.5, 0.5, 0.5), 0.0), center=(1e4, 0.0, 1e4), scl=1e3)
    total = bsdf_only_sum(ctx, spec, 32, 4)
    assert np.all(np.abs(total[..., :3] / 4.0 - 0.25) < 1e-3)


def test_the_furnace_closes_through_a_thin_lens(ctx):  # render/tests.rs:260-290
    spec = scenes.furnace(scenes.matte((0.5, 0.5, 0.5), 0.0), aperture=0.05, focus=1.5)
    total = bsdf_only_sum(ctx, spec, 32, 4)
    assert np.all(np.abs(total[..., :3] / 4.0 - 0.25) < 1e-3)


FURNACE_MATRIX = {  # render/tests.rs:422-488
    "metal r=0.05": lambda: scenes.metal(WHITE, 0.05),
    "metal r=0.5": lambda: scenes.metal(WHITE, 0.5),
    "metal r=1.0": lambda: scenes.metal(WHITE, 1.0),
    "glossy-diffuse r=0.05": lambda: scenes.glossy(WHITE, 0.0, 0.05),
    "glossy-diffuse r=0.5": lambda: scenes.glossy(WHITE, 0.0, 0.5),
    "glossy-diffuse r=1.0, rough base": lambda: scenes.glossy(WHITE, 1.0, 1.0),
    "half metal": lambda: scenes.material(base_color=WHITE, specular_weight=1.0, specular_roughness=0.5,
                                          metalness=0.5),
    "glossy ior=2.5": lambda: scenes.material(base_color=WHITE, specular_weight=1.0, specular_roughness=0.5,
                                              specular_ior=2.5),
    "glossy ior=1.1": lambda: scenes.material(base_color=WHITE, specular_weight=1.0, specular_roughness=0.8,
                                              specular_ior=1.1),
    "coat over diffuse": lambda: scenes.material(base_color=WHITE, specular_weight=1.0, specular_roughness=0.5,
                                                 coat_weight=1.0, coat_roughness=0.3),
    "coat over metal": lambda: scenes.material(base_color=WHITE, metalness=1.0, specular_weight=1.0,
                                               specular_roughness=0.5, coat_weight=1.0, coat_roughness=0.1),
    "fuzz over diffuse": lambda: scenes.material(base_color=WHITE, fuzz_weight=1.0, fuzz_roughness=0.5),
    "the full stack": lambda: scenes.material(base_color=WHITE, base_roughness=0.3, specular_weight=1.0,
                                              specular_roughness=0.4, metalness=0.3, coat_weight=0.7,
                                              coat_roughness=0.2, fuzz_weight=0.5, fuzz_roughness=0.7),
    "glass plane r=0.4": lambda: scenes.glass(0.4, 1.5),
    "thin glass r=0.4": lambda: scenes.material(transmission_weight=1.0, specular_weight=1.0,
                                                specular_roughness=0.4, thin_walled=1),
    "half opacity": lambda: scenes.material(base_color=WHITE, opacity=0.5),
}


# The OpenPBR model's own energy balance where it misses 1e-3: its
# Kulla-Conty compensation tables (tables.rs) are interpolated from 32² and
# 16³ grids, which leaves a bias at low roughness and high IOR, and the
# thin-walled lobe's split gains energy. Measured on a B200 at 256², 1,024 spp
# (67 M samples; the standard error is below 1e-4): relative deviation of the
# furnace mean from the sky's 0.5. test_furnace_is_the_oracles_model shows
# these are the model's, not FP32's: the device and the FP64-closure oracle
# give the same mean on the same samples.
OPENPBR_MODEL_BIAS = {
    "glossy-diffuse r=0.05": -1.2e-3,
    "glossy ior=2.5": -1.2e-3,
    "coat over diffuse": -1.2e-3,
    "the full stack": -1.0e-3,
    "thin glass r=0.4": +2.8e-3,
}


@pytest.mark.parametrize("label", list(FURNACE_MATRIX))
def test_openpbr_furnace_matrix(ctx, label):
    """White furnace through every lobe (render/tests.rs:422-488) at 256²,
    1,024 spp: the mean closes to 1e-3 of the sky, or, for the lobes whose
    model does not, to 5e-4 of the model's measured balance."""
    s = accumulate_mean(ctx, scenes.furnace(FURNACE_MATRIX[label](), size=256), 256, 1024)
    dev = s[..., :3].astype(np.float64).sum(axis=(0, 1)) / (256 * 256 * 1024) / 0.5 - 1.0
    bias = OPENPBR_MODEL_BIAS.get(label, 0.0)
    assert np.all(np.abs(dev - bias) < (5e-4 if bias else 1e-3)), (label, dev)


@pytest.mark.parametrize("label", list(OPENPBR_MODEL_BIAS) + ["metal r=0.5", "glass plane r=0.4"])
def test_furnace_is_the_oracles_model(ctx, label):
    """The furnace on the device and in the oracle over the same samples
    (64², 256 spp): the means agree to 1e-5, so the device's furnace balance
    is the restated model's, to FP32 rounding."""
    spec = scenes.furnace(FURNACE_MATRIX[label](), size=64)
    s = accumulate_mean(ctx, spec, 64, 256)
    ref = oracle.OracleScene(spec).render_sum(64, 64, 0, 256, 8)
    gpu = s[..., :3].astype(np.float64).sum()
    cpu = ref[..., :3].astype(np.float64).sum()
    assert abs(gpu / cpu - 1.0) < 1e-5, (label, gpu / cpu - 1.0)


def glass_sphere_spec():
    obj = scenes.Object(scenes.icosphere(3), scenes.rows(scenes.translate(0, 2, 0)), scenes.glass(0.2, 1.5))
    return scenes.SceneSpec("glass", [obj], scenes.Camera((0, 2, 4), (0, 2, 0)),
                            scenes.Environment.constant((0.5, 0.5, 0.5)), 32, 32, 128, 16)


def test_the_glass_furnace_closes(ctx):  # render/tests.rs:498-532
    """A glass sphere under a grey sky (16 bounces) at 256², 1,024 spp. Paths
    that still bounce inside after 16 vertices are cut, so the reference's
    bound is 1.5 %; measured: −1.1 %, the same as the oracle on the same
    samples."""
    spec = glass_sphere_spec()
    s = accumulate_mean(ctx, spec, 256, 1024, max_bounces=16)
    mean = s[..., :3].astype(np.float64).sum(axis=(0, 1)) / (256 * 256 * 1024)
    assert np.all(np.abs(mean / 0.5 - 1.0 + 0.011) < 1e-3), mean
    small = accumulate_mean(ctx, spec, 32, 128, max_bounces=16)[..., :3].astype(np.float64).sum()
    ref = oracle.OracleScene(spec).render_sum(32, 32, 0, 128, 16)[..., :3].astype(np.float64).sum()
    assert abs(small / ref - 1.0) < 1e-3


def delta_scene(light):
    obj = scenes.Object(scenes.ground_plane(5.0), scenes.rows(np.eye(4)), scenes.matte(WHITE, 0.0))
    cam = scenes.Camera((0.0, 1.0, 0.0), (0.0, 0.0, -1.0))
    return scenes.SceneSpec("delta", [obj], cam, scenes.Environment.constant((0, 0, 0)), 16, 16, 1, 8, [light])


def test_a_distant_light_is_analytically_exact(ctx):  # render/tests.rs:352-380
    spec = delta_scene(scenes.DeltaLight(1, (0.0, -1.0, 0.0), (math.pi,) * 3))
    img = Renderer(ctx).render(Scene(ctx, spec), 16, 16)
    assert np.all(np.abs(img[..., :3] - 1.0) < 2e-3)


def test_a_point_light_is_analytically_exact(ctx):  # render/tests.rs:384-420
    spec = delta_scene(scenes.DeltaLight(2, (0.0, 1000.0, 0.0), (math.pi * 1e6,) * 3))
    img = Renderer(ctx).render(Scene(ctx, spec), 16, 16)
    assert np.all(np.abs(img[..., :3] - 1.0) < 5e-3)


def test_rendering_is_bitwise_deterministic(ctx):  # render/tests.rs:1306-1316
    spec = scenes.chart(width=128, height=72, env_size=(256, 128))
    s, r = Scene(ctx, spec), Renderer(ctx, 12)
    assert np.array_equal(r.render(s, 128, 72), r.render(s, 128, 72))


def test_accumulation_adds_distinct_samples(ctx):  # render/tests.rs:1323-1370
    spec = scenes.cornell()
    s, r = Scene(ctx, spec), Renderer(ctx, 8)
    f = Film(ctx, 64, 64)
    for _ in range(3):
        r.accumulate(s, f)
    assert f.samples == 3
    s0, s1, s2 = (r.render(s, 64, 64, k) for k in range(3))
    assert not np.array_equal(s0, s1)
    assert np.array_equal(f.sums(), (s0 + s1) + s2)
    assert np.array_equal(f.averages(), ((s0 + s1) + s2) / np.float32(3.0))


def test_samples_per_wave_is_bitwise_invisible(ctx):
    """Several samples of every pixel in one wave (this engine's occupancy
    lever) must not change a single bit of the film."""
    spec = scenes.chart(width=96, height=64, env_size=(256, 128))
    s = Scene(ctx, spec)
    films = []
    for spw in (1, 3, 16):
        r = Renderer(ctx, 12, samples_per_wave=spw)
        f = Film(ctx, 96, 64)
        r.accumulate(s, f, 16)
        films.append(f.sums())
    assert np.array_equal(films[0], films[1]) and np.array_equal(films[0], films[2])


def test_layerless_shading_variant_is_bitwise_invisible(ctx):
    """A scene without coat, fuzz, transmission or thin walls shades with
    those lobes compiled out. Adding one coated triangle where no ray can
    reach it (inside an opaque icosphere) switches the scene to the full
    shading kernel and must leave the film unchanged but for the compiler's
    fused multiply-adds (measured: 20 of 6,144 pixels, 1.6e-7 relative)."""
    import dataclasses

    spec = scenes.chart(width=96, height=64, env_size=(256, 128))
    sphere = next(o for o in spec.objects if o.mesh.triangle_count == 1280)
    centre = np.asarray(sphere.transform, np.float64).reshape(3, 4)[:, 3]
    tri = scenes.Mesh(np.array([[0, 0, 0], [1e-3, 0, 0], [0, 1e-3, 0]], np.float32),
                      np.array([[0, 0, 1]] * 3, np.float32), np.zeros((3, 2), np.float32),
                      np.array([[0, 1, 2]], np.uint32))
    coated = scenes.matte((0.5, 0.5, 0.5))
    coated["coat_weight"] = 1.0
    xf = np.eye(4)
    xf[:3, 3] = centre
    hidden = dataclasses.replace(spec, objects=list(spec.objects) + [scenes.Object(tri, scenes.rows(xf), coated)])
    films = []
    for sp in (spec, hidden):
        f = Film(ctx, 96, 64)
        Renderer(ctx, 12).accumulate(Scene(ctx, sp), f, 8)
        films.append(f.sums())
    a, b = films
    assert np.all(np.abs(a - b) <= 1e-6 * np.abs(a))
    assert (np.abs(a - b).max(-1) > 0).mean() < 0.01


def test_pool_ranges_are_bitwise_equal(ctx):  # wavefront.rs:918-942
    spec = scenes.cornell()
    s = Scene(ctx, spec)
    full = Renderer(ctx, 8).render(s, 100, 60)
    ranged = Renderer(ctx, 8, capacity=1000).render(s, 100, 60)
    assert np.array_equal(full, ranged)


def test_reset_restarts_the_accumulation(ctx):  # render/tests.rs:1376-1400
    spec = scenes.cornell()
    s, r = Scene(ctx, spec), Renderer(ctx, 8)
    f = Film(ctx, 64, 64)
    r.accumulate(s, f, 2)
    f.reset()
    r.accumulate(s, f)
    assert f.samples == 1
    assert np.array_equal(f.sums(), r.render(s, 64, 64, 0))


def test_ragged_dimensions_cover_every_pixel(ctx):  # render/tests.rs:163-180
    spec = scenes.chart(env_size=(64, 32))
    img = Renderer(ctx, 12).render(Scene(ctx, spec), 33, 17)
    assert np.all(img[..., 3] == 1.0)
    assert np.all(np.isfinite(img)) and np.all(img[..., :3] >= 0)


def test_non_finite_contributions_are_dropped(ctx):  # render/tests.rs:1465-1520
    spec = scenes.cornell()
    spec.objects[-1].material["emission"] = (np.nan, 1.0, 1.0)
    s, r = Scene(ctx, spec), Renderer(ctx, 8)
    raw = r.render(s, 64, 64)
    f = Film(ctx, 64, 64)
    r.accumulate(s, f)
    sums = f.sums()
    bad = ~np.isfinite(raw).all(axis=-1)
    assert bad.any()
    assert np.all(sums[bad] == 0.0)
    assert np.array_equal(sums[~bad], raw[~bad])


def strategies_mean(ctx, spec, mode, size=32, samples=256):
    s = accumulate_mean(ctx, spec, size, samples, 8, mode)
    return s[..., :3].astype(np.float64).sum() / (size * size * samples)


def mis_scene_spec():  # wavefront.rs:1246-1300
    objs = [
        scenes.Object(scenes.icosphere(2), scenes.rows(scenes.translate(0, 1, 0)),
                      scenes.material(base_color=(0.6,) * 3, base_roughness=0.4, specular_weight=1.0,
                                      specular_roughness=0.3, metalness=0.5)),
        scenes.Object(scenes.ground_plane(4.0), scenes.rows(np.eye(4)), scenes.glossy((0.7,) * 3, 0.0, 0.2)),
        scenes.Object(scenes.icosphere(2), scenes.rows(scenes.translate(1.6, 0.6, 1.2) @ scenes.scale(0.6)),
                      scenes.glass(0.4, 1.5)),
        scenes.Object(scenes.icosphere(2), scenes.rows(scenes.translate(0, 3, 0) @ scenes.scale(0.7)),
                      scenes.emitter((4.0, 4.0, 4.0))),
    ]
    cam = scenes.Camera((0.0, 2.5, 6.0), (0.0, 1.0, 0.0), vfov_degrees=45.0)
    return scenes.SceneSpec("mis", objs, cam, scenes.Environment.constant((0, 0, 0)), 32, 32, 256, 8)


def env_mis_spec():  # wavefront.rs:1304-1340
    spec = mis_scene_spec()
    spec.objects = spec.objects[:2]
    w, h = 8, 4
    tex = np.full((h, w, 4), 0.2, np.float32)
    tex[1, :, :3] = 0.0
    tex[1, 4, :3] = 8.0
    tex[..., 3] = 1.0
    spec.environment = scenes.Environment(w, h, tex)
    return spec


@pytest.mark.parametrize("make", [mis_scene_spec, env_mis_spec], ids=["area-light", "environment"])
def test_light_sampling_strategies_agree(ctx, make):  # wavefront.rs:1510-1558
    spec = make()
    mis = strategies_mean(ctx, spec, LIGHT_SAMPLING_MIS)
    assert mis > 0.01
    for mode in (LIGHT_SAMPLING_BSDF, LIGHT_SAMPLING_NEE):
        v = strategies_mean(ctx, spec, mode)
        assert abs(v - mis) / mis < 0.03, (mode, v, mis)


@pytest.mark.parametrize("name", ["cornell", "chart"])
def test_image_parity_with_oracle(ctx, name):
    """The same samples through the kernels and through the CPU restatement.
    Paths follow identical sample sequences; they part only where FP32
    rounding differs (transcendentals, FMA contraction, the hardware
    bilinear filter), so the images agree far inside the noise."""
    spec = scenes.cornell(64, 64) if name == "cornell" else scenes.chart(96, 54, env_size=(256, 128))
    w, h, spp = spec.width, spec.height, 64
    r = Renderer(ctx, spec.max_bounces)
    f = Film(ctx, w, h)
    r.accumulate(Scene(ctx, spec), f, spp)
    gpu = f.averages()[..., :3].astype(np.float64)
    ref = oracle.OracleScene(spec).render_sum(w, h, 0, spp, spec.max_bounces)[..., :3].astype(np.float64) / spp
    rel_mse = np.mean((gpu - ref) ** 2 / (ref ** 2 + 1e-2))
    assert rel_mse < 1e-3, rel_mse
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 5e-3


def test_ray_counts_are_reported(ctx):
    spec = scenes.cornell(64, 64)
    r = Renderer(ctx, 8)
    f = Film(ctx, 64, 64)
    r.accumulate(Scene(ctx, spec), f, 4)
    st = r.stats()
    assert st["samples"] == 64 * 64 * 4
    assert st["extension_rays"] >= st["samples"]
    assert st["shadow_rays"] > 0
    assert st["overflow"] == 0
    ref = oracle.OracleScene(spec)
    ref.render_sum(64, 64, 0, 4, 8)
    # Identical sample sequences: the ray counts agree to rounding-induced path splits.
    assert abs(int(st["extension_rays"]) - int(ref.last_ray_counts[0])) / ref.last_ray_counts[0] < 0.01


def test_accumulate_range_matches_the_film_sequence(ctx):
    spec = scenes.cornell(32, 24, 4, 6)
    s = Scene(ctx, spec)
    r = Renderer(ctx, 6)
    a, b, c = Film(ctx, 32, 24), Film(ctx, 32, 24), Film(ctx, 32, 24)
    r.accumulate(s, a, 6)
    r.accumulate_range(s, b, 0, 6)
    assert np.array_equal(a.sums(), b.sums()) and b.samples == 6
    # Samples 6..9 continue the sequence where the film left off.
    r.accumulate(s, a, 4)
    r.accumulate_range(s, c, 0, 6)
    r.accumulate_range(s, c, 6, 4)
    assert np.array_equal(a.sums(), c.sums())
    # A disjoint range is a different, equally valid estimate.
    d = Film(ctx, 32, 24)
    r.accumulate_range(s, d, 1 << 20, 10)
    assert not np.array_equal(a.sums(), d.sums())
    assert abs(d.sums()[..., 0].mean() / a.sums()[..., 0].mean() - 1.0) < 0.2
