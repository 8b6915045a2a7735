"""Device parity against the CPU oracle, through the C ABI.

Bit-exact: Sobol-Burley values, the alias table, the environment CDF/pdf
tables (built on the GPU in FP64), environment sample indices, closest hits.
Tolerance: BSDF eval/pdf in FP32 against the FP64 oracle (1e-5 relative).
"""
import numpy as np
import pytest

import oracle
from cenote_b200 import Scene, scenes

pytestmark = pytest.mark.gpu

KEYS = [(0, 0), (7, 0), (123456, 3), (1, 1), (65535, 8), (921599, 9), (2**31 + 5, 12), (42, 103), (5, 2)]


@pytest.mark.parametrize("pixel,dim", KEYS)
def test_sampler_bit_exact(ctx, pixel, dim):
    pts, vals = ctx.probe_sampler(pixel, dim, 4096)
    ref_pts, ref_vals = oracle.sampler(pixel, dim, 4096)
    assert np.array_equal(pts.view(np.uint32), ref_pts.view(np.uint32))
    assert np.array_equal(vals.view(np.uint32), ref_vals.view(np.uint32))


def test_sampler_matches_committed_vectors(ctx):
    import pathlib
    g = np.load(pathlib.Path(__file__).parent / "golden" / "sampler.npz")
    for k, (pixel, dim) in enumerate(g["keys"]):
        pts, vals = ctx.probe_sampler(int(pixel), int(dim), g["points"].shape[1])
        assert np.array_equal(pts, g["points"][k]) and np.array_equal(vals, g["values"][k])


@pytest.mark.parametrize("pixel,dim", [(0, 0), (7, 0), (123456, 3)])
def test_sampler_is_stratified_on_the_device(ctx, pixel, dim):  # wavefront.rs:1041-1126
    pts, vals = ctx.probe_sampler(pixel, dim, 64)
    for bins in (np.bincount((pts[:, 1] * 8).astype(int) * 8 + (pts[:, 0] * 8).astype(int), minlength=64),
                 np.bincount((pts[:, 0] * 64).astype(int), minlength=64),
                 np.bincount((pts[:, 1] * 64).astype(int), minlength=64),
                 np.bincount((vals * 64).astype(int), minlength=64)):
        assert np.all(bins == 1)


@pytest.fixture(scope="module")
def chart_small(ctx):
    spec = scenes.chart(width=160, height=90, env_size=(512, 256))
    return spec, Scene(ctx, spec), oracle.OracleScene(spec)


@pytest.fixture(scope="module")
def cornell(ctx):
    spec = scenes.cornell()
    return spec, Scene(ctx, spec), oracle.OracleScene(spec)


def test_light_records_bit_exact(cornell, chart_small):
    for spec, dev, ref in (cornell, chart_small):
        a, b = dev.light_records(), ref.lights()
        assert len(a) == len(b) > 0
        assert a.tobytes() == b.tobytes()


def test_light_records_many_emitters(ctx):
    """A few hundred emissive triangles with spread-out powers: the alias
    table's stack order matters here."""
    rng = np.random.default_rng(11)
    objs = []
    for i in range(40):
        m = scenes.icosphere(0) if i % 2 else scenes.box(0.3, 0.2, 0.1)
        e = float(np.exp(rng.normal(0, 2)))
        xf = scenes.rows(scenes.translate(*(rng.random(3) * 10)) @ scenes.scale(0.2 + rng.random()))
        objs.append(scenes.Object(m, xf, scenes.emitter((e, e * 0.5, e * 0.25))))
    objs.append(scenes.Object(scenes.ground_plane(20), scenes.rows(np.eye(4)), scenes.matte((0.5, 0.5, 0.5))))
    spec = scenes.SceneSpec("emitters", objs, scenes.Camera((5, 5, 25), (5, 5, 5)),
                            scenes.Environment.constant((0.1, 0.1, 0.1)), 8, 8, 1, 4,
                            [scenes.DeltaLight(1, (0, -1, 0), (2, 2, 2)), scenes.DeltaLight(2, (3, 8, 3), (5, 5, 5))])
    dev, ref = Scene(ctx, spec), oracle.OracleScene(spec)
    assert dev.light_records().tobytes() == ref.lights().tobytes()
    assert dev.env_tables()[4] == ref.select_prob()


def test_env_tables_bit_exact(chart_small):
    spec, dev, ref = chart_small
    m, c, p, power, sel = dev.env_tables()
    rm, rc, rp = ref.env_tables()
    assert np.array_equal(m.view(np.uint32), rm.view(np.uint32))
    assert np.array_equal(c.view(np.uint32), rc.view(np.uint32))
    assert np.array_equal(p.view(np.uint32), rp.view(np.uint32))
    assert power == ref.env_power()
    assert sel == ref.select_prob()


def test_env_tables_bit_exact_full_size(ctx):
    """The 2048x1024 sky with its 0.5 degree sun: 2M texels of f64 prefix sums."""
    env = scenes.sky_hdri()
    m, c, p, power = oracle.env_tables(env.width, env.height, env.texels)
    spec = scenes.furnace(scenes.matte((0.5, 0.5, 0.5)))
    spec.environment = env
    dm, dc, dp, dpower, _ = Scene(ctx, spec).env_tables()
    assert np.array_equal(dm.view(np.uint32), m.view(np.uint32))
    assert np.array_equal(dc.view(np.uint32), c.view(np.uint32))
    assert np.array_equal(dp.view(np.uint32), p.view(np.uint32))
    assert dpower == power


def test_env_sample_indices_bit_exact(chart_small):
    spec, dev, ref = chart_small
    rng = np.random.default_rng(3)
    u = rng.random((200000, 2)).astype(np.float32)
    d, pdf, rc = dev.probe_env_sample(u)
    rd, rpdf, rrc = ref.env_sample(u)
    assert np.array_equal(rc, rrc)
    assert np.allclose(pdf, rpdf, rtol=1e-5, atol=0)
    assert np.allclose(d, rd, atol=2e-6)
    dirs = rng.normal(size=(100000, 3))
    dirs = (dirs / np.linalg.norm(dirs, axis=1, keepdims=True)).astype(np.float32)
    # CUDA's atan2f/acosf and glibc's may round a direction that sits within
    # an ulp of a texel edge into neighbouring texels: allow 0.1% such flips.
    a, b = dev.probe_env_pdf(dirs), ref.env_pdf(dirs)
    close = np.isclose(a, b, rtol=1e-5, atol=0)
    assert close.mean() > 0.999, close.mean()


def random_rays(spec, n, seed):
    rng = np.random.default_rng(seed)
    pts = np.concatenate([o.mesh.positions for o in spec.objects])
    lo, hi = pts.min(0) - 1, pts.max(0) + 1
    org = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d[: n // 16, 1] = 0.0
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return org, d


@pytest.mark.parametrize("queued", [False, True], ids=["per_lane", "warp_queue"])
@pytest.mark.parametrize("which", ["cornell", "chart_small"])
def test_closest_hits_bit_exact(request, which, queued):
    spec, dev, ref = request.getfixturevalue(which)
    org, d = random_rays(spec, 200000, seed=5)
    hits, t = dev.probe_intersect(org, d, queued=queued)
    rh, rt = ref.intersect(org, d)
    assert np.array_equal(hits, rh)
    assert np.array_equal(t.view(np.uint32), rt.view(np.uint32))
    assert (hits[:, 0] != 0xFFFFFFFF).mean() > 0.2


def test_shadow_queries_match(cornell):
    spec, dev, ref = cornell
    org, d = random_rays(spec, 50000, seed=9)
    rng = np.random.default_rng(2)
    tmax = (rng.random(len(org)) * 3).astype(np.float32)
    lights = ref.lights()
    targets = np.full((len(org), 2), 0xFFFFFFFF, np.uint32)
    pick = rng.random(len(org)) < 0.5
    li = rng.integers(0, len(lights), len(org))
    targets[pick, 0] = lights["instance"][li[pick]]
    targets[pick, 1] = lights["primitive"][li[pick]]
    targets[~pick, 1] = 0
    out = dev.probe_shadow(org, d, tmax, targets)
    ref_out = ref.shadow(org, d, tmax, targets)
    assert np.array_equal(out >= 0, ref_out >= 0)
    # The warp triangle queue answers every query as the per-lane walk does.
    queued = dev.probe_shadow(org, d, tmax, targets, queued=True)
    assert np.array_equal(queued, out)


def test_queued_probes_refuse_fractional_opacity(ctx):
    """The warp triangle queue tests candidates out of visit order, which
    fractional opacity's Bernoulli draws depend on: its shadow probe refuses
    such a scene (the wavefront walks them per lane)."""
    from cenote_b200 import CenoteError, Scene

    spec = scenes.textured(32, 24, 1, 2)  # a leaf quad cut out by an opacity map
    dev = Scene(ctx, spec)
    org = np.zeros((4, 3), np.float32)
    d = np.tile(np.array([[0, 0, 1]], np.float32), (4, 1))
    targets = np.full((4, 2), 0xFFFFFFFF, np.uint32)
    with pytest.raises(CenoteError):
        dev.probe_shadow(org, d, np.ones(4, np.float32), targets, queued=True)
    assert dev.probe_shadow(org, d, np.ones(4, np.float32), targets).shape == (4,)


# ---- BSDF: FP32 device vs FP64 oracle -------------------------------------------------

WHITE = (1.0, 1.0, 1.0)


def materials():
    m = scenes
    out = {
        "lambert": m.matte((0.8, 0.5, 0.3), 0.0),
        "eon rough": m.matte((0.7, 0.7, 0.7), 1.0),
        "glossy r=0.05": m.glossy((0.8, 0.35, 0.2), 0.0, 0.05),
        "glossy r=0.5": m.glossy((0.8, 0.35, 0.2), 0.3, 0.5),
        "metal r=0.2": m.metal((0.9, 0.6, 0.3), 0.2),
        "metal r=1": m.metal(WHITE, 1.0),
        "half metal": m.material(base_color=(0.8, 0.35, 0.2), specular_weight=1.0, specular_roughness=0.4,
                                 metalness=0.5),
        "glass r=0.4": m.glass(0.4, 1.5),
        "glass r=0.1 ior 2.2": m.glass(0.1, 2.2),
        "thin glass": m.material(transmission_weight=1.0, specular_weight=1.0, specular_roughness=0.4,
                                 thin_walled=1, transmission_color=(0.8, 0.9, 1.0)),
        "coat": m.material(base_color=(0.6, 0.2, 0.1), specular_weight=1.0, specular_roughness=0.5, coat_weight=1.0,
                           coat_roughness=0.3),
        "fuzz": m.material(base_color=(0.5, 0.5, 0.5), fuzz_weight=1.0, fuzz_roughness=0.5,
                           fuzz_color=(0.9, 0.7, 0.8)),
        "full stack": m.material(base_color=WHITE, base_roughness=0.3, specular_weight=1.0, specular_roughness=0.4,
                                 metalness=0.3, coat_weight=0.7, coat_roughness=0.2, fuzz_weight=0.5,
                                 fuzz_roughness=0.7),
        "tinted glass depth": m.material(transmission_weight=1.0, specular_weight=1.0, specular_roughness=0.3,
                                         transmission_color=(0.4, 1.0, 1.0), transmission_depth=0.5),
    }
    return out


def directions(n, seed):
    rng = np.random.default_rng(seed)
    wo = rng.normal(size=(n, 3))
    wo[:, 2] = np.abs(wo[:, 2]) + 0.05
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    return wo.astype(np.float32), wi.astype(np.float32)


def rel_err(a, ref, floor):
    return np.abs(a - ref) / np.maximum(np.abs(ref), floor)


def bsdf_errors(ctx, name, exiting):
    """Per pair: the larger of the value's and the pdf's error, relative to
    max(|oracle|, 1e-2). Values under 1e-2 per steradian are compared
    absolutely (an error of 1e-7 there counts as 1e-5), since a relative
    error of a value that rounds toward zero says nothing."""
    mat = materials()[name]
    wo, wi = directions(20000, seed=sum(map(ord, name)))
    f, pdf = ctx.probe_bsdf(mat, wo, wi, exiting)
    rf, rpdf = oracle.bsdf_eval(mat, wo, wi, exiting)
    assert np.all(np.isfinite(f)) and np.all(np.isfinite(pdf))
    ef = rel_err(f.astype(np.float64), rf, 1e-2).max(axis=1)
    ep = rel_err(pdf.astype(np.float64), rpdf, 1e-2)
    return np.maximum(ef, ep), wo, wi


def worst_pairs(e, wo, wi, k=4):
    return [(float(e[i]), round(float(wo[i, 2]), 4), round(float(wi[i, 2]), 4)) for i in np.argsort(-e)[:k]]


@pytest.mark.parametrize("name", list(materials()))
def test_bsdf_eval_pdf_fp32_vs_fp64(ctx, name):
    """Outside a medium, every one of 20,000 (wo, wi) pairs of every
    material: FP32 device eval and pdf within 1e-5 of the FP64 oracle
    (measured worst 4.6e-6, tinted glass; below 2e-6 elsewhere)."""
    e, wo, wi = bsdf_errors(ctx, name, False)
    assert e.max() <= 1e-5, (name, worst_pairs(e, wo, wi))


@pytest.mark.parametrize("name", list(materials()))
def test_bsdf_eval_pdf_inside_a_medium(ctx, name):
    """Leaving a medium the closure is a bare interface with the inverse IOR:
    near the critical angle the Fresnel term F tends to 1 with an unbounded
    slope, so the transmitted 1 - F, h·wi and the total-internal-reflection
    edge all cancel in FP32. At most 1 % of pairs above 1e-5 and none above
    2e-3 (measured on a B200: at most 155 of 20,000 pairs, metal r = 1;
    worst 1.2e-3, the full stack, a transmission at wi.z = -0.05)."""
    e, wo, wi = bsdf_errors(ctx, name, True)
    over = e > 1e-5
    assert over.mean() <= 1e-2, (name, over.mean(), worst_pairs(e, wo, wi))
    assert e.max() <= 2e-3, (name, worst_pairs(e, wo, wi))


@pytest.mark.parametrize("name", list(materials()))
def test_bsdf_sample_fp32_vs_fp64(ctx, name):
    mat = materials()[name]
    wo, _ = directions(20000, seed=7)
    u = np.random.default_rng(8).random((20000, 3)).astype(np.float32)
    wi, pdf, lobe = ctx.probe_bsdf_sample(mat, wo, u)
    rwi, rpdf, rlobe = oracle.bsdf_sample(mat, wo, u)
    same = lobe == rlobe
    assert same.mean() > 0.999
    ok = same & (rpdf > 0)
    assert np.abs(wi[ok] - rwi[ok]).max(axis=1).max() < 2e-4
    close = np.abs(wi[ok] - rwi[ok]).max(axis=1) < 1e-5
    assert close.mean() > 0.99
