"""The pbrt corpus against the reference's own renders, and the importer.

The fixtures tests/golden/corpus_*.npz (made by tests/golden/make_corpus.py)
hold two imported corpus scenes and the reference renderer's 64-spp output for
each (crates/cenote-pbrt/tests/corpus.rs:29-41, 84-114). The reference
renders are deterministic, so an implementation that draws the same samples
reproduces their noise too: the CPU oracle and the CUDA path are both held to
the reference's own bar (mean LDR-FLIP <= 0.01, corpus.rs:41) and to a relMSE
bound far below the Monte-Carlo noise between two different 64-spp renders.
"""
from __future__ import annotations

import math
import pathlib

import numpy as np
import pytest

from cenote_b200 import scenes
from cenote_b200.metrics import flip_ldr_linear, flip_map, rel_mse, to_ldr8
from cenote_b200.pbrt import FLIP_Z, import_pbrt_text

GOLDEN = pathlib.Path(__file__).parent / "golden"
CORPUS = ["cornell_box", "veach_mis"]
MAX_MEAN_FLIP = 0.01   # corpus.rs:41
MAX_REL_MSE = 1e-4     # a second, independent 64-spp render scores 4e-3 (cornell) and 0.4 (veach)


def load(name):
    spec, extra = scenes.load_spec(GOLDEN / f"corpus_{name}.npz")
    return spec, extra["golden"]


# ---- metric -------------------------------------------------------------------


def test_flip_identical_is_zero():
    rng = np.random.default_rng(1)
    img = rng.random((40, 56, 3))
    assert flip_ldr_linear(img, img) == 0.0


def test_flip_grows_with_error_and_stays_in_unit_range():
    rng = np.random.default_rng(2)
    img = rng.random((48, 64, 3)) * 0.8
    prev = 0.0
    for sigma in (0.01, 0.05, 0.2):
        m = flip_map(to_ldr8(img), to_ldr8(img + rng.normal(0, sigma, img.shape)))
        assert 0.0 <= m.min() and m.max() <= 1.0
        assert m.mean() > prev
        prev = m.mean()
    black, white = np.zeros((32, 32, 3)), np.ones((32, 32, 3))
    assert flip_ldr_linear(black, white) > 0.5


def test_ldr8_quantisation_clamps_and_rounds():
    v = to_ldr8(np.array([-1.0, 0.0, 0.5 / 255, 0.49, 1.0, 7.0]))
    assert np.allclose(v * 255, [0, 0, 1, 125, 255, 255])


def test_rel_mse():
    a = np.full((4, 4, 3), 0.5)
    assert rel_mse(a, a) == 0.0
    assert rel_mse(a * 1.1, a) == pytest.approx(0.05 ** 2 / (0.25 + 1e-2))


# ---- the oracle reproduces the reference's pixels ---------------------------------


@pytest.mark.parametrize("name", CORPUS)
def test_oracle_reproduces_reference_corpus_render(name):
    import oracle

    spec, golden = load(name)
    img = oracle.OracleScene(spec).render_sum(spec.width, spec.height, 0, spec.spp, spec.max_bounces)[..., :3]
    img = img / spec.spp
    assert flip_ldr_linear(golden, img) <= MAX_MEAN_FLIP
    assert rel_mse(img, golden) <= MAX_REL_MSE


# ---- importer ------------------------------------------------------------------


SCENE = """
Integrator "volpath" "integer maxdepth" [ 7 ]
Sampler "sobol" "integer pixelsamples" [ 32 ]
Film "rgb" "integer xresolution" [ 200 ] "integer yresolution" [ 100 ]
LookAt 0 1 5  0 1 0  0 1 0
Camera "perspective" "float fov" [ 30 ]
WorldBegin
  MakeNamedMaterial "red" "string type" [ "diffuse" ] "rgb reflectance" [ 0.5 0.1 0.1 ]
  NamedMaterial "red"
  Shape "trianglemesh" "integer indices" [ 0 1 2 ] "point3 P" [ 0 0 0  1 0 0  0 1 0 ]
  AttributeBegin
    ReverseOrientation
    Shape "trianglemesh" "integer indices" [ 0 1 2 ] "point3 P" [ 0 0 0  1 0 0  0 1 0 ]
      "normal N" [ 0 0 1  0 0 1  0 0 1 ]
  AttributeEnd
  AttributeBegin
    AreaLightSource "diffuse" "rgb L" [ 4 3 2 ] "float scale" [ 2 ]
    Translate 0 2 0
    Shape "sphere" "float radius" [ 0.25 ]
  AttributeEnd
  Material "conductor" "rgb eta" [ 0.2 0.9 1.1 ] "rgb k" [ 3.9 2.4 2.2 ] "float roughness" [ 0.0625 ]
  Shape "trianglemesh" "integer indices" [ 0 1 2 ] "point3 P" [ 0 0 0  1 0 0  0 1 0 ]
  Material "dielectric" "float eta" [ 1.33 ] "float roughness" [ 0.04 ] "bool remaproughness" [ false ]
  Shape "trianglemesh" "integer indices" [ 0 1 2 ] "point3 P" [ 0 0 0  1 0 0  0 1 0 ]
  Shape "bilinearmesh" "point3 P" [ 0 0 0  1 0 0  0 1 0  1 1 0 ]
  MakeNamedMedium "fog" "string type" [ "homogeneous" ]
WorldEnd
"""


def test_import_settings_and_camera():
    spec = import_pbrt_text(SCENE)
    assert (spec.width, spec.height, spec.spp, spec.max_bounces) == (200, 100, 32, 7)
    # fov names the shorter axis, here the vertical one; camera flipped into
    # the renderer's right-handed frame by diag(1, 1, -1).
    assert spec.camera.vfov_degrees == pytest.approx(30.0)
    assert np.allclose(spec.camera.position, (0, 1, -5))
    assert np.allclose(np.subtract(spec.camera.look_at, spec.camera.position), (0, 0, 1))
    tall = import_pbrt_text(SCENE.replace("[ 200 ]", "[ 50 ]"))
    expect = 2 * math.degrees(math.atan(math.tan(math.radians(15)) * 100 / 50))
    assert tall.camera.vfov_degrees == pytest.approx(expect)


def test_import_transforms_winding_and_normals():
    spec = import_pbrt_text(SCENE)
    a, b = spec.objects[0], spec.objects[1]
    assert np.allclose(np.asarray(a.transform).reshape(3, 4), FLIP_Z[:3])
    assert (b.mesh.indices == a.mesh.indices[:, [0, 2, 1]]).all()
    assert np.allclose(b.mesh.normals, [0, 0, -1])
    # Missing normals are derived from the winding.
    assert np.allclose(a.mesh.normals, [0, 0, 1])


def test_import_materials_and_area_light():
    spec = import_pbrt_text(SCENE)
    red, light, metal, water = (spec.objects[i].material for i in (0, 2, 3, 4))
    assert red["specular_weight"] == 0.0 and red["metalness"] == 0.0
    assert np.allclose(red["base_color"], scenes.acescg((0.5, 0.1, 0.1)), atol=1e-6)
    assert np.allclose(light["emission"], scenes.acescg((4, 3, 2)) * 2, rtol=1e-6)
    assert spec.objects[2].mesh.triangle_count == 2 * 32 * 64 - 2 * 64
    assert np.allclose(np.asarray(spec.objects[2].transform).reshape(3, 4)[:, 3], (0, 2, 0))
    assert metal["metalness"] == 1.0
    assert metal["specular_roughness"] == pytest.approx(0.0625 ** 0.25)
    f0 = ((np.array([0.2, 0.9, 1.1]) - 1) ** 2 + np.array([3.9, 2.4, 2.2]) ** 2) / \
         ((np.array([0.2, 0.9, 1.1]) + 1) ** 2 + np.array([3.9, 2.4, 2.2]) ** 2)
    assert np.allclose(metal["base_color"], scenes.acescg(f0), atol=1e-5)
    assert water["transmission_weight"] == 1.0
    assert water["specular_ior"] == pytest.approx(1.33)
    assert water["specular_roughness"] == pytest.approx(0.2)


def test_import_warns_on_unsupported_input():
    spec = import_pbrt_text(SCENE)
    assert len(spec.objects) == 5
    assert any("bilinearmesh" in w for w in spec.warnings)
    assert any("MakeNamedMedium" in w for w in spec.warnings)


def test_import_rejects_a_file_without_world():
    with pytest.raises(ValueError):
        import_pbrt_text('Camera "perspective"\n')


def test_spec_archive_round_trip(tmp_path):
    spec = scenes.cornell(64, 48, 4, 3)
    spec.delta_lights = [scenes.DeltaLight(2, (0.0, 1.5, 0.0), (1.0, 2.0, 3.0))]
    scenes.save_spec(tmp_path / "s.npz", spec, note=np.arange(3))
    back, extra = scenes.load_spec(tmp_path / "s.npz")
    assert (back.width, back.height, back.spp, back.max_bounces) == (64, 48, 4, 3)
    assert back.camera == spec.camera or np.allclose(back.camera.position, spec.camera.position)
    assert len(back.objects) == len(spec.objects)
    for o, p in zip(spec.objects, back.objects):
        assert o.material.tobytes() == p.material.tobytes()
        assert (o.mesh.indices == p.mesh.indices).all() and (o.mesh.positions == p.mesh.positions).all()
    assert back.delta_lights[0].kind == 2 and (extra["note"] == np.arange(3)).all()


# ---- the CUDA path reproduces the reference's pixels ------------------------------


@pytest.mark.gpu
@pytest.mark.parametrize("name", CORPUS)
def test_gpu_reproduces_reference_corpus_render(ctx, name):
    from cenote_b200 import Film, Renderer, Scene

    spec, golden = load(name)
    scene = Scene(ctx, spec)
    renderer = Renderer(ctx, spec.max_bounces)
    film = Film(ctx, spec.width, spec.height)
    renderer.accumulate(scene, film, spec.spp)
    img = film.averages()
    assert np.isfinite(img).all()
    flip = flip_ldr_linear(golden, img[..., :3])
    assert flip <= MAX_MEAN_FLIP, flip
    assert rel_mse(img[..., :3], golden) <= MAX_REL_MSE
