"""Scene files in the reference's change-set format (.ron).

The format is crates/cenote/src/scene/changeset.rs (ops upserting named
objects, Remove) read through crates/cenote/src/format.rs; lowering follows
description.rs / lower.rs. The scenes below are written for these tests.
"""
from __future__ import annotations

import math
import struct
import zlib

import numpy as np
import pytest

from cenote_b200 import scenes
from cenote_b200.pbrt import _lower, _openpbr
from cenote_b200.scene_file import Enum, load_scene_file, parse_ron, read_ply, read_png, transform_matrix

BOX = """
// a lamp above a floor, and a tilted panel
(
    version: 1,
    ops: [
        Settings((name: "main", resolution: Some((64, 48)), spp: Some(8), max_bounces: Some(5))),
        Camera((name: "main", position: Some((0.0, 2.0, 5.0)), look_at: Some((0.0, 0.5, 0.0)),
                vfov_degrees: Some(35.0))),
        Mesh((name: "plane", source: Some(Inline(
            positions: [(-1.0, 0.0, -1.0), (-1.0, 0.0, 1.0), (1.0, 0.0, 1.0), (1.0, 0.0, -1.0)],
            normals: Some([(0.0, 1.0, 0.0), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0)]),
            uvs: Some([(0.0, 0.0), (0.0, 1.0), (1.0, 1.0), (1.0, 0.0)]),
            triangles: [(0, 1, 2), (0, 2, 3)],
        )))),
        Material((name: "floor", base_color: Some(Constant((0.6, 0.5, 0.4))),
                  specular_roughness: Some(Constant(0.3)))),
        Material((name: "panel", base_color: Some(Constant((0.9, 0.9, 0.9))), base_metalness: Some(Constant(1.0)),
                  specular_roughness: Some(Constant(0.2)), coat_weight: Some(0.5))),
        Material((name: "lamp", base_color: Some(Constant((0.0, 0.0, 0.0))), specular_weight: Some(0.0),
                  emission_color: Some(Constant((1.0, 0.9, 0.7))), emission_luminance: Some(10.0))),
        Instance((name: "floor", mesh: Some("plane"), material: Some("floor"),
                  transform: Some(Trs(scale: (4.0, 1.0, 4.0))))),
        Instance((name: "panel", mesh: Some("plane"), material: Some("panel"),
                  transform: Some(Trs(translate: (0.5, 0.8, -0.5), rotate_degrees: (70.0, 20.0, 0.0),
                                      scale: (0.6, 1.0, 0.6))))),
        Instance((name: "lamp", mesh: Some("plane"), material: Some("lamp"),
                  transform: Some(Trs(translate: (0.0, 3.0, 0.0), rotate_degrees: (180.0, 0.0, 0.0),
                                      scale: (0.4, 1.0, 0.4))))),
        Light((name: "sun", light: Some(Distant(direction: (0.0, -1.0, -0.2), irradiance: (1.0, 1.0, 1.0))))),
        Instance((name: "gone", mesh: Some("plane"), material: Some("floor"))),
        Remove(Instance, "gone"),
        Material((name: "floor", coat_weight: Some(0.25))),
    ],
)
"""


def test_ron_values():
    v = parse_ron('(a: 1, b: -2.5e1, c: "x\\"y", d: [1, 2, (3, 4)], e: Some(true), f: None, '
                  'g: Foo((h: 1)), i: Bar(1.0, 2), j: Unit, /* note */ k: Some(Trs(scale: (1.0, 2.0, 3.0))))')
    assert v["a"] == 1 and v["b"] == -25.0 and v["c"] == 'x"y' and v["d"] == [1, 2, (3, 4)]
    assert v["e"] is True and v["f"] is None
    assert isinstance(v["g"], Enum) and v["g"].name == "Foo" and v["g"].payload == [{"h": 1}]
    assert v["i"].payload == [1.0, 2] and v["j"].name == "Unit" and v["j"].payload is None
    assert v["k"].name == "Trs" and v["k"].payload == {"scale": (1.0, 2.0, 3.0)}
    with pytest.raises(ValueError):
        parse_ron("(a: 1")


def test_trs_order():
    # translate . Rz . Ry . Rx . scale (description.rs:134-159)
    t = parse_ron("Trs(translate: (1.0, 2.0, 3.0), rotate_degrees: (90.0, 0.0, 0.0), scale: (2.0, 2.0, 2.0))")
    m = transform_matrix(t)
    p = m @ np.array([0.0, 1.0, 0.0, 1.0])
    assert np.allclose(p[:3], [1.0, 2.0, 5.0])  # +y scaled to 2, rotated 90 about x -> +z
    t2 = parse_ron("Trs(rotate_degrees: (90.0, 90.0, 0.0))")
    v = transform_matrix(t2) @ np.array([0.0, 1.0, 0.0, 0.0])  # Rx then Ry: +y -> +z -> +x
    assert np.allclose(v[:3], [1.0, 0.0, 0.0], atol=1e-9)
    mat = transform_matrix(parse_ron("Matrix(((1.0, 0.0, 0.0, 5.0), (0.0, 1.0, 0.0, 6.0), (0.0, 0.0, 1.0, 7.0)))"))
    assert np.allclose(mat[:3, 3], [5, 6, 7])


def test_load_applies_the_change_set(tmp_path):
    f = tmp_path / "box.ron"
    f.write_text(BOX)
    spec = load_scene_file(f)
    assert (spec.width, spec.height, spec.spp, spec.max_bounces) == (64, 48, 8, 5)
    assert len(spec.objects) == 3  # "gone" was removed
    cam = spec.camera
    assert cam.vfov_degrees == 35.0 and np.allclose(cam.position, (0, 2, 5))
    assert cam.focus_distance == pytest.approx(math.dist((0, 2, 5), (0, 0.5, 0)))
    by_material = {o.material.tobytes(): o for o in spec.objects}
    floor = _lower(_openpbr(base_color=(0.6, 0.5, 0.4), specular_roughness=0.3, coat_weight=0.25))
    assert floor.tobytes() in by_material  # the later patch added coat_weight, kept the rest
    lamp = [o for o in spec.objects if o.material["emission"][0] > 0][0]
    assert np.allclose(lamp.material["emission"], scenes.acescg((1.0, 0.9, 0.7)) * 10.0, rtol=1e-6)
    assert len(spec.delta_lights) == 1 and spec.delta_lights[0].kind == 1
    d = np.array([0.0, -1.0, -0.2])
    assert np.allclose(spec.delta_lights[0].anchor, d / np.linalg.norm(d))


def png_bytes(img, filt):
    """A PNG with every row under filter type `filt` (written here for the test)."""
    h, w, ch = img.shape
    a = img.astype(np.int32)
    rows = []
    for y in range(h):
        line = a[y].reshape(-1)
        prev = a[y - 1].reshape(-1) if y else np.zeros_like(line)
        left = np.concatenate([np.zeros(ch, np.int32), line[:-ch]])
        ul = np.concatenate([np.zeros(ch, np.int32), prev[:-ch]])
        if filt == 0:
            p = 0
        elif filt == 1:
            p = left
        elif filt == 2:
            p = prev
        elif filt == 3:
            p = (left + prev) // 2
        else:
            pa, pb, pc = np.abs(prev - ul), np.abs(left - ul), np.abs(left + prev - 2 * ul)
            p = np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, prev, ul))
        rows.append(bytes([filt]) + ((line - p) & 0xFF).astype(np.uint8).tobytes())
    ctype = {1: 0, 2: 4, 3: 2, 4: 6}[ch]

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(b"".join(rows))) + chunk(b"IEND", b""))


@pytest.mark.parametrize("filt", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("ch", [1, 3, 4])
def test_png_reader(tmp_path, filt, ch):
    img = np.random.default_rng(filt * 7 + ch).integers(0, 256, (9, 13, ch), dtype=np.uint8)
    p = tmp_path / "x.png"
    p.write_bytes(png_bytes(img, filt))
    assert np.array_equal(read_png(p), img)


def test_ply_reader(tmp_path):
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    ascii_ply = ("ply\nformat ascii 1.0\nelement vertex 4\nproperty float x\nproperty float y\nproperty float z\n"
                 "property float u\nproperty float v\nelement face 1\nproperty list uchar int vertex_indices\n"
                 "end_header\n" + "".join(f"{a} {b} {c} {a} {b}\n" for a, b, c in pos) + "4 0 1 2 3\n")
    (tmp_path / "a.ply").write_text(ascii_ply)
    p, n, uv, idx = read_ply(tmp_path / "a.ply")
    assert np.allclose(p, pos) and n is None and np.allclose(uv, pos[:, :2])
    assert idx.tolist() == [[0, 1, 2], [0, 2, 3]]
    header = (b"ply\nformat binary_little_endian 1.0\nelement vertex 4\nproperty float x\nproperty float y\n"
              b"property float z\nproperty float nx\nproperty float ny\nproperty float nz\nelement face 2\n"
              b"property list uchar uint vertex_indices\nend_header\n")
    body = b"".join(struct.pack("<6f", *v, 0, 0, 1) for v in pos)
    body += struct.pack("<B3I", 3, 0, 1, 2) + struct.pack("<B3I", 3, 0, 2, 3)
    (tmp_path / "b.ply").write_bytes(header + body)
    p, n, uv, idx = read_ply(tmp_path / "b.ply")
    assert np.allclose(p, pos) and np.allclose(n, [0, 0, 1]) and uv is None and idx.tolist() == [[0, 1, 2], [0, 2, 3]]


def test_textured_material_and_ply_mesh(tmp_path):
    img = np.random.default_rng(1).integers(0, 256, (8, 8, 3), dtype=np.uint8)
    (tmp_path / "tex.png").write_bytes(png_bytes(img, 4))
    (tmp_path / "tri.ply").write_text("ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\n"
                                      "property float z\nelement face 1\nproperty list uchar int vertex_indices\n"
                                      "end_header\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n")
    (tmp_path / "t.ron").write_text("""(version: 1, ops: [
        Mesh((name: "tri", source: Some(Ply(path: "tri.ply")))),
        Material((name: "m", base_color: Some(Texture((path: "tex.png"))),
                  specular_roughness: Some(Texture((path: "tex.png"))))),
        Instance((name: "i", mesh: Some("tri"), material: Some("m"))),
    ])""")
    spec = load_scene_file(tmp_path / "t.ron", 16, 16)
    assert len(spec.textures) == 2  # colour (BC7, sRGB view) and data (BC4 on red) of one image
    fmts = sorted(t.format for t in spec.textures)
    assert fmts == [scenes.TEX_BC4_UNORM, scenes.TEX_BC7_SRGB]
    m = spec.objects[0].material
    assert m["base_color_texture"] != m["specular_roughness_texture"]
    assert np.allclose(spec.objects[0].mesh.normals, [0, 0, 1])


def test_float_textures_are_prepared_like_the_reference(tmp_path):
    """An EXR texture (texture.rs:283-405): as a colour, BC6H unsigned; as
    data, quantised to 8 bits and BC4 on red; the colour decodes to the
    source within BC6H's precision."""
    from cenote_b200.exr import write_exr
    import oracle

    rng = np.random.default_rng(3)
    img = (0.5 + rng.random((8, 8, 1)) * np.array([1.0, 0.9, 0.8])).astype(np.float32)
    write_exr(tmp_path / "hdr.exr", {"R": img[..., 0], "G": img[..., 1], "B": img[..., 2]})
    (tmp_path / "tri.ply").write_text("ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\n"
                                      "property float z\nelement face 1\nproperty list uchar int vertex_indices\n"
                                      "end_header\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n")
    (tmp_path / "t.ron").write_text("""(version: 1, ops: [
        Mesh((name: "tri", source: Some(Ply(path: "tri.ply")))),
        Material((name: "m", base_color: Some(Texture((path: "hdr.exr"))),
                  specular_roughness: Some(Texture((path: "hdr.exr"))))),
        Instance((name: "i", mesh: Some("tri"), material: Some("m"))),
    ])""")
    spec = load_scene_file(tmp_path / "t.ron", 16, 16)
    fmts = sorted(t.format for t in spec.textures)
    assert fmts == [scenes.TEX_BC4_UNORM, scenes.TEX_BC6H_UF16]
    colour = next(t for t in spec.textures if t.format == scenes.TEX_BC6H_UF16)
    back = oracle.texture_decode(colour)[..., :3]
    assert np.abs(back / img - 1.0).max() < 0.08  # white noise over 1.6 stops in 16 palette steps


@pytest.mark.gpu
def test_gpu_scene_file_renders_like_the_oracle(ctx, tmp_path):
    """A scene loaded from the change-set file, rendered by the CUDA path and
    by the oracle over the same samples (the file's 64x48, 5 bounces, at 256
    spp): relMSE under 1e-4 (value floor 0.01) and mean LDR-FLIP under 0.01,
    the reference's image bar (crates/cenote-pbrt/tests/corpus.rs:41). The
    same scene built through the API renders bitwise the same."""
    import oracle
    from cenote_b200 import Film, Renderer, Scene
    from cenote_b200.metrics import flip_ldr_linear, rel_mse

    f = tmp_path / "box.ron"
    f.write_text(BOX)
    spec = load_scene_file(f)
    twin = scenes.SceneSpec("twin", list(spec.objects), spec.camera, spec.environment, spec.width, spec.height,
                            spec.spp, spec.max_bounces, list(spec.delta_lights))
    spp = 256
    out = []
    for s in (spec, twin):
        r = Renderer(ctx, s.max_bounces)
        film = Film(ctx, s.width, s.height)
        r.accumulate(Scene(ctx, s), film, spp)
        out.append(film.averages())
    assert np.array_equal(out[0], out[1])
    gpu = out[0][..., :3]
    ref = oracle.OracleScene(spec).render_sum(spec.width, spec.height, 0, spp, spec.max_bounces)[..., :3] / spp
    assert gpu.mean() > 0.0
    assert rel_mse(gpu, ref, 1e-4) < 1e-4, rel_mse(gpu, ref, 1e-4)
    assert flip_ldr_linear(ref, gpu) < 0.01
