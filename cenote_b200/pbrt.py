"""A pbrt-v4 importer for the subset the reference's corpus scenes use.

It lowers pbrt's graphics state onto the same scene data the reference's
importer produces (crates/cenote-pbrt/src/map/mod.rs, shape.rs, color.rs), so
a corpus scene renders here as it does there:

* the handedness conjugation diag(1, 1, -1) on every world transform, or the
  identity when the camera transform is itself reflective (map/mod.rs:62-77,
  505-512);
* `fov` names the shorter image axis (map/mod.rs:515-520);
* `rgb L` of a diffuse area light imports verbatim, times `scale`
  (map/mod.rs:707-760, trap 1);
* materials: `diffuse` (reflectance, specular weight 0), `conductor` (F0 from
  eta/k at normal incidence, color.rs:8-15, or `reflectance`; metalness 1),
  `dielectric`/`thindielectric`, `coateddiffuse` (map/mod.rs:1039-1083), with
  pbrt roughness → OpenPBR roughness as r^(1/4) (remapped) or r^(1/2)
  (map/mod.rs:1177-1218, trap 2); unset fields take OpenPBR's defaults
  (crates/cenote/src/scene/description.rs:313-340) and colours enter through
  Rec.709 -> ACEScg (crates/cenote/src/scene/lower.rs:316-373);
* `trianglemesh` verbatim (flipped per ReverseOrientation XOR a mirroring
  transform), `plymesh` read as stored (map/mod.rs:579-598: no flip), `sphere`
  tessellated 32 rings x 64 segments (shape.rs:108-154), missing normals
  derived smooth and area-weighted;
* `imagemap` textures on colour slots (map/mod.rs:1223-1258, 1300-1358):
  the image feeds the slot, whose constant becomes 1;
* an image `infinite` light: its square equal-area octahedral EXR resampled
  to the equirect sky the renderer reads, orientation and `scale` baked in
  (crates/cenote-pbrt/src/env.rs:36-176, map/mod.rs:853-907); an image-less
  one becomes a constant sky;
* media (`MakeNamedMedium`, `MediumInterface`) are ignored with a warning, as
  the reference's importer ignores them (map/mod.rs:402-408);
* `Integrator` maxdepth -> bounce cap, `Sampler` pixelsamples -> spp, `Film`
  resolution.

Unsupported directives and parameters are collected in `warnings`.
"""
from __future__ import annotations

import math
import re
from pathlib import Path

import numpy as np

from . import scenes

_TOKEN = re.compile(r'"[^"]*"|\[|\]|[^\s\[\]"#]+|#[^\n]*')


def _tokens(text: str):
    for m in _TOKEN.finditer(text):
        t = m.group(0)
        if t.startswith("#"):
            continue
        yield t


class _Params(dict):
    """name -> (type, values)."""

    def get_one(self, name, default=None):
        v = self.get(name)
        return default if v is None else v[1][0]

    def values(self, name):
        v = self.get(name)
        return None if v is None else v[1]

    def type_of(self, name):
        v = self.get(name)
        return None if v is None else v[0]


def _parse(text: str):
    """Yield (directive, names, params) tuples."""
    toks = list(_tokens(text))
    i = 0
    n = len(toks)

    def value(t):
        if t.startswith('"'):
            return t[1:-1]
        if t in ("true", "false"):
            return t == "true"
        return float(t)

    while i < n:
        d = toks[i]
        i += 1
        names, nums = [], []
        while i < n and toks[i].startswith('"') and " " not in toks[i][1:-1]:
            names.append(toks[i][1:-1])
            i += 1
        if i < n and toks[i] == "[" and d in ("Transform", "ConcatTransform"):
            j = toks.index("]", i)
            nums = [float(t) for t in toks[i + 1:j]]
            i = j + 1
        while i < n and re.fullmatch(r"[-+0-9.eE]+", toks[i]):
            nums.append(float(toks[i]))
            i += 1
        params = _Params()
        while i < n and toks[i].startswith('"') and " " in toks[i][1:-1]:
            typ, name = toks[i][1:-1].split()
            i += 1
            if toks[i] == "[":
                j = toks.index("]", i)
                vals = [value(t) for t in toks[i + 1:j]]
                i = j + 1
            else:
                vals = [value(toks[i])]
                i += 1
            if typ == "bool":
                vals = [v if isinstance(v, bool) else str(v) == "true" for v in vals]
            params[name] = (typ, vals)
        yield d, names, nums, params


def _mat4_colmajor(nums):
    return np.array(nums, np.float64).reshape(4, 4).T


def _translate(x, y, z):
    m = np.eye(4)
    m[:3, 3] = (x, y, z)
    return m


def _rotate(deg, axis):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    s, c = math.sin(math.radians(deg)), math.cos(math.radians(deg))
    x, y, z = a
    m = np.eye(4)
    m[:3, :3] = [[x * x + (1 - x * x) * c, x * y * (1 - c) - z * s, x * z * (1 - c) + y * s],
                 [x * y * (1 - c) + z * s, y * y + (1 - y * y) * c, y * z * (1 - c) - x * s],
                 [x * z * (1 - c) - y * s, y * z * (1 - c) + x * s, z * z + (1 - z * z) * c]]
    return m


def _look_at(eye, at, up):
    """pbrt's LookAt: the world-from-camera inverse (a left-handed frame)."""
    eye, at, up = (np.asarray(v, np.float64) for v in (eye, at, up))
    d = at - eye
    d /= np.linalg.norm(d)
    right = np.cross(up / np.linalg.norm(up), d)
    right /= np.linalg.norm(right)
    new_up = np.cross(d, right)
    cam_to_world = np.eye(4)
    cam_to_world[:3, 0], cam_to_world[:3, 1], cam_to_world[:3, 2], cam_to_world[:3, 3] = right, new_up, d, eye
    return np.linalg.inv(cam_to_world)


FLIP_Z = np.diag([1.0, 1.0, -1.0, 1.0])


def _conductor_f0(eta, k):
    eta = np.asarray(eta, np.float32)
    k = np.asarray(k, np.float32)
    return ((eta - np.float32(1.0)) ** 2 + k * k) / ((eta + np.float32(1.0)) ** 2 + k * k)


NAMED_METAL_F0 = {"Cu": (0.955, 0.638, 0.538), "Au": (1.000, 0.782, 0.344), "Ag": (0.972, 0.960, 0.915),
                  "Al": (0.913, 0.921, 0.925)}


def sphere_mesh(radius: float) -> scenes.Mesh:
    rings, segments = 32, 64
    pos, nrm, uv = [], [], []
    for ring in range(rings + 1):
        v = np.float32(ring) / np.float32(rings)
        theta = v * np.float32(math.pi)
        st, ct = np.sin(theta, dtype=np.float32), np.cos(theta, dtype=np.float32)
        for seg in range(segments + 1):
            u = np.float32(seg) / np.float32(segments)
            phi = u * np.float32(2 * math.pi)
            n = np.array([st * np.cos(phi, dtype=np.float32), st * np.sin(phi, dtype=np.float32), ct], np.float32)
            pos.append(n * np.float32(radius))
            nrm.append(n)
            uv.append((u, v))
    tris = []
    row = segments + 1
    for ring in range(rings):
        for seg in range(segments):
            a = ring * row + seg
            b = a + row
            if ring != 0:
                tris.append((a, b, a + 1))
            if ring != rings - 1:
                tris.append((a + 1, b, b + 1))
    return scenes.Mesh(np.array(pos, np.float32), np.array(nrm, np.float32), np.array(uv, np.float32),
                       np.array(tris, np.uint32))


def _cross32(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    f = np.float32
    return np.stack([a[:, 1] * b[:, 2] - b[:, 1] * a[:, 2], a[:, 2] * b[:, 0] - b[:, 2] * a[:, 0],
                     a[:, 0] * b[:, 1] - b[:, 0] * a[:, 1]], -1).astype(f)


def derive_normals(positions: np.ndarray, indices: np.ndarray) -> np.ndarray:
    """Smooth, area-weighted vertex normals from the winding, in the
    reference's f32 arithmetic (crates/cenote/src/scene/lower.rs:532-550):
    each face's unnormalised cross product adds onto its corners in triangle
    order, then each sum is scaled by the reciprocal of its length; a vertex
    whose sum cannot normalise takes +Y."""
    f = np.float32
    p = np.asarray(positions, f)
    idx = np.asarray(indices, np.int64).reshape(-1, 3)
    face = _cross32(p[idx[:, 1]] - p[idx[:, 0]], p[idx[:, 2]] - p[idx[:, 0]])
    n = np.zeros_like(p)
    np.add.at(n, idx.ravel(), np.repeat(face, 3, axis=0))  # f32, corners in triangle order
    dot = ((n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2]).astype(f)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        rcp = (f(1.0) / np.sqrt(dot)).astype(f)
    ok = np.isfinite(rcp) & (rcp > 0)
    out = np.where(ok[:, None], n * np.where(ok, rcp, f(0.0))[:, None], np.array([0.0, 1.0, 0.0], f))
    return out.astype(f)


def _inverse3_f32(m: np.ndarray) -> np.ndarray:
    """A 3x3 inverse as glam's Mat3::inverse computes it in f32: the columns'
    cross products over the determinant."""
    f = np.float32
    c = np.asarray(m, f).T  # c[k] = column k
    t0 = _cross32(c[1][None], c[2][None])[0]
    t1 = _cross32(c[2][None], c[0][None])[0]
    t2 = _cross32(c[0][None], c[1][None])[0]
    det = f((c[2][0] * t2[0] + c[2][1] * t2[1]) + c[2][2] * t2[2])
    inv = f(1.0) / det
    return np.stack([t0 * inv, t1 * inv, t2 * inv], 0).astype(f)  # rows = the transposed columns


class _State:
    def __init__(self):
        self.ctm = np.eye(4)
        self.material = None  # dict of material overrides
        self.area = None      # (rgb, scale)
        self.reverse = False

    def copy(self):
        s = _State()
        s.ctm = self.ctm.copy()
        s.material = self.material
        s.area = self.area
        s.reverse = self.reverse
        return s


def _openpbr(**kw):
    """OpenPBR's own defaults (description.rs:313-340), then overrides, lowered."""
    d = dict(base_color=(0.8, 0.8, 0.8), base_diffuse_roughness=0.0, metalness=0.0, specular_weight=1.0,
             specular_roughness=0.3, specular_ior=1.5, transmission_weight=0.0, transmission_color=(1.0, 1.0, 1.0),
             transmission_depth=0.0, coat_weight=0.0, coat_color=(1.0, 1.0, 1.0), coat_roughness=0.0, coat_ior=1.6,
             coat_darkening=1.0, fuzz_weight=0.0, fuzz_color=(1.0, 1.0, 1.0), fuzz_roughness=0.5,
             emission_luminance=0.0, emission_color=(1.0, 1.0, 1.0), opacity=1.0, thin_walled=False)
    d.update(kw)
    return d


def _lower(d) -> np.ndarray:
    """crates/cenote/src/scene/lower.rs:316-373."""
    coat_weight = float(np.clip(d["coat_weight"], 0.0, 1.0))
    coat_color = np.maximum(scenes.acescg(d["coat_color"]), 0.0)
    m = scenes.matte(scenes.acescg(d["base_color"]), float(np.clip(d["base_diffuse_roughness"], 0, 1)))
    m["metalness"] = float(np.clip(d["metalness"], 0, 1))
    m["specular_weight"] = max(float(d["specular_weight"]), 0.0)
    m["specular_roughness"] = float(d["specular_roughness"])
    m["specular_ior"] = max(float(d["specular_ior"]), 1e-4)
    m["transmission_weight"] = float(np.clip(d["transmission_weight"], 0, 1))
    m["transmission_color"] = np.clip(scenes.acescg(d["transmission_color"]), 0.0, 1.0)
    m["transmission_depth"] = max(float(d["transmission_depth"]), 0.0)
    m["coat_color"] = coat_color
    m["coat_weight"] = coat_weight
    m["coat_roughness"] = float(np.clip(d["coat_roughness"], 0, 1))
    m["coat_ior"] = max(float(d["coat_ior"]), 1.0)
    m["coat_darkening"] = float(np.clip(d["coat_darkening"], 0, 1))
    m["fuzz_weight"] = float(np.clip(d["fuzz_weight"], 0, 1))
    m["fuzz_color"] = np.maximum(scenes.acescg(d["fuzz_color"]), 0.0)
    m["fuzz_roughness"] = float(np.clip(d["fuzz_roughness"], 0, 1))
    m["opacity"] = float(np.clip(d["opacity"], 0, 1))
    m["thin_walled"] = 1 if d["thin_walled"] else 0
    lerp = np.float32(1.0) * (np.float32(1.0) - np.float32(coat_weight)) + coat_color * np.float32(coat_weight)
    m["emission"] = (scenes.acescg(d["emission_color"]) * np.float32(d["emission_luminance"])) * lerp
    return m


def _sphere_to_square(d: np.ndarray) -> np.ndarray:
    """Clarberg's equal-area sphere -> square map (env.rs:103-128), f32:
    +z at the square's centre, -z at its corners. d: (N, 3) unit vectors."""
    f = np.float32
    x, y, z = np.abs(d[:, 0]), np.abs(d[:, 1]), np.abs(d[:, 2])
    r = np.sqrt(np.maximum(f(1.0) - z, f(0.0)))
    a, b = np.maximum(x, y), np.minimum(x, y)
    with np.errstate(divide="ignore", invalid="ignore"):
        b = np.where(a == 0, f(0.0), b / np.where(a == 0, f(1.0), a)).astype(f)
    phi = (np.arctan(b.astype(np.float64)).astype(f) * f(2.0 / math.pi)).astype(f)
    phi = np.where(x < y, f(1.0) - phi, phi)
    v = phi * r
    u = r - v
    neg = d[:, 2] < 0
    u, v = np.where(neg, f(1.0) - v, u), np.where(neg, f(1.0) - u, v)
    u = np.copysign(u, d[:, 0])
    v = np.copysign(v, d[:, 1])
    return np.stack([f(0.5) * (u + f(1.0)), f(0.5) * (v + f(1.0))], -1).astype(f)


def _wrap_square(x: np.ndarray, y: np.ndarray):
    """Mirror taps back into the square across the octahedron's seams
    (env.rs:130-150, pbrt's WrapEqualAreaSquare)."""
    f = np.float32
    lo, hi = x < 0, x > 1
    x = np.where(lo, -x, np.where(hi, f(2.0) - x, x))
    y = np.where(lo | hi, f(1.0) - y, y)
    lo, hi = y < 0, y > 1
    x = np.where(lo | hi, f(1.0) - x, x)
    y = np.where(lo, -y, np.where(hi, f(2.0) - y, y))
    return x.astype(f), y.astype(f)


def resample_octahedral(texels: np.ndarray, world_from_light: np.ndarray, scale: float) -> np.ndarray:
    """A square equal-area octahedral sky (S, S, 3), linear Rec.709, as the
    equirect image (S, 2S, 3) the renderer's environment reads (row 0 the +Y
    zenith, the horizontal centre facing -Z), radiance times `scale`, each
    direction mapped into the light's frame first (env.rs:36-77, 88-100,
    152-176), in f32."""
    f = np.float32
    size = texels.shape[0]
    if texels.shape[1] != size:
        raise ValueError(f"an infinite light's image is {texels.shape[1]}x{size}: pbrt-v4 skies are square "
                         "equal-area octahedral images")
    ow = min(2 * size, 4096)
    oh = ow // 2
    light_from_world = _inverse3_f32(world_from_light)
    u = ((np.arange(ow, dtype=f) + f(0.5)) / f(ow)).astype(f)
    v = ((np.arange(oh, dtype=f) + f(0.5)) / f(oh)).astype(f)
    uu, vv = np.meshgrid(u, v)
    phi = (f(2.0 * math.pi) * (uu - f(0.5))).astype(f)
    theta = (f(math.pi) * vv).astype(f)
    # f32 sines and cosines correctly rounded (through f64), as the C
    # library's sinf/cosf return them.
    t64, p64 = theta.astype(np.float64), phi.astype(np.float64)
    st, ct = np.sin(t64).astype(f), np.cos(t64).astype(f)
    d = np.stack([st * np.sin(p64).astype(f), ct, -st * np.cos(p64).astype(f)], -1).reshape(-1, 3).astype(f)
    m = light_from_world
    ld = np.stack([(m[r, 0] * d[:, 0] + m[r, 1] * d[:, 1]) + m[r, 2] * d[:, 2] for r in range(3)], -1).astype(f)
    dot = ((ld[:, 0] * ld[:, 0] + ld[:, 1] * ld[:, 1]) + ld[:, 2] * ld[:, 2]).astype(f)
    ld = (ld * (f(1.0) / np.sqrt(dot)).astype(f)[:, None]).astype(f)
    uv = _sphere_to_square(ld)
    sz = f(size)
    px, py = (uv[:, 0] * sz - f(0.5)).astype(f), (uv[:, 1] * sz - f(0.5)).astype(f)
    x0, y0 = np.floor(px).astype(f), np.floor(py).astype(f)
    fx, fy = (px - x0).astype(f), (py - y0).astype(f)
    flat = np.asarray(texels, f).reshape(-1, 3)
    out = np.zeros((len(px), 3), f)
    for dx, dy, w in ((0, 0, (f(1) - fx) * (f(1) - fy)), (1, 0, fx * (f(1) - fy)), (0, 1, (f(1) - fx) * fy),
                      (1, 1, fx * fy)):
        tx, ty = _wrap_square(((x0 + f(dx) + f(0.5)) / sz).astype(f), ((y0 + f(dy) + f(0.5)) / sz).astype(f))
        ix = np.minimum((tx * sz).astype(np.int64), size - 1)
        iy = np.minimum((ty * sz).astype(np.int64), size - 1)
        out = (out + w.astype(f)[:, None] * flat[iy * size + ix]).astype(f)
    return (out * f(scale)).astype(f).reshape(oh, ow, 3)


def sky_environment(octahedral: np.ndarray, world_from_light: np.ndarray, scale: float) -> scenes.Environment:
    """The renderer's environment for an image infinite light: the
    octahedral sky resampled to equirect, then to ACEScg."""
    return scenes.environment_rec709(resample_octahedral(np.asarray(octahedral, np.float32), world_from_light, scale))


class PbrtImport:
    def __init__(self, base: Path | None = None):
        self.base = Path(base) if base is not None else Path(".")
        self.textures = []       # scenes.Texture, the bindless table
        self.named_textures = {}  # name -> (path, encoding)
        self.texture_slots = {}   # (path, srgb) -> table index
        self.environment = scenes.Environment.constant((0.0, 0.0, 0.0))
        self.sky = False
        self.sky_source = None  # (octahedral Rec.709 texels, world_from_light, scale) of an image sky
        self.warnings = []
        self.named = {}
        self.objects = []
        self.res = (1280, 720)
        self.spp = 64
        self.max_bounces = 5
        self.camera = None
        self.conjugation = FLIP_Z

    def _roughness(self, p: _Params):
        remap = p.get_one("remaproughness", True)
        r = p.get_one("roughness")
        aniso = [p.get_one(n) for n in ("uroughness", "vroughness") if n in p]
        if aniso:
            r = sum(aniso) / len(aniso)
        r = 0.0 if r is None else max(float(r), 0.0)
        return r ** (0.25 if remap else 0.5)

    def _texture_slot(self, name: str, color: bool) -> int:
        """The table index of named imagemap texture `name` (an 8-bit PNG)."""
        from .scene_file import read_png
        path, encoding = self.named_textures[name]
        srgb = color if encoding is None else encoding == "sRGB"
        key = (str(path), srgb)
        if key not in self.texture_slots:
            img = read_png(path)
            if img.shape[2] == 1:
                img = np.repeat(img, 3, 2)
            if img.shape[2] == 2:
                img = np.concatenate([np.repeat(img[..., :1], 3, 2), img[..., 1:]], 2)
            if img.shape[2] == 3:
                img = np.concatenate([img, np.full(img.shape[:2] + (1,), 255, np.uint8)], 2)
            self.textures.append(scenes.prepared_texture(img, "color" if color else "data", srgb))
            self.texture_slots[key] = len(self.textures) - 1
        return self.texture_slots[key]

    def _material(self, ty, p: _Params):
        refl = p.values("reflectance")
        if ty == "diffuse" and p.type_of("reflectance") == "texture":
            name = str(refl[0])
            if name in self.named_textures:
                d = _openpbr(base_color=(1.0, 1.0, 1.0), specular_weight=0.0)
                d["base_color_texture"] = self._texture_slot(name, True)
                return d
            self.warnings.append(f'unknown texture "{name}": mid-grey used')
            return _openpbr(base_color=(0.5, 0.5, 0.5), specular_weight=0.0)
        if ty == "diffuse":
            return _openpbr(base_color=tuple(refl) if refl else (0.5, 0.5, 0.5), specular_weight=0.0)
        if ty == "coateddiffuse":
            return _openpbr(base_color=tuple(refl) if refl else (0.5, 0.5, 0.5), specular_weight=0.0,
                            coat_weight=1.0, coat_ior=float(p.get_one("eta", 1.5)),
                            coat_roughness=self._roughness(p))
        if ty == "conductor":
            if refl:
                f0 = tuple(refl)
            else:
                eta, k = p.values("eta"), p.values("k")
                if eta and k and p.type_of("eta") in ("rgb", "color") and p.type_of("k") in ("rgb", "color"):
                    f0 = tuple(_conductor_f0(eta, k))
                else:
                    name = str((eta or k or ["metal-Cu-eta"])[0])
                    metal = name.replace("metal-", "").replace("-eta", "").replace("-k", "")
                    f0 = NAMED_METAL_F0.get(metal, NAMED_METAL_F0["Cu"])
            return _openpbr(metalness=1.0, base_color=f0, specular_roughness=self._roughness(p))
        if ty in ("dielectric", "thindielectric"):
            d = _openpbr(transmission_weight=1.0, specular_ior=float(p.get_one("eta", 1.5)))
            if ty == "thindielectric":
                d["thin_walled"] = True
            else:
                d["specular_roughness"] = self._roughness(p)
            return d
        self.warnings.append(f'material "{ty}" is not supported: OpenPBR defaults used')
        return _openpbr()

    def run(self, path: Path):
        return self.run_text(Path(path).read_text())

    def run_text(self, text: str):
        st = _State()
        stack = []
        cam_ctm = np.eye(4)
        fov = 90.0
        lens = (0.0, 1e6)
        in_world = False
        for d, names, nums, p in _parse(text):
            if d in ("AttributeBegin", "TransformBegin"):
                stack.append(st.copy())
            elif d in ("AttributeEnd", "TransformEnd"):
                old = stack.pop()
                if d == "TransformEnd":
                    st.ctm = old.ctm
                else:
                    st = old
            elif d == "Transform":
                st.ctm = _mat4_colmajor(nums)
            elif d == "ConcatTransform":
                st.ctm = st.ctm @ _mat4_colmajor(nums)
            elif d == "Translate":
                st.ctm = st.ctm @ _translate(*nums[:3])
            elif d == "Scale":
                st.ctm = st.ctm @ np.diag([nums[0], nums[1], nums[2], 1.0])
            elif d == "Rotate":
                st.ctm = st.ctm @ _rotate(nums[0], nums[1:4])
            elif d == "LookAt":
                st.ctm = st.ctm @ _look_at(nums[0:3], nums[3:6], nums[6:9])
            elif d == "Identity":
                st.ctm = np.eye(4)
            elif d == "ReverseOrientation":
                st.reverse = not st.reverse
            elif d == "Integrator":
                md = p.get_one("maxdepth")
                if md is not None:
                    self.max_bounces = max(1, int(md))
            elif d == "Sampler":
                self.spp = int(p.get_one("pixelsamples", 16))
            elif d == "Film":
                self.res = (int(p.get_one("xresolution", 1280)), int(p.get_one("yresolution", 720)))
            elif d == "Camera":
                cam_ctm = st.ctm.copy()
                fov = float(p.get_one("fov", 90.0))
                lens = (float(p.get_one("lensradius", 0.0)), float(p.get_one("focaldistance", 1e6)))
            elif d == "WorldBegin":
                in_world = True
                st.ctm = np.eye(4)
                world_from_camera = np.linalg.inv(cam_ctm)
                self.conjugation = np.eye(4) if np.linalg.det(world_from_camera[:3, :3]) < 0 else FLIP_Z
                w, h = self.res
                vfov = fov if w >= h else 2.0 * math.degrees(math.atan(math.tan(math.radians(fov) / 2) * h / w))
                c2w = self.conjugation @ world_from_camera
                pos = c2w[:3, 3]
                fwd = c2w[:3, 2] / np.linalg.norm(c2w[:3, 2])
                up = c2w[:3, 1]
                self.camera = scenes.Camera(tuple(pos), tuple(pos + fwd), tuple(up), vfov,
                                            aperture_radius=lens[0],
                                            focus_distance=lens[1] if lens[0] > 0 else 1.0)
            elif d == "MakeNamedMaterial":
                self.named[names[0]] = self._material(p.get_one("type", "diffuse"), p)
            elif d == "NamedMaterial":
                st.material = self.named.get(names[0])
                if st.material is None:
                    self.warnings.append(f'unknown material "{names[0]}"')
            elif d == "Material":
                st.material = self._material(names[0] if names else "diffuse", p)
            elif d == "AreaLightSource":
                if names and names[0] == "diffuse":
                    st.area = (tuple(p.values("L") or (1.0, 1.0, 1.0)), float(p.get_one("scale", 1.0)))
                    if p.get_one("twosided", False):
                        self.warnings.append("two-sided area light imported one-sided")
                else:
                    st.area = None
                    self.warnings.append(f"area light {names} is not supported")
            elif d == "Shape":
                self._shape(names[0], p, st)
            elif d == "Texture":
                if len(names) >= 3 and names[2] == "imagemap" and p.get_one("filename") is not None:
                    enc = p.get_one("encoding")
                    self.named_textures[names[0]] = (self.base / str(p.get_one("filename")),
                                                     enc if enc in ("sRGB", "linear") else None)
                else:
                    self.warnings.append(f"texture {names} is not supported")
            elif d == "LightSource":
                self._light(names[0] if names else "", p, st)
            elif d in ("MakeNamedMedium", "MediumInterface"):
                self.warnings.append(f"{d}: participating media are not supported, ignored")
            elif d in ("WorldEnd", "PixelFilter", "ColorSpace", "Option"):
                pass
            else:
                self.warnings.append(f"directive {d} is not supported")
        if not in_world or self.camera is None:
            raise ValueError("pbrt file has no WorldBegin / Camera")
        return self

    def _light(self, ty, p: _Params, st: _State):
        if ty != "infinite":
            self.warnings.append(f'light "{ty}" is not supported')
            return
        if self.sky:
            self.warnings.append("one environment is rendered: a further infinite light is skipped")
            return
        scale = float(p.get_one("scale", 1.0))
        if p.get_one("filename") is not None:
            from .exr import read_exr
            ch = read_exr(self.base / str(p.get_one("filename")))
            src = np.stack([ch["R"], ch["G"], ch["B"]], -1).astype(np.float32)
            world_from_light = (self.conjugation @ st.ctm)[:3, :3].astype(np.float32)
            self.sky_source = (src, world_from_light, scale)
            self.environment = sky_environment(src, world_from_light, scale)
        else:
            rgb = np.asarray(p.values("L") or (1.0, 1.0, 1.0), np.float32) * np.float32(scale)
            self.environment = scenes.environment_rec709(np.tile(rgb.reshape(1, 1, 3), (1, 2, 1)))
        self.sky = True

    def _shape(self, ty, p: _Params, st: _State):
        flip = st.reverse ^ (np.linalg.det(st.ctm[:3, :3]) < 0)
        if ty == "trianglemesh":
            pos = np.asarray(p.values("P"), np.float32).reshape(-1, 3)
            idx = p.values("indices")
            idx = np.asarray(idx if idx is not None else [0, 1, 2], np.uint32).reshape(-1, 3)
            nrm = p.values("N")
            nrm = None if nrm is None else np.asarray(nrm, np.float32).reshape(-1, 3)
            uv = p.values("uv")
            uv = np.zeros((len(pos), 2), np.float32) if uv is None else np.asarray(uv, np.float32).reshape(-1, 2)
            if flip:
                if nrm is not None:
                    nrm = -nrm
                idx = idx[:, [0, 2, 1]].copy()
            if nrm is None:
                nrm = derive_normals(pos, idx)
            mesh = scenes.Mesh(pos, nrm, uv, idx)
        elif ty == "plymesh":
            from .scene_file import read_ply
            if flip:
                self.warnings.append("ReverseOrientation on a plymesh is ignored")
            pos, nrm, uv, idx = read_ply(self.base / str(p.get_one("filename")))
            nrm = derive_normals(pos, idx) if nrm is None else nrm
            uv = np.zeros((len(pos), 2), np.float32) if uv is None else uv
            mesh = scenes.Mesh(pos, nrm, uv, idx)
        elif ty == "sphere":
            mesh = sphere_mesh(float(p.get_one("radius", 1.0)))
        else:
            self.warnings.append(f'shape "{ty}" is not supported: skipped')
            return
        base = st.material if st.material is not None else _openpbr(base_color=(0.5, 0.5, 0.5), specular_weight=0.0)
        if st.area is not None:
            base = dict(base, emission_color=st.area[0], emission_luminance=st.area[1])
        xf = scenes.rows(self.conjugation @ st.ctm)
        slot = base.get("base_color_texture")
        mat = _lower({k: v for k, v in base.items() if k != "base_color_texture"})
        if slot is not None:
            mat["base_color_texture"] = slot
        self.objects.append(scenes.Object(mesh, xf, mat))

    def spec(self, name="pbrt") -> scenes.SceneSpec:
        w, h = self.res
        return scenes.SceneSpec(name, self.objects, self.camera, self.environment, w, h, self.spp, self.max_bounces,
                                textures=list(self.textures))


def import_pbrt(path, width=None, height=None) -> scenes.SceneSpec:
    """Import a pbrt-v4 file; width/height override its Film resolution."""
    return import_pbrt_text(Path(path).read_text(), width, height, Path(path).parent.name, Path(path).parent)


def import_pbrt_text(text: str, width=None, height=None, name="pbrt", base=None) -> scenes.SceneSpec:
    """Import pbrt-v4 text; files it names resolve against `base`."""
    imp = PbrtImport(base).run_text(text)
    spec = imp.spec(name)
    spec.sky_source = imp.sky_source
    if width:
        spec.width = width
    if height:
        spec.height = height
    spec.warnings = imp.warnings
    return spec
