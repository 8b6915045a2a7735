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
  transform), `sphere` tessellated 32 rings x 64 segments (shape.rs:108-154),
  missing normals derived smooth and area-weighted;
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


def derive_normals(positions: np.ndarray, indices: np.ndarray) -> np.ndarray:
    """Smooth, area-weighted vertex normals from the winding."""
    p = positions.astype(np.float64)
    face = np.cross(p[indices[:, 1]] - p[indices[:, 0]], p[indices[:, 2]] - p[indices[:, 0]])
    n = np.zeros_like(p)
    for k in range(3):
        np.add.at(n, indices[:, k], face)
    length = np.linalg.norm(n, axis=1, keepdims=True)
    n = np.where(length > 0, n / np.maximum(length, 1e-300), np.array([0.0, 0.0, 1.0]))
    return n.astype(np.float32)


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


class PbrtImport:
    def __init__(self):
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

    def _material(self, ty, p: _Params):
        refl = p.values("reflectance")
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
            elif d in ("WorldEnd", "PixelFilter", "ColorSpace", "Option"):
                pass
            else:
                self.warnings.append(f"directive {d} is not supported")
        if not in_world or self.camera is None:
            raise ValueError("pbrt file has no WorldBegin / Camera")
        return self

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
        elif ty == "sphere":
            mesh = sphere_mesh(float(p.get_one("radius", 1.0)))
        else:
            self.warnings.append(f'shape "{ty}" is not supported: skipped')
            return
        base = st.material if st.material is not None else _openpbr(base_color=(0.5, 0.5, 0.5), specular_weight=0.0)
        if st.area is not None:
            base = dict(base, emission_color=st.area[0], emission_luminance=st.area[1])
        xf = scenes.rows(self.conjugation @ st.ctm)
        self.objects.append(scenes.Object(mesh, xf, _lower(base)))

    def spec(self, name="pbrt") -> scenes.SceneSpec:
        w, h = self.res
        return scenes.SceneSpec(name, self.objects, self.camera, scenes.Environment.constant((0.0, 0.0, 0.0)), w, h,
                                self.spp, self.max_bounces)


def import_pbrt(path, width=None, height=None) -> scenes.SceneSpec:
    """Import a pbrt-v4 file; width/height override its Film resolution."""
    return import_pbrt_text(Path(path).read_text(), width, height, Path(path).parent.name)


def import_pbrt_text(text: str, width=None, height=None, name="pbrt") -> scenes.SceneSpec:
    imp = PbrtImport().run_text(text)
    spec = imp.spec(name)
    if width:
        spec.width = width
    if height:
        spec.height = height
    spec.warnings = imp.warnings
    return spec
