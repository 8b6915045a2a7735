"""Scene files: the reference's `.ron` change-set format, loaded into a SceneSpec.

A scene file is `(version: 1, ops: [...])`, an ordered list of edits applied
to an empty scene (crates/cenote/src/scene/changeset.rs:76-118, format.rs:
70-107): each op upserts a named mesh, instance, material, light, camera,
environment or settings object (fields not mentioned keep their values, new
objects start at their defaults), and `Remove(Kind, "name")` deletes one.
Lowering follows crates/cenote/src/scene/description.rs and lower.rs:
`Trs` = translate · Rz · Ry · Rx · scale (description.rs:134-159), OpenPBR
defaults for unmentioned material fields, colours as linear Rec.709 converted
to ACEScg, delta lights (lower.rs:237-266), an EXR environment converted per
texel (environment.rs:82-96), textured parameters read from PNG (8-bit, sRGB
for colour slots unless `color_space: Some(Linear)`) or EXR (linear) and
normal maps always linear. Relative paths resolve against the file's
directory (changeset.rs:300-320).

The RON reader is written for this format: structs and tuples in
parentheses, lists, `Some(..)`/`None`, enum variants with named or positional
payloads, strings, numbers, booleans and comments.
"""
from __future__ import annotations

import math
import re
import struct
import zlib
from pathlib import Path

import numpy as np

from . import scenes
from .pbrt import _lower, _openpbr, derive_normals

# ---- RON ---------------------------------------------------------------------------

_TOK = re.compile(r'\s+|//[^\n]*|/\*.*?\*/|"(?:[^"\\]|\\.)*"|[-+]?(?:\d+\.?\d*(?:[eE][-+]?\d+)?|\.\d+)|'
                  r'[A-Za-z_][A-Za-z0-9_]*|[()\[\]{},:]', re.S)


class Enum:
    """A RON enum variant or named struct: `name` and its payload (a dict of
    named fields, or a list of positional values)."""

    def __init__(self, name, payload):
        self.name, self.payload = name, payload

    def __repr__(self):
        return f"{self.name}{self.payload!r}"


def parse_ron(text: str):
    toks = []
    pos = 0
    while pos < len(text):
        m = _TOK.match(text, pos)
        if not m:
            raise ValueError(f"RON: unexpected character at {pos}: {text[pos:pos + 20]!r}")
        t = m.group(0)
        pos = m.end()
        if t.strip() and not t.startswith("//") and not t.startswith("/*"):
            toks.append(t)
    i = 0

    def peek():
        return toks[i] if i < len(toks) else None

    def take(expect=None):
        nonlocal i
        if i >= len(toks):
            raise ValueError("RON: unexpected end")
        t = toks[i]
        if expect is not None and t != expect:
            raise ValueError(f"RON: expected {expect!r}, got {t!r}")
        i += 1
        return t

    def group(close):
        """Items up to `close`: a dict when they are `key: value`, else a list."""
        named, items = None, []
        while peek() != close:
            if i + 1 < len(toks) and re.match(r"[A-Za-z_]", toks[i]) and toks[i + 1] == ":":
                key = take()
                take(":")
                named = named if named is not None else {}
                named[key] = value()
            else:
                items.append(value())
            if peek() == ",":
                take(",")
        take(close)
        return named if named is not None else items

    def value():
        t = take()
        if t == "(":
            g = group(")")
            return g if isinstance(g, dict) else tuple(g)
        if t == "[":
            return group("]")
        if t.startswith('"'):
            return bytes(t[1:-1], "utf-8").decode("unicode_escape")
        if t in ("true", "false"):
            return t == "true"
        if t == "None":
            return None
        if re.match(r"[-+.\d]", t):
            return float(t) if re.search(r"[.eE]", t) else int(t)
        if peek() == "(":
            take("(")
            g = group(")")
            if t == "Some":
                return g[0] if isinstance(g, list) else g
            return Enum(t, g)
        return Enum(t, None)

    v = value()
    if i != len(toks):
        raise ValueError("RON: trailing tokens")
    return v


# ---- images ------------------------------------------------------------------------------


def read_png(path) -> np.ndarray:
    """8-bit non-interlaced PNG (grey, grey+alpha, RGB, RGBA) as uint8 (H, W, C)."""
    data = Path(path).read_bytes()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError(f"{path}: not a PNG")
    pos, idat, w = 8, b"", None
    while pos < len(data):
        n, kind = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if kind == b"IHDR":
            w, h, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body)
            if depth != 8 or interlace or ctype not in (0, 2, 4, 6):
                raise ValueError(f"{path}: only 8-bit, non-interlaced grey/RGB(A) PNGs are read")
            ch = {0: 1, 2: 3, 4: 2, 6: 4}[ctype]
        elif kind == b"IDAT":
            idat += body
        elif kind == b"IEND":
            break
    raw = np.frombuffer(zlib.decompress(idat), np.uint8)
    stride = w * ch
    out = np.zeros((h, stride), np.int32)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        f = raw[y * (stride + 1)]
        line = raw[y * (stride + 1) + 1:(y + 1) * (stride + 1)].astype(np.int32)
        cur = np.zeros(stride, np.int32)
        for x in range(stride):
            a = cur[x - ch] if x >= ch else 0
            b = prev[x]
            c = prev[x - ch] if x >= ch else 0
            if f == 0:
                p = 0
            elif f == 1:
                p = a
            elif f == 2:
                p = b
            elif f == 3:
                p = (a + b) // 2
            else:
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            cur[x] = (line[x] + p) & 0xFF
        out[y] = cur
        prev = cur
    return out.reshape(h, w, ch).astype(np.uint8)


def read_ply(path):
    """PLY meshes (ascii or binary little-endian): positions, optional
    normals and uvs, triangulated faces (fans)."""
    data = Path(path).read_bytes()
    end = data.index(b"end_header") + len(b"end_header")
    end = data.index(b"\n", end) + 1
    header = data[:end].decode("ascii").splitlines()
    fmt = next(l.split()[1] for l in header if l.startswith("format"))
    elements, cur = [], None
    for line in header:
        p = line.split()
        if p[:1] == ["element"]:
            cur = [p[1], int(p[2]), []]
            elements.append(cur)
        elif p[:1] == ["property"]:
            cur[2].append(p[1:])
    types = {"char": "b", "uchar": "B", "int8": "b", "uint8": "B", "short": "h", "ushort": "H", "int16": "h",
             "uint16": "H", "int": "i", "uint": "I", "int32": "i", "uint32": "I", "float": "f", "float32": "f",
             "double": "d", "float64": "d"}
    body = data[end:]
    if fmt == "ascii":
        words = body.split()
        k = 0
    else:
        if fmt != "binary_little_endian":
            raise ValueError(f"{path}: {fmt} PLY is not read")
        off = 0
    verts, faces = {}, []
    for name, count, props in elements:
        if name == "vertex":
            cols = {q[-1]: [] for q in props}
        for _ in range(count):
            row = {}
            for q in props:
                if q[0] == "list":
                    ct, it = types[q[1]], types[q[2]]
                    if fmt == "ascii":
                        n = int(words[k]); k += 1
                        vals = [float(w) for w in words[k:k + n]]; k += n
                    else:
                        n = struct.unpack_from("<" + ct, body, off)[0]; off += struct.calcsize(ct)
                        vals = list(struct.unpack_from(f"<{n}{it}", body, off)); off += n * struct.calcsize(it)
                    row[q[-1]] = vals
                else:
                    t = types[q[0]]
                    if fmt == "ascii":
                        row[q[-1]] = float(words[k]); k += 1
                    else:
                        row[q[-1]] = struct.unpack_from("<" + t, body, off)[0]; off += struct.calcsize(t)
            if name == "vertex":
                for key, val in row.items():
                    cols[key].append(val)
            elif name == "face":
                idx = row.get("vertex_indices", row.get("vertex_index"))
                for j in range(1, len(idx) - 1):
                    faces.append((int(idx[0]), int(idx[j]), int(idx[j + 1])))
        if name == "vertex":
            verts = cols
    pos = np.stack([verts["x"], verts["y"], verts["z"]], -1).astype(np.float32)
    nrm = np.stack([verts["nx"], verts["ny"], verts["nz"]], -1).astype(np.float32) if "nx" in verts else None
    uk = next(((a, b) for a, b in (("u", "v"), ("s", "t"), ("texture_u", "texture_v")) if a in verts), None)
    uv = np.stack([verts[uk[0]], verts[uk[1]]], -1).astype(np.float32) if uk else None
    return pos, nrm, uv, np.asarray(faces, np.uint32).reshape(-1, 3)


# ---- the change set ------------------------------------------------------------------------

KINDS = ("Mesh", "Instance", "Material", "Light", "Camera", "Environment", "Settings")


def _rot(axis, deg):
    a = math.radians(deg)
    c, s = math.cos(a), math.sin(a)
    m = np.eye(4)
    i, j = {"x": (1, 2), "y": (2, 0), "z": (0, 1)}[axis]
    m[i, i], m[i, j], m[j, i], m[j, j] = c, -s, s, c
    return m


def transform_matrix(t) -> np.ndarray:
    """description.rs:134-159: Trs = T · Rz · Ry · Rx · S, or Matrix rows."""
    if t is None:
        return np.eye(4)
    if t.name == "Trs":
        p = t.payload or {}
        tr, rd, sc = p.get("translate", (0, 0, 0)), p.get("rotate_degrees", (0, 0, 0)), p.get("scale", (1, 1, 1))
        return scenes.translate(*tr) @ _rot("z", rd[2]) @ _rot("y", rd[1]) @ _rot("x", rd[0]) @ np.diag(
            [sc[0], sc[1], sc[2], 1.0])
    if t.name == "Matrix":
        rows = t.payload[0]
        m = np.eye(4)
        m[:3] = np.asarray(rows, np.float64)
        return m
    raise ValueError(f"unknown transform {t.name}")


class SceneFile:
    """The objects of an applied change set, by kind and name."""

    def __init__(self, base: Path):
        self.base = base
        self.objects = {k: {} for k in KINDS}

    def apply(self, ops) -> None:
        for op in ops:
            if not isinstance(op, Enum):
                raise ValueError(f"not an op: {op!r}")
            if op.name == "Remove":
                kind, name = op.payload
                if name not in self.objects[kind.name]:
                    raise ValueError(f"Remove: no {kind.name} named {name!r}")
                self.objects[kind.name].pop(name)
                continue
            if op.name not in KINDS:
                raise ValueError(f"unknown op {op.name}")
            patch = op.payload[0] if isinstance(op.payload, list) else op.payload
            name = patch["name"]
            target = self.objects[op.name].setdefault(name, {})
            for key, val in patch.items():
                if key != "name" and val is not None:
                    target[key] = val

    def path(self, p) -> Path:
        q = Path(p)
        return q if q.is_absolute() else self.base / q


def _texture(sf: SceneFile, ref: dict, kind: str, cache: dict, textures: list) -> int:
    """A texture slot for `ref` (payload of Texture(..)); kind: color, data, normal."""
    path = sf.path(ref["path"])
    space = ref.get("color_space")
    key = (str(path), kind, space.name if space else None)
    if key in cache:
        return cache[key]
    if path.suffix.lower() == ".exr":
        from .exr import read_exr
        ch = read_exr(path)
        rgba = np.stack([ch["R"], ch.get("G", ch["R"]), ch.get("B", ch["R"]),
                         ch.get("A", np.ones_like(ch["R"]))], -1).astype(np.float32)
        tex = scenes.prepared_float_texture(rgba, kind)
    else:
        img = read_png(path)
        if img.shape[2] == 1:
            img = np.repeat(img, 3, 2)
        if img.shape[2] == 2:
            img = np.concatenate([np.repeat(img[..., :1], 3, 2), img[..., 1:]], 2)
        if img.shape[2] == 3:
            img = np.concatenate([img, np.full(img.shape[:2] + (1,), 255, np.uint8)], 2)
        srgb = kind == "color" and (space is None or space.name == "Srgb")
        tex = scenes.prepared_texture(img, kind, srgb)
    textures.append(tex)
    cache[key] = len(textures) - 1
    return cache[key]


def lower(sf: SceneFile, width=None, height=None) -> scenes.SceneSpec:
    """The applied scene as a SceneSpec (lower.rs, prep.rs)."""
    textures, cache = [], {}
    materials = {}
    for name, m in sf.objects["Material"].items():
        d = _openpbr()
        slots = {}
        for key, val in m.items():
            field = {"base_metalness": "metalness", "geometry_opacity": "opacity",
                     "geometry_thin_walled": "thin_walled"}.get(key, key)
            if isinstance(val, Enum) and val.name == "Constant":
                d[field] = val.payload[0]
            elif isinstance(val, Enum) and val.name == "Texture":
                kind = "color" if key in ("base_color", "emission_color") else "data"
                slots[key] = _texture(sf, val.payload if isinstance(val.payload, dict) else val.payload[0], kind,
                                      cache, textures)
            elif key == "geometry_normal":
                ref = val.payload if isinstance(val, Enum) else val
                slots[key] = _texture(sf, ref if isinstance(ref, dict) else ref[0], "normal", cache, textures)
            else:
                d[field] = val
        if "base_color" in slots:
            d["base_color"] = (1.0, 1.0, 1.0)
        if "emission_color" in slots:
            d["emission_color"] = (1.0, 1.0, 1.0)
        mat = _lower(d)
        for key, slot in slots.items():
            mat[{"base_color": "base_color_texture", "base_metalness": "metalness_texture",
                 "specular_roughness": "specular_roughness_texture", "emission_color": "emission_texture",
                 "geometry_opacity": "opacity_texture", "geometry_normal": "normal_texture"}[key]] = slot
        materials[name] = mat
    meshes = {}
    for name, m in sf.objects["Mesh"].items():
        src = m.get("source")
        if src is None:
            raise ValueError(f"mesh {name!r} has no source")
        if src.name == "Inline":
            p = src.payload
            pos = np.asarray(p["positions"], np.float32).reshape(-1, 3)
            idx = np.asarray(p["triangles"], np.uint32).reshape(-1, 3)
            nrm = p.get("normals")
            uv = p.get("uvs")
        elif src.name == "Ply":
            pos, nrm, uv, idx = read_ply(sf.path(src.payload["path"]))
        else:
            raise ValueError(f"mesh source {src.name} is not supported")
        nrm = derive_normals(pos, idx) if nrm is None else np.asarray(nrm, np.float32).reshape(-1, 3)
        uv = np.zeros((len(pos), 2), np.float32) if uv is None else np.asarray(uv, np.float32).reshape(-1, 2)
        meshes[name] = scenes.Mesh(pos, nrm, uv, idx)
    default_mat = _lower(_openpbr())
    objects = []
    for name in sorted(sf.objects["Instance"]):
        inst = sf.objects["Instance"][name]
        mesh = meshes[inst["mesh"]]
        mat = materials.get(inst.get("material"), default_mat)
        objects.append(scenes.Object(mesh, scenes.rows(transform_matrix(inst.get("transform"))), mat,
                                     bool(inst.get("camera_visible", True))))
    cams = sf.objects["Camera"]
    c = cams[sorted(cams)[0]] if cams else {}
    position = tuple(c.get("position", (0.0, 0.0, 5.0)))
    look_at = tuple(c.get("look_at", (0.0, 0.0, 0.0)))
    focus = c.get("focus_distance")
    if focus is None:
        focus = float(np.linalg.norm(np.subtract(look_at, position)))
    camera = scenes.Camera(position, look_at, tuple(c.get("up", (0.0, 1.0, 0.0))), float(c.get("vfov_degrees", 40.0)),
                           float(c.get("aperture_radius", 0.0)), float(focus))
    envs = sf.objects["Environment"]
    env = scenes.Environment.constant((0.0, 0.0, 0.0))
    if envs:
        e = envs[sorted(envs)[0]]
        if e.get("path") is not None:
            from .exr import read_exr
            ch = read_exr(sf.path(e["path"]))
            env = scenes.environment_rec709(np.stack([ch["R"], ch["G"], ch["B"]], -1))
    deltas = []
    for name in sorted(sf.objects["Light"]):
        light = sf.objects["Light"][name].get("light")
        if light is None:
            continue
        p = light.payload
        if light.name == "Distant":
            d = np.asarray(p["direction"], np.float64)
            d = d / np.linalg.norm(d)
            deltas.append(scenes.DeltaLight(1, tuple(d), tuple(scenes.acescg(p["irradiance"]))))
        elif light.name == "Point":
            deltas.append(scenes.DeltaLight(2, tuple(p["position"]), tuple(scenes.acescg(p["intensity"]))))
    st = sf.objects["Settings"]
    s = st[sorted(st)[0]] if st else {}
    res = s.get("resolution", (1280, 720))
    spec = scenes.SceneSpec(sf.base.name, objects, camera, env, int(width or res[0]), int(height or res[1]),
                            int(s.get("spp", 64)), int(s.get("max_bounces", 8)), deltas, textures)
    return spec


def load_scene_file(path, width=None, height=None) -> scenes.SceneSpec:
    """Load a `.ron` scene file (format.rs:107) into a SceneSpec."""
    path = Path(path)
    doc = parse_ron(path.read_text())
    if not isinstance(doc, dict) or doc.get("version") != 1:
        raise ValueError(f"{path}: not a version-1 scene file")
    sf = SceneFile(path.parent)
    sf.apply(doc.get("ops", []))
    return lower(sf, width, height)
