"""Procedural scene inputs: meshes, materials, cameras and environments.

Everything here is plain data (numpy float32/uint32 arrays and the 144-byte
material record), the same arrays whether they go to the CUDA library or to a
CPU check. The material constructors follow crates/cenote/src/material.rs:118-248,
the solids crates/cenote/src/scene/shapes.rs:21-117, and authored colours enter
through the Rec.709 -> ACEScg matrix of crates/cenote/src/color.rs:351-361.

The named workloads:

* ``cornell``   -- a closed box of five 2x2 quads, two white boxes and a 0.5x0.5
  ceiling emitter (36 triangles), pinhole 40 deg, 256x256, 16 spp, 8 bounces.
* ``chart``     -- a 5x5 grid of radius-0.4 icospheres (subdivision 3) sweeping
  roughness along x and metalness along z on a 20x20 glossy ground, a 1x1
  warm quad light and a procedural 2048x1024 HDRI sky with a 0.5 deg sun;
  1280x720, 64 spp, 12 bounces.
* ``terrain``   -- a 1024^2 fBm heightfield with 500 instanced glass, coated and
  fuzz meshes and 4096 lognormal-power emissive triangles; 1920x1080, 64 spp,
  16 bounces.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TEXTURE_NONE = 0xFFFFFFFF

MATERIAL_DTYPE = np.dtype(
    [
        ("base_color", "<f4", 3),
        ("base_roughness", "<f4"),
        ("emission", "<f4", 3),
        ("metalness", "<f4"),
        ("specular_weight", "<f4"),
        ("specular_roughness", "<f4"),
        ("specular_ior", "<f4"),
        ("transmission_weight", "<f4"),
        ("transmission_color", "<f4", 3),
        ("transmission_depth", "<f4"),
        ("coat_color", "<f4", 3),
        ("coat_weight", "<f4"),
        ("coat_roughness", "<f4"),
        ("coat_ior", "<f4"),
        ("coat_darkening", "<f4"),
        ("fuzz_weight", "<f4"),
        ("fuzz_color", "<f4", 3),
        ("fuzz_roughness", "<f4"),
        ("opacity", "<f4"),
        ("thin_walled", "<u4"),
        ("base_color_texture", "<u4"),
        ("specular_roughness_texture", "<u4"),
        ("metalness_texture", "<u4"),
        ("emission_texture", "<u4"),
        ("opacity_texture", "<u4"),
        ("normal_texture", "<u4"),
    ]
)
assert MATERIAL_DTYPE.itemsize == 144

# color.rs:351-355, applied as a column-major Mat3 in f32.
_ACESCG_FROM_REC709 = np.array(
    [
        [0.6130974, 0.33952314, 0.04737945],
        [0.07019373, 0.9163539, 0.013452399],
        [0.020615594, 0.10956978, 0.86981466],
    ],
    dtype=np.float32,
)


def acescg(rec709) -> np.ndarray:
    """Linear Rec.709 -> ACEScg, summed left to right in f32 like glam."""
    c = np.asarray(rec709, dtype=np.float32)
    m = _ACESCG_FROM_REC709
    out = np.empty(3, dtype=np.float32)
    for r in range(3):
        out[r] = (m[r, 0] * c[0] + m[r, 1] * c[1]) + m[r, 2] * c[2]
    return out


def material(**overrides) -> np.ndarray:
    """Material::matte(white, 0) with fields overridden (material.rs:122-151)."""
    m = np.zeros((), dtype=MATERIAL_DTYPE)
    m["base_color"] = (1.0, 1.0, 1.0)
    m["base_roughness"] = 0.0
    m["emission"] = (0.0, 0.0, 0.0)
    m["metalness"] = 0.0
    m["specular_weight"] = 0.0
    m["specular_roughness"] = 0.0
    m["specular_ior"] = 1.5
    m["transmission_weight"] = 0.0
    m["transmission_color"] = (1.0, 1.0, 1.0)
    m["transmission_depth"] = 0.0
    m["coat_color"] = (1.0, 1.0, 1.0)
    m["coat_weight"] = 0.0
    m["coat_roughness"] = 0.0
    m["coat_ior"] = 1.6
    m["coat_darkening"] = 1.0
    m["fuzz_weight"] = 0.0
    m["fuzz_color"] = (1.0, 1.0, 1.0)
    m["fuzz_roughness"] = 0.5
    m["opacity"] = 1.0
    m["thin_walled"] = 0
    for k in (
        "base_color_texture",
        "specular_roughness_texture",
        "metalness_texture",
        "emission_texture",
        "opacity_texture",
        "normal_texture",
    ):
        m[k] = TEXTURE_NONE
    for k, v in overrides.items():
        m[k] = v
    return m


def matte(base_color, base_roughness=0.0):
    return material(base_color=base_color, base_roughness=base_roughness)


def glossy(base_color, base_roughness, specular_roughness):
    return material(base_color=base_color, base_roughness=base_roughness, specular_weight=1.0,
                    specular_roughness=specular_roughness)


def metal(base_color, specular_roughness):
    return material(base_color=base_color, metalness=1.0, specular_weight=1.0,
                    specular_roughness=specular_roughness)


def glass(specular_roughness, specular_ior):
    return material(transmission_weight=1.0, specular_weight=1.0, specular_roughness=specular_roughness,
                    specular_ior=specular_ior)


def emitter(emission):
    return material(base_color=(0.0, 0.0, 0.0), emission=emission)


# ---- meshes -----------------------------------------------------------------


@dataclass
class Mesh:
    positions: np.ndarray  # (V, 3) f32
    normals: np.ndarray    # (V, 3) f32
    uvs: np.ndarray        # (V, 2) f32
    indices: np.ndarray    # (T, 3) u32, counter-clockwise outward

    @property
    def triangle_count(self) -> int:
        return int(self.indices.shape[0])


def _mesh(p, n, uv, idx) -> Mesh:
    return Mesh(np.ascontiguousarray(p, np.float32), np.ascontiguousarray(n, np.float32),
                np.ascontiguousarray(uv, np.float32), np.ascontiguousarray(idx, np.uint32))


def icosphere(subdivisions: int) -> Mesh:
    """Unit icosphere by 4-way splits with a shared midpoint cache (shapes.rs:21-57)."""
    phi = np.float32((1.0 + math.sqrt(5.0)) / 2.0)
    base = [[-1, phi, 0], [1, phi, 0], [-1, -phi, 0], [1, -phi, 0], [0, -1, phi], [0, 1, phi],
            [0, -1, -phi], [0, 1, -phi], [phi, 0, -1], [phi, 0, 1], [-phi, 0, -1], [-phi, 0, 1]]
    pos = [np.asarray(p, np.float32) / np.float32(np.sqrt(np.float32(np.dot(np.asarray(p, np.float32),
                                                                              np.asarray(p, np.float32)))))
           for p in base]
    tris = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
            [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
            [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    for _ in range(subdivisions):
        cache: dict = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = (pos[a] + pos[b]) * np.float32(0.5)
                m = m / np.float32(np.sqrt(np.float32(np.dot(m, m))))
                cache[key] = len(pos)
                pos.append(m.astype(np.float32))
            return cache[key]

        faces = []
        for a, b, c in tris:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            faces += [[a, ab, ca], [ab, b, bc], [ca, bc, c], [ab, bc, ca]]
        tris = faces
    p = np.stack(pos).astype(np.float32)
    return _mesh(p, p.copy(), np.zeros((len(p), 2), np.float32), np.asarray(tris, np.uint32))


def quad(corners, normal=None, uvs=None) -> Mesh:
    """Two triangles over four corners given counter-clockwise seen from the front."""
    c = np.asarray(corners, np.float32)
    n = np.cross(c[1] - c[0], c[2] - c[0]) if normal is None else np.asarray(normal, np.float32)
    n = (n / np.linalg.norm(n)).astype(np.float32)
    uv = np.array([[0, 0], [0, 1], [1, 1], [1, 0]], np.float32) if uvs is None else uvs
    return _mesh(c, np.tile(n, (4, 1)), uv, [[0, 1, 2], [0, 2, 3]])


def ground_plane(half_extent: float) -> Mesh:
    """The XZ plane at y = 0, normal +Y (shapes.rs:117-139)."""
    e = half_extent
    return _mesh([[-e, 0, -e], [-e, 0, e], [e, 0, e], [e, 0, -e]], [[0, 1, 0]] * 4,
                 [[0, 0], [0, 1], [1, 1], [1, 0]], [[0, 1, 2], [0, 2, 3]])


def box(sx: float, sy: float, sz: float) -> Mesh:
    """An axis-aligned box centred at the origin, flat-shaded, 12 outward triangles."""
    hx, hy, hz = sx / 2, sy / 2, sz / 2
    faces = [  # (normal, 4 corners counter-clockwise from outside)
        ((1, 0, 0), [(hx, -hy, hz), (hx, -hy, -hz), (hx, hy, -hz), (hx, hy, hz)]),
        ((-1, 0, 0), [(-hx, -hy, -hz), (-hx, -hy, hz), (-hx, hy, hz), (-hx, hy, -hz)]),
        ((0, 1, 0), [(-hx, hy, hz), (hx, hy, hz), (hx, hy, -hz), (-hx, hy, -hz)]),
        ((0, -1, 0), [(-hx, -hy, -hz), (hx, -hy, -hz), (hx, -hy, hz), (-hx, -hy, hz)]),
        ((0, 0, 1), [(-hx, -hy, hz), (hx, -hy, hz), (hx, hy, hz), (-hx, hy, hz)]),
        ((0, 0, -1), [(hx, -hy, -hz), (-hx, -hy, -hz), (-hx, hy, -hz), (hx, hy, -hz)]),
    ]
    p, n, uv, idx = [], [], [], []
    for normal, corners in faces:
        b = len(p)
        p += corners
        n += [normal] * 4
        uv += [(0, 0), (1, 0), (1, 1), (0, 1)]
        idx += [[b, b + 1, b + 2], [b, b + 2, b + 3]]
    return _mesh(p, n, uv, idx)


# ---- transforms -----------------------------------------------------------------


def translate(x, y, z) -> np.ndarray:
    m = np.eye(4)
    m[:3, 3] = (x, y, z)
    return m


def rotate_y(deg) -> np.ndarray:
    a = math.radians(deg)
    m = np.eye(4)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = math.cos(a), math.sin(a), -math.sin(a), math.cos(a)
    return m


def rotate_x(deg) -> np.ndarray:
    a = math.radians(deg)
    m = np.eye(4)
    m[1, 1], m[1, 2], m[2, 1], m[2, 2] = math.cos(a), -math.sin(a), math.sin(a), math.cos(a)
    return m


def scale(s) -> np.ndarray:
    m = np.eye(4)
    m[0, 0] = m[1, 1] = m[2, 2] = s
    return m


def rows(m4: np.ndarray) -> np.ndarray:
    """The top three rows of a 4x4 as the 12 f32 values a record carries."""
    return np.ascontiguousarray(np.asarray(m4, np.float64)[:3, :4], np.float32).reshape(12)


# ---- scenes ---------------------------------------------------------------------


@dataclass
class Object:
    mesh: Mesh
    transform: np.ndarray  # 12 f32, rows of a 3x4
    material: np.ndarray   # MATERIAL_DTYPE scalar
    camera_visible: bool = True


@dataclass
class Camera:
    position: tuple
    look_at: tuple
    up: tuple = (0.0, 1.0, 0.0)
    vfov_degrees: float = 40.0
    aperture_radius: float = 0.0
    focus_distance: float = 1.0


@dataclass
class Environment:
    width: int
    height: int
    texels: np.ndarray  # (H, W, 4) f32, ACEScg, row 0 = +Y

    @staticmethod
    def constant(rgb) -> "Environment":
        t = np.array([[[rgb[0], rgb[1], rgb[2], 1.0]]], np.float32)
        return Environment(1, 1, t)


def environment_rec709(rgb: np.ndarray) -> Environment:
    """An environment from linear Rec.709 texels (H, W, 3), row 0 the +Y
    zenith: converted to ACEScg as the reference's environment loader does,
    each channel summed left to right in f32 as `acescg` does for colours,
    negatives clamped to zero."""
    h, w = rgb.shape[:2]
    c = np.asarray(rgb, np.float32).reshape(-1, 3)
    m = _ACESCG_FROM_REC709
    ac = np.stack([(m[r, 0] * c[:, 0] + m[r, 1] * c[:, 1]) + m[r, 2] * c[:, 2] for r in range(3)], -1)
    ac = np.maximum(ac, np.float32(0.0))
    tex = np.concatenate([ac.reshape(h, w, 3), np.ones((h, w, 1), np.float32)], -1).astype(np.float32)
    return Environment(w, h, np.ascontiguousarray(tex))


@dataclass
class DeltaLight:
    kind: int  # 1 distant (anchor = unit travel direction), 2 point (anchor = position)
    anchor: tuple
    emission: tuple


# Texture formats of the bindless table (include/cenote_c.h CENOTE_TEXTURE_*).
TEX_RGBA8_SRGB, TEX_RGBA8_UNORM, TEX_RGBA32F = 1, 2, 3
TEX_BC1_SRGB, TEX_BC1_UNORM, TEX_BC4_UNORM, TEX_BC5_UNORM = 4, 5, 6, 7
TEX_BC7_SRGB, TEX_BC7_UNORM = 8, 9
TEX_BC6H_UF16, TEX_BC6H_SF16 = 10, 11


@dataclass
class Texture:
    """One slot of the bindless table: `data` is the texels (RGBA8 as uint8
    (H, W, 4), RGBA32F as float32 (H, W, 4)) or the BC blocks as uint8."""
    format: int
    width: int
    height: int
    data: np.ndarray


def rgba8_texture(rgb, srgb: bool = True, alpha=None) -> Texture:
    """An RGBA8 texture from float RGB in [0, 1] (H, W, 3), stored sRGB-encoded
    (colour) or linear (scalars, normal maps)."""
    rgb = np.clip(np.asarray(rgb, np.float32), np.float32(0), np.float32(1))
    if srgb:
        rgb = np.where(rgb <= np.float32(0.0031308), rgb * np.float32(12.92),
                       np.float32(1.055) * rgb ** np.float32(1 / 2.4) - np.float32(0.055))
    h, w = rgb.shape[:2]
    px = np.empty((h, w, 4), np.uint8)
    px[..., :3] = (rgb * np.float32(255) + np.float32(0.5)).astype(np.uint8)
    px[..., 3] = 255 if alpha is None else (np.clip(alpha, 0, 1) * 255 + 0.5).astype(np.uint8)
    return Texture(TEX_RGBA8_SRGB if srgb else TEX_RGBA8_UNORM, w, h, px)


def prepared_texture(rgba8, usage: str = "color", srgb: bool = True) -> Texture:
    """An 8-bit image (H, W, 4) stored the way the reference's texture prep
    stores it (crates/cenote/src/texture.rs:249-405): colour as BC7 (an sRGB
    view when `srgb`), scalars as BC4 on red, tangent-space normals as BC5 on
    x/y. Colour is encoded opaque, as the reference's encoder profile does
    (texture.rs:273-276, opaque settings): its alpha becomes 255 (no slot
    reads a colour texture's alpha), which also opens BC7's two-subset RGB
    modes to it. An image whose sides are not multiples of 4 stays RGBA8
    (the reference pads it to whole blocks instead)."""
    from . import encode_texture  # host BC encoder of the library

    rgba8 = np.ascontiguousarray(rgba8, np.uint8)
    h, w = rgba8.shape[:2]
    tex = Texture(TEX_RGBA8_SRGB if srgb else TEX_RGBA8_UNORM, w, h, rgba8)
    if w % 4 or h % 4:
        return tex
    if usage == "color":
        rgba8 = rgba8.copy()
        rgba8[..., 3] = 255
        tex = Texture(tex.format, w, h, rgba8)
    fmt = {"color": TEX_BC7_SRGB if srgb else TEX_BC7_UNORM, "data": TEX_BC4_UNORM, "normal": TEX_BC5_UNORM}[usage]
    return encode_texture(fmt, tex)


def prepared_float_texture(rgba32f, usage: str = "color") -> Texture:
    """A float image (H, W, 4) stored the way the reference's prep stores it
    (texture.rs:283-405): colour as BC6H unsigned (negatives clamp to zero,
    alpha dropped), scalars and normal maps quantised to 8 bits
    (round(clamp(v, 0, 1) * 255)) and then BC4 / BC5. Sides that are not
    multiples of 4 keep RGBA32F for colour."""
    from . import encode_texture_float

    rgba32f = np.ascontiguousarray(rgba32f, np.float32)
    h, w = rgba32f.shape[:2]
    if usage == "color":
        tex = Texture(TEX_RGBA32F, w, h, rgba32f)
        return tex if (w % 4 or h % 4) else encode_texture_float(TEX_BC6H_UF16, tex)
    q = np.rint(np.clip(rgba32f, 0.0, 1.0) * np.float32(255)).astype(np.uint8)
    return prepared_texture(q, usage, srgb=False)


def _lerp_axis(n: int, cells: int, wrap: bool):
    """Lattice indices and smoothstep weights of n samples over `cells` cells."""
    x = np.arange(n) * cells / n if wrap else np.linspace(0.0, cells, n, endpoint=False) + 0.5 * cells / n
    i0 = np.floor(x).astype(int)
    f = x - i0
    i0 = i0 % cells if wrap else np.minimum(i0, cells - 1)
    i1 = (i0 + 1) % cells if wrap else i0 + 1
    return i0, i1, f * f * (3 - 2 * f)


def _octave(lattice: np.ndarray, n: int, wrap: bool) -> np.ndarray:
    """Separable smoothstep interpolation of a lattice to n x n: along x on
    the lattice rows first, then one row gather along z."""
    cells = lattice.shape[0] - (0 if wrap else 1)
    i0, i1, f = _lerp_axis(n, cells, wrap)
    rows_x = lattice[:, i0] * (1 - f)[None, :] + lattice[:, i1] * f[None, :]
    return rows_x[i0] * (1 - f)[:, None] + rows_x[i1] * f[:, None]


def value_noise(size: int, seed: int, octaves: int = 4, base: int = 8) -> np.ndarray:
    """Seeded tileable value noise in [0, 1], (size, size): smoothstep-
    interpolated lattice values, octaves summed with halving amplitude."""
    rng = np.random.default_rng(seed)
    out = np.zeros((size, size))
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = base << o
        out += amp * _octave(rng.random((cells, cells)), size, True)
        total += amp
        amp *= 0.5
    return out / total


def normal_map_from_height(height: np.ndarray, strength: float = 4.0) -> np.ndarray:
    """Tangent-space normals (x, y in [0, 1] encoding) of a tileable height field."""
    gx = (np.roll(height, -1, 1) - np.roll(height, 1, 1)) * 0.5 * strength
    gy = (np.roll(height, -1, 0) - np.roll(height, 1, 0)) * 0.5 * strength
    n = np.stack([-gx, -gy, np.ones_like(height)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    return n * 0.5 + 0.5


@dataclass
class SceneSpec:
    name: str
    objects: list
    camera: Camera
    environment: Environment
    width: int
    height: int
    spp: int
    max_bounces: int
    delta_lights: list = field(default_factory=list)
    textures: list = field(default_factory=list)

    @property
    def triangle_count(self) -> int:
        return sum(o.mesh.triangle_count for o in self.objects)


def cornell(width=256, height=256, spp=16, max_bounces=8) -> SceneSpec:
    white = matte(acescg((0.73, 0.73, 0.73)))
    red = matte(acescg((0.63, 0.065, 0.05)))
    green = matte(acescg((0.14, 0.45, 0.09)))
    ident = rows(np.eye(4))
    objs = [
        Object(quad([(-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1)]), ident, white),     # floor, +y
        Object(quad([(-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)]), ident, white),     # ceiling, -y
        Object(quad([(-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)]), ident, white),   # back, +z
        Object(quad([(-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1)]), ident, red),     # left, +x
        Object(quad([(1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)]), ident, green),       # right, -x
        Object(box(0.6, 0.6, 0.6), rows(translate(0.33, 0.3, 0.3) @ rotate_y(17.0)), white),
        Object(box(0.6, 1.2, 0.6), rows(translate(-0.33, 0.6, -0.3) @ rotate_y(-18.0)), white),
        Object(quad([(-0.25, 1.999, -0.25), (0.25, 1.999, -0.25), (0.25, 1.999, 0.25), (-0.25, 1.999, 0.25)]),
               ident, emitter(acescg((17.0, 12.0, 4.0)))),
    ]
    cam = Camera((0.0, 1.0, 3.8), (0.0, 1.0, 0.0), vfov_degrees=40.0)
    return SceneSpec("cornell", objs, cam, Environment.constant((0.0, 0.0, 0.0)), width, height, spp, max_bounces)


def sky_hdri(width=2048, height=1024, sun_elevation_deg=35.0, sun_azimuth_deg=30.0, sun_sigma_deg=0.5,
             sun_peak=5.0e4) -> Environment:
    """Gradient sky (0.3, 0.5, 1.0) at the zenith to white at the horizon, a dim
    ground below it, plus a Gaussian sun lobe; texel centres follow the
    equirect mapping of crates/cenote/shaders/environment.slang:74-85."""
    u = (np.arange(width, dtype=np.float64) + 0.5) / width
    v = (np.arange(height, dtype=np.float64) + 0.5) / height
    phi = 2.0 * np.pi * (u - 0.5)
    theta = np.pi * v
    st, ct = np.sin(theta)[:, None], np.cos(theta)[:, None]
    d = np.stack([st * np.sin(phi)[None, :], np.broadcast_to(ct, (height, width)), -st * np.cos(phi)[None, :]], -1)
    y = d[..., 1]
    t = np.sqrt(np.clip(y, 0.0, 1.0))[..., None]
    sky = (1.0 - t) * np.array([1.0, 1.0, 1.0]) + t * np.array([0.3, 0.5, 1.0])
    ground = np.array([0.25, 0.22, 0.2]) * np.clip(1.0 + y, 0.2, 1.0)[..., None]
    rgb = np.where((y >= 0.0)[..., None], sky, ground)
    el, az = math.radians(sun_elevation_deg), math.radians(sun_azimuth_deg)
    sun = np.array([math.cos(el) * math.sin(az), math.sin(el), -math.cos(el) * math.cos(az)])
    ang = np.arccos(np.clip(d @ sun, -1.0, 1.0))
    sig = math.radians(sun_sigma_deg)
    lobe = sun_peak * np.exp(-0.5 * (ang / sig) ** 2)
    rgb = rgb + lobe[..., None] * np.array([1.0, 0.95, 0.85])
    tex = np.empty((height, width, 4), np.float32)
    tex[..., :3] = rgb
    tex[..., 3] = 1.0
    return Environment(width, height, tex)


def chart(width=1280, height=720, spp=64, max_bounces=12, env_size=(2048, 1024)) -> SceneSpec:
    sphere = icosphere(3)
    base = acescg((0.8, 0.35, 0.2))
    objs = []
    for iz in range(5):
        for ix in range(5):
            rough = ix / 4.0
            metalness = iz / 4.0
            m = glossy(base, 0.0, rough)
            m["metalness"] = metalness
            xf = translate((ix - 2) * 1.0, 0.4, (iz - 2) * 1.0) @ scale(0.4)
            objs.append(Object(sphere, rows(xf), m))
    objs.append(Object(ground_plane(10.0), rows(np.eye(4)), glossy(acescg((0.5, 0.5, 0.5)), 0.0, 0.3)))
    light = quad([(-0.5, 0, -0.5), (0.5, 0, -0.5), (0.5, 0, 0.5), (-0.5, 0, 0.5)])  # faces -y
    objs.append(Object(light, rows(translate(1.5, 3.0, 1.5) @ rotate_x(-20.0)), emitter(acescg((8.0, 6.0, 4.0)))))
    cam = Camera((0.0, 2.6, 5.8), (0.0, 0.35, 0.0), vfov_degrees=40.0)
    return SceneSpec("chart", objs, cam, sky_hdri(*env_size), width, height, spp, max_bounces)


def furnace(mat, size=32, sky=0.5, center=(0.0, 0.0, 0.0), scl=1.0, aperture=0.0, focus=1.0) -> SceneSpec:
    """One large plane under a uniform grey sky, camera just above it looking
    obliquely down (render/tests.rs:51-84)."""
    c = np.asarray(center, np.float64)
    obj = Object(ground_plane(5.0), rows(translate(*c) @ scale(scl)), mat)
    cam = Camera(tuple(c + (0.0, scl, 0.0)), tuple(c + (0.0, 0.0, -scl)), vfov_degrees=40.0,
                 aperture_radius=aperture, focus_distance=focus)
    return SceneSpec("furnace", [obj], cam, Environment.constant((sky, sky, sky)), size, size, 16, 8)


SCENES = {"cornell": cornell, "chart": chart}


# ---- flat archive -----------------------------------------------------------------


def save_spec(path, spec: SceneSpec, **extra) -> None:
    """Store a scene description as one .npz: meshes, transforms, materials,
    camera, environment, delta lights and settings. `extra` arrays ride along."""
    arrs = {}
    for i, o in enumerate(spec.objects):
        m = o.mesh
        arrs.update({f"o{i}_positions": m.positions, f"o{i}_normals": m.normals, f"o{i}_uvs": m.uvs,
                     f"o{i}_indices": m.indices, f"o{i}_transform": np.asarray(o.transform, np.float32),
                     f"o{i}_material": np.frombuffer(np.asarray(o.material, MATERIAL_DTYPE).tobytes(), np.uint8),
                     f"o{i}_visible": np.array(o.camera_visible)})
    c = spec.camera
    arrs["camera"] = np.array([*c.position, *c.look_at, *c.up, c.vfov_degrees, c.aperture_radius,
                               c.focus_distance], np.float64)
    arrs["env"] = np.asarray(spec.environment.texels, np.float32)
    arrs["delta"] = np.array([[d.kind, *d.anchor, *d.emission] for d in spec.delta_lights], np.float64).reshape(-1, 7)
    arrs["settings"] = np.array([spec.width, spec.height, spec.spp, spec.max_bounces, len(spec.objects)], np.int64)
    arrs["name"] = np.array(spec.name)
    for k, t in enumerate(spec.textures):
        arrs[f"t{k}_shape"] = np.array([t.format, t.width, t.height], np.int64)
        arrs[f"t{k}_data"] = np.asarray(t.data)
    arrs.update({f"x_{k}": np.asarray(v) for k, v in extra.items()})
    np.savez_compressed(path, **arrs)


def load_spec(path) -> tuple[SceneSpec, dict]:
    """Inverse of save_spec: the scene and the extra arrays stored with it."""
    z = np.load(path)
    w, h, spp, mb, n = (int(v) for v in z["settings"])
    objs = []
    for i in range(n):
        mesh = Mesh(z[f"o{i}_positions"], z[f"o{i}_normals"], z[f"o{i}_uvs"], z[f"o{i}_indices"])
        mat = np.frombuffer(z[f"o{i}_material"].tobytes(), MATERIAL_DTYPE)[0]
        objs.append(Object(mesh, z[f"o{i}_transform"], mat, bool(z[f"o{i}_visible"])))
    c = z["camera"]
    cam = Camera(tuple(c[0:3]), tuple(c[3:6]), tuple(c[6:9]), float(c[9]), float(c[10]), float(c[11]))
    env = z["env"]
    deltas = [DeltaLight(int(d[0]), tuple(d[1:4]), tuple(d[4:7])) for d in z["delta"]]
    textures = []
    while f"t{len(textures)}_shape" in z.files:
        k = len(textures)
        fmt, tw, th = (int(v) for v in z[f"t{k}_shape"])
        textures.append(Texture(fmt, tw, th, z[f"t{k}_data"]))
    spec = SceneSpec(str(z["name"]), objs, cam, Environment(env.shape[1], env.shape[0], env), w, h, spp, mb, deltas,
                     textures)
    return spec, {k[2:]: z[k] for k in z.files if k.startswith("x_")}


def textured(width=160, height=90, spp=8, max_bounces=6, size=64, seed=7, color_format=TEX_BC1_SRGB,
             float_format=TEX_RGBA32F) -> SceneSpec:
    """Every texture slot and format on one small set: a ground tiled 4x with a
    base colour in `color_format` (BC1 or BC7 sRGB), a BC5 normal map and a BC4 roughness map; a metal
    panel with an RGBA8 metalness map; a leaf quad cut out by a BC4 opacity
    map; a ceiling emitter whose emission an RGBA8 sRGB map modulates; a
    float base colour on a back wall (`float_format`: RGBA32F or BC6H). Textures are seeded value noise."""
    from . import encode_texture  # host BC encoder of the library

    noise = [value_noise(size, seed + k) for k in range(6)]
    col = np.stack([0.2 + 0.7 * noise[0], 0.2 + 0.6 * noise[1], 0.1 + 0.5 * noise[0] * noise[2]], -1)
    textures = [
        encode_texture(color_format, rgba8_texture(col, srgb=True)),                                 # 0 base colour
        encode_texture(TEX_BC5_UNORM, rgba8_texture(normal_map_from_height(noise[3], 6.0), False)),  # 1 normal
        encode_texture(TEX_BC4_UNORM, rgba8_texture(np.repeat(0.15 + 0.8 * noise[4][..., None], 3, -1), False)),
        rgba8_texture(np.repeat((noise[5] > 0.5)[..., None].astype(float), 3, -1), srgb=False),       # 3 metalness
        encode_texture(TEX_BC4_UNORM, rgba8_texture(np.repeat((noise[2] > 0.45)[..., None].astype(float), 3, -1),
                                                    False)),                                          # 4 opacity
        rgba8_texture(np.stack([np.linspace(0.2, 1, size)[None, :].repeat(size, 0)] * 3, -1), srgb=True),  # 5 emission
        Texture(TEX_RGBA32F, 8, 8, np.ascontiguousarray(
            np.concatenate([np.random.default_rng(seed).random((8, 8, 3)), np.ones((8, 8, 1))], -1), np.float32)),
    ]
    if float_format == TEX_BC6H_UF16:  # the back wall's float colour as BC6H, as texture prep stores HDR colour
        from . import encode_texture_float

        textures[-1] = encode_texture_float(TEX_BC6H_UF16, textures[-1])
    ident = rows(np.eye(4))
    tiled = np.array([[0, 0], [0, 4], [4, 4], [4, 0]], np.float32)
    ground = material(base_color=(0.8, 0.8, 0.8), specular_weight=1.0, specular_roughness=0.5)
    ground["base_color_texture"], ground["normal_texture"], ground["specular_roughness_texture"] = 0, 1, 2
    panel = metal(acescg((0.9, 0.7, 0.5)), 0.25)
    panel["metalness_texture"] = 3
    leaf = matte(acescg((0.3, 0.6, 0.2)))
    leaf["opacity_texture"] = 4
    lamp = emitter(acescg((6.0, 5.0, 4.0)))
    lamp["emission_texture"] = 5
    wall = matte(acescg((1.0, 1.0, 1.0)))
    wall["base_color_texture"] = 6
    objs = [
        Object(quad([(-3, 0, -3), (-3, 0, 3), (3, 0, 3), (3, 0, -3)], uvs=tiled), ident, ground),
        Object(quad([(-1.6, 0, -1.0), (-0.4, 0, -1.4), (-0.4, 1.2, -1.4), (-1.6, 1.2, -1.0)]), ident, panel),
        Object(quad([(0.2, 0.1, 0.2), (1.4, 0.1, 0.2), (1.4, 1.3, -0.2), (0.2, 1.3, -0.2)]), ident, leaf),
        Object(quad([(-0.8, 2.5, -0.8), (0.8, 2.5, -0.8), (0.8, 2.5, 0.8), (-0.8, 2.5, 0.8)]), ident, lamp),
        Object(quad([(-3, 0, -2.5), (3, 0, -2.5), (3, 3, -2.5), (-3, 3, -2.5)]), ident, wall),
    ]
    cam = Camera((0.0, 1.4, 4.0), (0.0, 0.6, 0.0), vfov_degrees=45.0)
    return SceneSpec("textured", objs, cam, Environment.constant((0.15, 0.18, 0.25)), width, height, spp,
                     max_bounces, textures=textures)


# ---- the large scene --------------------------------------------------------------


def fbm_heightfield(n: int, seed: int, octaves: int = 6) -> np.ndarray:
    """Seeded fBm (value noise, lacunarity 2, gain 0.5) on an n x n grid, in [0, 1]."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, n))
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = 4 << o
        out += amp * _octave(rng.random((cells + 1, cells + 1)), n, False)
        total += amp
        amp *= 0.5
    return out / total


def grid_mesh(heights: np.ndarray, x0: float, z0: float, cell: float, uv_scale: float) -> Mesh:
    """A heightfield patch: vertices at (x0 + j·cell, h[i, j], z0 + i·cell),
    two triangles per cell wound upward, smooth normals from central differences."""
    h = np.asarray(heights, np.float64)
    r, c = h.shape
    jj, ii = np.meshgrid(np.arange(c), np.arange(r))
    pos = np.stack([x0 + jj * cell, h, z0 + ii * cell], -1).reshape(-1, 3)
    gx = np.gradient(h, cell, axis=1)
    gz = np.gradient(h, cell, axis=0)
    n = np.stack([-gx, np.ones_like(h), -gz], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    uv = np.stack([jj / (c - 1), ii / (r - 1)], -1).reshape(-1, 2) * uv_scale
    a = (ii[:-1, :-1] * c + jj[:-1, :-1]).reshape(-1)
    tris = np.concatenate([np.stack([a, a + c, a + 1], -1), np.stack([a + 1, a + c, a + c + 1], -1)])
    return _mesh(pos, n.reshape(-1, 3), uv, tris)


def torus(major: float, minor: float, nu: int = 32, nv: int = 32) -> Mesh:
    u = np.arange(nu) * 2 * np.pi / nu
    v = np.arange(nv) * 2 * np.pi / nv
    uu, vv = np.meshgrid(u, v, indexing="ij")
    cx, cz = np.cos(uu), np.sin(uu)
    pos = np.stack([(major + minor * np.cos(vv)) * cx, minor * np.sin(vv), (major + minor * np.cos(vv)) * cz], -1)
    nrm = np.stack([np.cos(vv) * cx, np.sin(vv), np.cos(vv) * cz], -1)
    uv = np.stack([uu / (2 * np.pi), vv / (2 * np.pi)], -1)
    i, j = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    a = (i * nv + j).reshape(-1)
    b = (((i + 1) % nu) * nv + j).reshape(-1)
    c = (i * nv + (j + 1) % nv).reshape(-1)
    d = (((i + 1) % nu) * nv + (j + 1) % nv).reshape(-1)
    tris = np.concatenate([np.stack([a, c, b], -1), np.stack([b, c, d], -1)])
    return _mesh(pos.reshape(-1, 3), nrm.reshape(-1, 3), uv.reshape(-1, 2), tris)


def uv_sphere(rings: int = 16, segments: int = 64) -> Mesh:
    """Unit UV sphere, 2·rings·segments − 2·segments triangles."""
    th = np.arange(rings + 1) * np.pi / rings
    ph = np.arange(segments + 1) * 2 * np.pi / segments
    t, p = np.meshgrid(th, ph, indexing="ij")
    n = np.stack([np.sin(t) * np.cos(p), np.cos(t), np.sin(t) * np.sin(p)], -1).reshape(-1, 3)
    uv = np.stack([p / (2 * np.pi), t / np.pi], -1).reshape(-1, 2)
    row = segments + 1
    tris = []
    for r in range(rings):
        for s in range(segments):
            a = r * row + s
            b = a + row
            if r != 0:
                tris.append((a, a + 1, b))
            if r != rings - 1:
                tris.append((a + 1, b + 1, b))
    return _mesh(n, n.copy(), uv, np.asarray(tris))


def superquadric(e: float = 0.3, rings: int = 16, segments: int = 64) -> Mesh:
    """A rounded box (superellipsoid with exponent e), 1,920 triangles by default."""
    sph = uv_sphere(rings, segments)
    p = sph.positions.astype(np.float64)
    q = np.sign(p) * np.abs(p) ** e
    return _mesh(q, derive_flat_normals(q, sph.indices), sph.uvs, sph.indices)


def derive_flat_normals(p, idx):
    face = np.cross(p[idx[:, 1]] - p[idx[:, 0]], p[idx[:, 2]] - p[idx[:, 0]])
    n = np.zeros_like(p)
    for k in range(3):
        np.add.at(n, idx[:, k], face)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    return np.where(ln > 0, n / np.maximum(ln, 1e-30), [0.0, 1.0, 0.0])


def large(width=1920, height=1080, spp=64, max_bounces=16, grid=1024, instances=500, emitters=4096,
          texture_size=1024, textures=128, seed=1) -> SceneSpec:
    """The large scene: an fBm terrain of (grid−1)²·2 triangles (1024² grid:
    2.09 M) in 8×8 tiles, each with its own BC1 base-colour and BC5 normal map
    (128 seeded value-noise textures of texture_size²); `instances` copies of
    three ~2k-triangle meshes — glass (IOR 1.5, absorption 0.2 per unit), a
    clear-coated torus and a fuzz-covered rounded box — placed on the terrain;
    `emitters` small emissive triangles whose powers are lognormal(0, 2); a
    procedural sun-and-sky environment."""
    from . import encode_texture

    rng = np.random.default_rng(seed)
    extent = 200.0
    cell = extent / (grid - 1)
    hf = fbm_heightfield(grid, seed) * 18.0
    tiles = 8
    per = (grid - 1) // tiles
    objs, texs = [], []
    ident = rows(np.eye(4))
    for k in range(textures // 2):
        col_noise = value_noise(texture_size, seed * 1000 + 2 * k, octaves=5, base=8)
        hue = rng.random(3) * 0.4 + np.array([0.25, 0.25, 0.15])
        col = np.clip(hue[None, None, :] * (0.5 + col_noise[..., None]), 0, 1)
        texs.append(encode_texture(TEX_BC1_SRGB, rgba8_texture(col, srgb=True)))
        bump = value_noise(texture_size, seed * 1000 + 2 * k + 1, octaves=5, base=16)
        texs.append(encode_texture(TEX_BC5_UNORM, rgba8_texture(normal_map_from_height(bump, 8.0), srgb=False)))
    for ti in range(tiles):
        for tj in range(tiles):
            r0, c0 = ti * per, tj * per
            r1 = grid - 1 if ti == tiles - 1 else r0 + per
            c1 = grid - 1 if tj == tiles - 1 else c0 + per
            patch = hf[r0:r1 + 1, c0:c1 + 1]
            mesh = grid_mesh(patch, -extent / 2 + c0 * cell, -extent / 2 + r0 * cell, cell, 8.0)
            t = (ti * tiles + tj) % (textures // 2)
            m = material(base_color=(1.0, 1.0, 1.0), specular_weight=1.0, specular_roughness=0.6)
            m["base_color_texture"], m["normal_texture"] = 2 * t, 2 * t + 1
            objs.append(Object(mesh, ident, m))

    def height_at(x, z):
        j = int(np.clip((x + extent / 2) / cell, 0, grid - 1))
        i = int(np.clip((z + extent / 2) / cell, 0, grid - 1))
        return float(hf[i, j])

    glass = material(base_color=(1.0, 1.0, 1.0), specular_weight=1.0, specular_roughness=0.0, specular_ior=1.5,
                     transmission_weight=1.0, transmission_color=np.exp(-0.2) * np.ones(3), transmission_depth=1.0)
    coated = material(base_color=acescg((0.6, 0.1, 0.08)), specular_weight=1.0, specular_roughness=0.4,
                      coat_weight=1.0, coat_roughness=0.05, coat_ior=1.5)
    fuzzy = material(base_color=acescg((0.2, 0.3, 0.6)), specular_weight=0.5, specular_roughness=0.5,
                     fuzz_weight=1.0, fuzz_color=(1.0, 0.9, 0.8), fuzz_roughness=0.5)
    shapes = [(uv_sphere(16, 64), glass), (torus(1.0, 0.35, 32, 32), coated), (superquadric(0.35), fuzzy)]
    span = extent * 0.35
    for k in range(instances):
        mesh, mat = shapes[k % 3]
        x, z = rng.uniform(-span, span, 2)
        s = rng.uniform(0.8, 2.5)
        rot = rotate_y(rng.uniform(0, 360))
        objs.append(Object(mesh, rows(translate(x, height_at(x, z) + s, z) @ rot @ scale(s)), mat))
    powers = rng.lognormal(0.0, 2.0, emitters)
    for k in range(emitters):
        x, z = rng.uniform(-span, span, 2)
        y = height_at(x, z) + rng.uniform(3.0, 12.0)
        a = rng.uniform(0, 2 * np.pi)
        size = 0.35
        p0 = np.array([x, y, z])
        p1 = p0 + size * np.array([np.cos(a), 0.0, np.sin(a)])
        p2 = p0 + size * np.array([np.cos(a + 2.0), -0.3, np.sin(a + 2.0)])
        tri = _mesh([p0, p1, p2], [np.cross(p1 - p0, p2 - p0) / np.linalg.norm(np.cross(p1 - p0, p2 - p0))] * 3,
                    [[0, 0], [1, 0], [0, 1]], [[0, 1, 2]])
        objs.append(Object(tri, ident, emitter(acescg((1.0, 0.85, 0.6)) * np.float32(powers[k] * 4.0))))
    look = np.array([0.0, height_at(0.0, 0.0) + 2.0, 0.0])
    eye = look + np.array([0.0, 28.0, 75.0])
    cam = Camera(tuple(eye), tuple(look), vfov_degrees=45.0)
    env = sky_hdri(1024, 512, sun_elevation_deg=25.0)
    return SceneSpec("large", objs, cam, env, width, height, spp, max_bounces, textures=texs)


def ceiling_box(width=256, height=256, spp=16, max_bounces=8) -> SceneSpec:
    """The closed box with its emitter turned to face the ceiling, 0.4 below
    it: light reaches the room only by a bounce off the ceiling, so next-event
    estimation from most surfaces finds the lamp's back face and the
    directional distribution of incident light is sharply peaked."""
    spec = cornell(width, height, spp, max_bounces)
    lamp = spec.objects[-1]
    q = quad([(-0.25, 1.6, -0.25), (-0.25, 1.6, 0.25), (0.25, 1.6, 0.25), (0.25, 1.6, -0.25)])
    spec.objects[-1] = Object(q, lamp.transform, lamp.material)
    spec.name = "ceiling_box"
    return spec


SCENES.update(textured=textured, large=large, ceiling_box=ceiling_box)
