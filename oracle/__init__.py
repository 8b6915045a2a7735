"""CPU oracle — test infrastructure only.

A C++ restatement of cenote's path-tracing hot path (crates/cenote/shaders/*.slang
and the host tables in crates/cenote/src/{lights,environment,tables,color}.rs),
compiled from oracle/*.cpp into oracle/_build/liboracle.so and called through
ctypes. Only the tests, the smoke check and bench.py's CPU-baseline leg use it,
as the checker; the shipped library never imports, links or runs it.

Parity pins: every host table is checked against the reference's own tests
(lights.rs:320-475, environment.rs:258-324, color.rs:39-59), restated in
tests/test_oracle_golden.py. The reference cannot be run here (Rust + Vulkan; no
cargo, slangc or Vulkan device on this machine or the GPU box), but it commits
its own 64-spp renders of two pbrt scenes
(crates/cenote-pbrt/tests/golden/{cornell-box,veach-mis}.exr): imported with
cenote_b200.pbrt and rendered here with the same Sobol-Burley samples, the
oracle reproduces those pixels' noise (tests/test_corpus.py), which pins the
image path to reference pixels, alongside the reference's physical tests
(furnaces, analytic lights, MIS agreement).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
TABLES = None
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def library() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    lib = C.CDLL(str(LIB_PATH))
    P, U32, F, D = C.c_void_p, C.c_uint32, C.c_float, C.c_double
    sig = {
        "oracle_scene_create": (P, [P, U32, P, U32, U32, P, P, U32, P, P, U32]),
        "oracle_scene_destroy": (None, [P]),
        "oracle_scene_light_count": (U32, [P]),
        "oracle_scene_lights": (None, [P, P]),
        "oracle_scene_select_prob": (F, [P]),
        "oracle_scene_env_power": (D, [P]),
        "oracle_scene_env_tables": (None, [P, P, P, P]),
        "oracle_texture_decode": (C.c_int, [U32, U32, U32, P, P]),
        "oracle_texture_sample": (C.c_int, [U32, U32, U32, P, U32, P, U32, P]),
        "oracle_render": (None, [P, U32, U32, U32, U32, U32, U32, U32, P, P, P, P, P]),
        "oracle_camera_basis": (None, [P, F, P, P, P]),
        "oracle_sampler": (None, [U32, U32, U32, P, P]),
        "oracle_hash_uniform": (F, [U32, U32, U32, U32]),
        "oracle_bsdf_eval": (None, [P, P, P, P, U32, U32, P, P]),
        "oracle_bsdf_sample": (None, [P, P, P, P, U32, U32, P, P, P]),
        "oracle_build_lights": (U32, [P, P, P, U32, P, U32, P, P]),
        "oracle_env_tables": (None, [U32, U32, P, P, P, P, P]),
        "oracle_env_sample": (None, [P, P, U32, P, P, P]),
        "oracle_env_pdf": (None, [P, P, U32, P]),
        "oracle_intersect": (None, [P, P, P, U32, P, P]),
        "oracle_shadow": (None, [P, P, P, P, P, U32, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def bsdf_tables() -> np.ndarray:
    """The 16,928-float table buffer (ggx_energy.bin ++ ltc_sheen.bin)."""
    global TABLES
    if TABLES is None:
        data = HERE.parent / "cenote_b200" / "data"
        TABLES = np.concatenate([np.fromfile(data / "ggx_energy.bin", "<f4"),
                                 np.fromfile(data / "ltc_sheen.bin", "<f4")]).astype(np.float32)
        assert TABLES.size == 16928
    return TABLES


def _p(a):
    return a.ctypes.data


class _Object(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("normals", C.c_void_p), ("uvs", C.c_void_p), ("indices", C.c_void_p),
                ("vertex_count", C.c_uint32), ("triangle_count", C.c_uint32), ("transform", C.c_float * 12),
                ("material", C.c_uint8 * 144), ("camera_visible", C.c_uint32), ("pad", C.c_uint32)]


class _Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3),
                ("vfov_degrees", C.c_float), ("aperture_radius", C.c_float), ("focus_distance", C.c_float)]


class _Delta(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("anchor", C.c_float * 3), ("emission", C.c_float * 3)]


LIGHT_RECORD_DTYPE = np.dtype([
    ("anchor", "<f4", 3), ("pdf", "<f4"), ("edge1", "<f4", 3), ("alias_threshold", "<f4"), ("edge2", "<f4", 3),
    ("alias_index", "<u4"), ("emission", "<f4", 3), ("instance", "<u4"), ("kind", "<u4"), ("primitive", "<u4"),
    ("pad", "<u4", 2),
])


def _camera(cam) -> _Camera:
    c = _Camera()
    c.position[:] = [float(v) for v in cam.position]
    c.look_at[:] = [float(v) for v in cam.look_at]
    c.up[:] = [float(v) for v in cam.up]
    c.vfov_degrees = cam.vfov_degrees
    c.aperture_radius = cam.aperture_radius
    c.focus_distance = cam.focus_distance
    return c


def texture_decode(tex) -> np.ndarray:
    """Linear RGBA float texels (H, W, 4) of a scenes.Texture."""
    out = np.zeros((tex.height, tex.width, 4), np.float32)
    data = np.ascontiguousarray(tex.data)
    if library().oracle_texture_decode(tex.format, tex.width, tex.height, _p(data), _p(out)) != 0:
        raise ValueError("texture the oracle cannot decode")
    return out


def texture_sample(tex, uv, mode=0) -> np.ndarray:
    u = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    out = np.zeros((len(u), 4), np.float32)
    data = np.ascontiguousarray(tex.data)
    if library().oracle_texture_sample(tex.format, tex.width, tex.height, _p(data), mode, _p(u), len(u), _p(out)) != 0:
        raise ValueError("texture the oracle cannot decode")
    return out


class _Texture(C.Structure):
    _fields_ = [("format", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32), ("pad", C.c_uint32),
                ("data", C.c_void_p)]


class OracleScene:
    def __init__(self, spec):
        lib = library()
        self.spec = spec
        keep = []
        objs = (_Object * len(spec.objects))()
        for i, o in enumerate(spec.objects):
            arrs = [np.ascontiguousarray(a) for a in (o.mesh.positions, o.mesh.normals, o.mesh.uvs, o.mesh.indices)]
            keep += arrs
            objs[i].positions, objs[i].normals, objs[i].uvs, objs[i].indices = [_p(a) for a in arrs]
            objs[i].vertex_count = len(o.mesh.positions)
            objs[i].triangle_count = len(o.mesh.indices)
            objs[i].transform[:] = [float(v) for v in np.asarray(o.transform, np.float32)]
            C.memmove(objs[i].material, np.asarray(o.material).tobytes(), 144)
            objs[i].camera_visible = 1 if o.camera_visible else 0
        cam = _camera(spec.camera)
        env = spec.environment
        tex = np.ascontiguousarray(env.texels, np.float32)
        deltas = (_Delta * max(1, len(spec.delta_lights)))()
        for i, d in enumerate(spec.delta_lights):
            deltas[i].kind = d.kind
            deltas[i].anchor[:] = list(d.anchor)
            deltas[i].emission[:] = list(d.emission)
        tables = bsdf_tables()
        textures = getattr(spec, "textures", [])
        texs = (_Texture * max(1, len(textures)))()
        for k, t in enumerate(textures):
            data = np.ascontiguousarray(t.data)
            keep.append(data)
            texs[k].format, texs[k].width, texs[k].height = t.format, t.width, t.height
            texs[k].data = _p(data)
        self._h = lib.oracle_scene_create(objs, len(spec.objects), C.byref(cam), env.width, env.height, _p(tex), deltas,
                                          len(spec.delta_lights), _p(tables), texs, len(textures))
        if not self._h:
            raise ValueError("the oracle rejected the scene: a texture it cannot decode or a slot past the table")

    def render_sum(self, width, height, sample_begin, sample_count, max_bounces, light_sampling=0, threads=0,
                   out=None):
        import os
        if out is None:
            out = np.zeros((height, width, 4), np.float32)
        counts = np.zeros(2, np.uint64)
        threads = threads or os.cpu_count() or 1
        library().oracle_render(self._h, width, height, sample_begin, sample_count, max_bounces, light_sampling,
                                threads, _p(out), _p(counts), None, None, None)
        self.last_ray_counts = counts
        return out

    def render_guides(self, width, height, sample_begin, sample_count, max_bounces, light_sampling=0, threads=0):
        """Beauty and guide sums: dict of beauty/albedo/normal (H, W, 4) and depth (H, W)."""
        import os
        out = {k: np.zeros((height, width, 4), np.float32) for k in ("beauty", "albedo", "normal")}
        out["depth"] = np.zeros((height, width), np.float32)
        counts = np.zeros(2, np.uint64)
        threads = threads or os.cpu_count() or 1
        library().oracle_render(self._h, width, height, sample_begin, sample_count, max_bounces, light_sampling,
                                threads, _p(out["beauty"]), _p(counts), _p(out["albedo"]), _p(out["normal"]),
                                _p(out["depth"]))
        self.last_ray_counts = counts
        return out

    def lights(self) -> np.ndarray:
        n = library().oracle_scene_light_count(self._h)
        out = np.zeros(n, LIGHT_RECORD_DTYPE)
        if n:
            library().oracle_scene_lights(self._h, _p(out))
        return out

    def select_prob(self) -> float:
        return float(library().oracle_scene_select_prob(self._h))

    def env_power(self) -> float:
        return float(library().oracle_scene_env_power(self._h))

    def env_tables(self):
        env = self.spec.environment
        w, h = env.width, env.height
        m = np.zeros(h + 1, np.float32)
        c = np.zeros(h * (w + 1), np.float32)
        p = np.zeros(h * w, np.float32)
        library().oracle_scene_env_tables(self._h, _p(m), _p(c), _p(p))
        return m, c, p

    def env_sample(self, u):
        u = np.ascontiguousarray(u, np.float32)
        n = len(u)
        d = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        rc = np.zeros((n, 2), np.uint32)
        library().oracle_env_sample(self._h, _p(u), n, _p(d), _p(pdf), _p(rc))
        return d, pdf, rc

    def env_pdf(self, dirs):
        d = np.ascontiguousarray(dirs, np.float32)
        out = np.zeros(len(d), np.float32)
        library().oracle_env_pdf(self._h, _p(d), len(d), _p(out))
        return out

    def intersect(self, origins, directions):
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(directions, np.float32)
        n = len(o)
        hits = np.zeros((n, 4), np.uint32)
        t = np.zeros(n, np.float32)
        library().oracle_intersect(self._h, _p(o), _p(d), n, _p(hits), _p(t))
        return hits, t

    def shadow(self, origins, directions, tmax, targets):
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(directions, np.float32)
        tm = np.ascontiguousarray(tmax, np.float32)
        tg = np.ascontiguousarray(targets, np.uint32)
        out = np.zeros(len(o), np.float32)
        library().oracle_shadow(self._h, _p(o), _p(d), _p(tm), _p(tg), len(o), _p(out))
        return out

    def close(self):
        if getattr(self, "_h", None):
            library().oracle_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def camera_basis(cam, aspect):
    r = np.zeros(3, np.float32)
    u = np.zeros(3, np.float32)
    f = np.zeros(3, np.float32)
    c = _camera(cam)
    library().oracle_camera_basis(C.byref(c), aspect, _p(r), _p(u), _p(f))
    return r, u, f


def sampler(pixel, dimension, count):
    pts = np.zeros((count, 2), np.float32)
    vals = np.zeros(count, np.float32)
    library().oracle_sampler(pixel, dimension, count, _p(pts), _p(vals))
    return pts, vals


def hash_uniform(pixel, sample, bounce, crossing):
    return float(library().oracle_hash_uniform(pixel, sample, bounce, crossing))


def bsdf_eval(material, wo, wi, exiting=False):
    wo = np.ascontiguousarray(wo, np.float32)
    wi = np.ascontiguousarray(wi, np.float32)
    n = len(wo)
    f = np.zeros((n, 3), np.float64)
    pdf = np.zeros(n, np.float64)
    m = np.ascontiguousarray(np.asarray(material))
    library().oracle_bsdf_eval(_p(m), _p(bsdf_tables()), _p(wo), _p(wi), n, int(exiting), _p(f), _p(pdf))
    return f, pdf


def bsdf_sample(material, wo, u, exiting=False):
    wo = np.ascontiguousarray(wo, np.float32)
    u = np.ascontiguousarray(u, np.float32)
    n = len(wo)
    wi = np.zeros((n, 3), np.float64)
    pdf = np.zeros(n, np.float64)
    lobe = np.zeros(n, np.uint32)
    m = np.ascontiguousarray(np.asarray(material))
    library().oracle_bsdf_sample(_p(m), _p(bsdf_tables()), _p(wo), _p(u), n, int(exiting), _p(wi), _p(pdf), _p(lobe))
    return wi, pdf, lobe


def build_lights(triangles, deltas=()):
    """triangles: list of (corners (3,3), emission (3,), instance, primitive);
    deltas: list of (kind, anchor, emission). Returns (records, total_power)."""
    n = len(triangles)
    corners = np.zeros((max(n, 1), 9), np.float32)
    em = np.zeros((max(n, 1), 3), np.float32)
    ids = np.zeros((max(n, 1), 2), np.uint32)
    for i, (c, e, inst, prim) in enumerate(triangles):
        corners[i] = np.asarray(c, np.float32).reshape(9)
        em[i] = e
        ids[i] = (inst, prim)
    d = (_Delta * max(1, len(deltas)))()
    for i, (kind, anchor, emission) in enumerate(deltas):
        d[i].kind = kind
        d[i].anchor[:] = list(anchor)
        d[i].emission[:] = list(emission)
    out = np.zeros(n + len(deltas), LIGHT_RECORD_DTYPE)
    total = C.c_double()
    library().oracle_build_lights(_p(corners), _p(em), _p(ids), n, d, len(deltas), _p(out) if len(out) else None,
                                  C.byref(total))
    return out, total.value


def env_tables(width, height, texels):
    t = np.ascontiguousarray(texels, np.float32)
    m = np.zeros(height + 1, np.float32)
    c = np.zeros(height * (width + 1), np.float32)
    p = np.zeros(height * width, np.float32)
    power = C.c_double()
    library().oracle_env_tables(width, height, _p(t), _p(m), _p(c), _p(p), C.byref(power))
    return m, c, p, power.value
