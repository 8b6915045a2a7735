"""cenote_b200 — a B200-native wavefront path tracer behind cenote's scene/renderer API.

Python binds the C ABI in ``include/cenote_c.h`` (``libcenote_b200.so``, built
in-tree by ``cenote_b200.build``) through ctypes. The classes mirror the
reference crate's types:

    Context          crates/cenote/src/gpu/mod.rs:93          (Context::new)
    Scene            crates/cenote/src/scene/mod.rs:254       (Scene::new)
    Renderer         crates/cenote/src/render/mod.rs:151-311  (with_max_bounces, render, accumulate)
    Film             crates/cenote/src/render/film.rs:102-217 (new, reset, samples, averages)

Errors surface as ``CenoteError`` carrying the library's status code (the
reference's ``cenote::Error`` variants, crates/cenote/src/error.rs:10-72). There
is no fallback: without the built library or a capable GPU every entry point
raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import scenes
from .scenes import SceneSpec

__all__ = ["CenoteError", "Context", "Scene", "Renderer", "Film", "library", "scenes", "LIGHT_SAMPLING_MIS",
           "LIGHT_SAMPLING_BSDF", "LIGHT_SAMPLING_NEE", "EXPORTED_SYMBOLS"]

LIGHT_SAMPLING_MIS, LIGHT_SAMPLING_BSDF, LIGHT_SAMPLING_NEE = 0, 1, 2
# CENOTE_B200_LIB selects another build of the same library (tuning variants).
LIB_PATH = Path(os.environ.get("CENOTE_B200_LIB", Path(__file__).resolve().parent / "libcenote_b200.so"))

STATUS = {
    0: "ok", -1: "invalid argument", -2: "device error", -3: "no capable GPU", -4: "allocation failed",
    -5: "scene error", -6: "timeout", -7: "device bound exceeded", -8: "over budget",
}


class CenoteError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, 'error')} ({code}): {message}")
        self.code = code


class Material(C.Structure):
    _fields_ = [
        ("base_color", C.c_float * 3), ("base_roughness", C.c_float), ("emission", C.c_float * 3),
        ("metalness", C.c_float), ("specular_weight", C.c_float), ("specular_roughness", C.c_float),
        ("specular_ior", C.c_float), ("transmission_weight", C.c_float), ("transmission_color", C.c_float * 3),
        ("transmission_depth", C.c_float), ("coat_color", C.c_float * 3), ("coat_weight", C.c_float),
        ("coat_roughness", C.c_float), ("coat_ior", C.c_float), ("coat_darkening", C.c_float),
        ("fuzz_weight", C.c_float), ("fuzz_color", C.c_float * 3), ("fuzz_roughness", C.c_float),
        ("opacity", C.c_float), ("thin_walled", C.c_uint32), ("base_color_texture", C.c_uint32),
        ("specular_roughness_texture", C.c_uint32), ("metalness_texture", C.c_uint32),
        ("emission_texture", C.c_uint32), ("opacity_texture", C.c_uint32), ("normal_texture", C.c_uint32),
    ]


assert C.sizeof(Material) == 144


class Object(C.Structure):
    _fields_ = [
        ("positions", C.c_void_p), ("normals", C.c_void_p), ("uvs", C.c_void_p), ("indices", C.c_void_p),
        ("vertex_count", C.c_uint32), ("triangle_count", C.c_uint32), ("transform", C.c_float * 12),
        ("material", Material), ("camera_visible", C.c_uint32), ("pad", C.c_uint32),
    ]


class CameraC(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3),
                ("vfov_degrees", C.c_float), ("aperture_radius", C.c_float), ("focus_distance", C.c_float)]


class EnvironmentC(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("texels", C.c_void_p)]


class DeltaLightC(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("anchor", C.c_float * 3), ("emission", C.c_float * 3)]


class TuningC(C.Structure):
    _fields_ = [("material_sort", C.c_uint32), ("samples_per_wave", C.c_uint32), ("refill_idle", C.c_uint32),
                ("top_nodes", C.c_uint32), ("l2_window", C.c_uint32), ("per_lane_triangles", C.c_uint32),
                ("ms_per_sample", C.c_float), ("block_size", C.c_uint32), ("stack_depth", C.c_uint32),
                ("sort_by_location", C.c_uint32)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("samples", C.c_uint64),
                ("node_visits", C.c_uint64), ("triangle_tests", C.c_uint64), ("gpu_ms", C.c_float),
                ("raygen_ms", C.c_float), ("intersect_ms", C.c_float), ("shade_ms", C.c_float),
                ("shadow_ms", C.c_float), ("film_ms", C.c_float), ("kernel_launches", C.c_uint32),
                ("waves", C.c_uint32), ("samples_per_wave", C.c_uint32), ("overflow", C.c_uint32),
                ("surface_hits", C.c_uint64)]


PROFILE_TIMING, PROFILE_COUNTS = 1, 2


LIGHT_RECORD_DTYPE = np.dtype([
    ("anchor", "<f4", 3), ("pdf", "<f4"), ("edge1", "<f4", 3), ("alias_threshold", "<f4"), ("edge2", "<f4", 3),
    ("alias_index", "<u4"), ("emission", "<f4", 3), ("instance", "<u4"), ("kind", "<u4"), ("primitive", "<u4"),
    ("pad", "<u4", 2),
])
assert LIGHT_RECORD_DTYPE.itemsize == 80

# Every entry point include/cenote_c.h declares.
EXPORTED_SYMBOLS = [
    "cenote_last_error", "cenote_context_create", "cenote_context_destroy", "cenote_context_stream",
    "cenote_synchronize", "cenote_scene_create", "cenote_scene_destroy", "cenote_scene_set_camera",
    "cenote_scene_prep_times", "cenote_scene_device_bytes", "cenote_scene_light_records", "cenote_scene_env_tables",
    "cenote_renderer_create", "cenote_renderer_destroy", "cenote_renderer_set_samples_per_wave",
    "cenote_renderer_stats", "cenote_renderer_set_profiling", "cenote_render_once", "cenote_film_create", "cenote_film_destroy", "cenote_film_reset",
    "cenote_film_samples", "cenote_accumulate", "cenote_accumulate_n", "cenote_film_averages", "cenote_film_sums",
    "cenote_film_device_sums", "cenote_probe_sampler", "cenote_probe_bsdf", "cenote_probe_bsdf_sample",
    "cenote_probe_intersect", "cenote_probe_intersect_queued", "cenote_probe_shadow", "cenote_probe_shadow_queued", "cenote_probe_env_sample", "cenote_probe_env_pdf",
    "cenote_env_tables_static", "cenote_scene_create_textured", "cenote_texture_bytes", "cenote_texture_encode",
    "cenote_texture_encode_float",
    "cenote_probe_texture", "cenote_server_create", "cenote_server_destroy", "cenote_job_submit", "cenote_job_poll",
    "cenote_job_wait", "cenote_job_result", "cenote_job_release", "cenote_server_stats", "cenote_guide_create",
    "cenote_guide_destroy", "cenote_guide_params", "cenote_guide_set_params", "cenote_guide_forward",
    "cenote_guide_train_step", "cenote_renderer_set_guide", "cenote_accumulate_range", "cenote_film_tonemap",
    "cenote_film_tonemap_device", "cenote_film_restore",
    "cenote_scene_add_delta_light", "cenote_renderer_set_material_sort", "cenote_renderer_set_tuning",
    "cenote_renderer_get_tuning", "cenote_renderer_autotune", "cenote_context_set_bvh_builder",
    "cenote_scene_bvh_builder",
]

_lib = None


def library() -> C.CDLL:
    """Load libcenote_b200.so (raises if it was never built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise CenoteError(-3, f"{LIB_PATH.name} is not built; run `python -m cenote_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    P, U32, I32, F = C.c_void_p, C.c_uint32, C.c_int32, C.c_float
    sig = {
        "cenote_last_error": (C.c_char_p, []),
        "cenote_context_create": (I32, [P, P]),
        "cenote_context_destroy": (None, [P]),
        "cenote_context_stream": (P, [P]),
        "cenote_synchronize": (I32, [P]),
        "cenote_scene_create": (I32, [P, P, U32, P, P, P, U32, P]),
        "cenote_scene_create_textured": (I32, [P, P, U32, P, P, P, U32, P, U32, P]),
        "cenote_texture_bytes": (C.c_uint64, [U32, U32, U32]),
        "cenote_texture_encode": (I32, [U32, P, U32, U32, P]),
        "cenote_texture_encode_float": (I32, [U32, P, U32, U32, P]),
        "cenote_probe_texture": (I32, [P, U32, U32, P, U32, P]),
        "cenote_server_create": (I32, [P, C.c_uint64, P, P]),
        "cenote_server_destroy": (None, [P]),
        "cenote_job_submit": (I32, [P, P, U32, U32, U32, U32, P, P, P]),
        "cenote_job_poll": (I32, [P, C.c_uint64, P]),
        "cenote_job_wait": (I32, [P, C.c_uint64, C.c_double]),
        "cenote_job_result": (I32, [P, C.c_uint64, P]),
        "cenote_job_release": (I32, [P, C.c_uint64]),
        "cenote_server_stats": (I32, [P, P]),
        "cenote_guide_create": (I32, [P, C.c_uint64, P]),
        "cenote_guide_destroy": (None, [P]),
        "cenote_guide_params": (I32, [P, P]),
        "cenote_guide_set_params": (I32, [P, P]),
        "cenote_guide_forward": (I32, [P, P, U32, P]),
        "cenote_guide_train_step": (I32, [P, P, P, P, U32, F, P, P]),
        "cenote_renderer_set_guide": (I32, [P, P, F, U32, F]),
        "cenote_accumulate_range": (I32, [P, P, P, U32, U32]),
        "cenote_film_tonemap": (I32, [P, F, P]),
        "cenote_film_tonemap_device": (I32, [P, F, P]),
        "cenote_film_restore": (I32, [P, P, U32]),
        "cenote_scene_add_delta_light": (I32, [P, P]),
        "cenote_renderer_set_material_sort": (I32, [P, U32]),
        "cenote_renderer_set_tuning": (I32, [P, P]),
        "cenote_renderer_get_tuning": (I32, [P, P]),
        "cenote_renderer_autotune": (I32, [P, P, U32, U32, P]),
        "cenote_context_set_bvh_builder": (I32, [P, U32]),
        "cenote_scene_bvh_builder": (U32, [P]),
        "cenote_scene_destroy": (None, [P]),
        "cenote_scene_set_camera": (I32, [P, P]),
        "cenote_scene_prep_times": (I32, [P, P]),
        "cenote_scene_device_bytes": (C.c_uint64, [P]),
        "cenote_scene_light_records": (I32, [P, P, P]),
        "cenote_scene_env_tables": (I32, [P, P, P, P, P, P]),
        "cenote_renderer_create": (I32, [P, U32, U32, U32, P]),
        "cenote_renderer_destroy": (None, [P]),
        "cenote_renderer_set_samples_per_wave": (I32, [P, U32]),
        "cenote_renderer_stats": (I32, [P, P]),
        "cenote_renderer_set_profiling": (I32, [P, U32]),
        "cenote_render_once": (I32, [P, P, U32, U32, U32, P]),
        "cenote_film_create": (I32, [P, U32, U32, P]),
        "cenote_film_destroy": (None, [P]),
        "cenote_film_reset": (I32, [P]),
        "cenote_film_samples": (U32, [P]),
        "cenote_accumulate": (I32, [P, P, P]),
        "cenote_accumulate_n": (I32, [P, P, P, U32]),
        "cenote_film_averages": (I32, [P, P, P, P, P]),
        "cenote_film_sums": (I32, [P, P]),
        "cenote_film_device_sums": (P, [P]),
        "cenote_probe_sampler": (I32, [P, U32, U32, U32, P, P]),
        "cenote_probe_bsdf": (I32, [P, P, P, P, U32, U32, P, P]),
        "cenote_probe_bsdf_sample": (I32, [P, P, P, P, U32, U32, P, P, P]),
        "cenote_probe_intersect": (I32, [P, P, P, U32, P, P]),
        "cenote_probe_intersect_queued": (I32, [P, P, P, U32, P, P]),
        "cenote_probe_shadow": (I32, [P, P, P, P, P, U32, P]),
        "cenote_probe_shadow_queued": (I32, [P, P, P, P, P, U32, P]),
        "cenote_probe_env_sample": (I32, [P, P, U32, P, P, P]),
        "cenote_probe_env_pdf": (I32, [P, P, U32, P]),
        "cenote_env_tables_static": (I32, [P, P, U32, U32, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(code: int) -> None:
    if code != 0:
        msg = library().cenote_last_error()
        raise CenoteError(code, msg.decode() if msg else "")


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _c_material(m) -> Material:
    out = Material()
    C.memmove(C.addressof(out), np.asarray(m, scenes.MATERIAL_DTYPE).tobytes(), 144)
    return out


def _c_camera(cam: scenes.Camera) -> CameraC:
    c = CameraC()
    c.position[:] = [float(v) for v in cam.position]
    c.look_at[:] = [float(v) for v in cam.look_at]
    c.up[:] = [float(v) for v in cam.up]
    c.vfov_degrees = cam.vfov_degrees
    c.aperture_radius = cam.aperture_radius
    c.focus_distance = cam.focus_distance
    return c


BVH_HOST_SAH, BVH_GPU_PLOC, BVH_GPU_SAH, BVH_AUTO = 0, 1, 2, 3


class Context:
    """One CUDA device and the stream every handle made from it shares."""

    def __init__(self, device: int = 0):
        lib = library()
        h = C.c_void_p()
        opts = Options(device)
        _check(lib.cenote_context_create(C.byref(opts), C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return library().cenote_context_stream(self._h) or 0

    def synchronize(self) -> None:
        _check(library().cenote_synchronize(self._h))

    def set_bvh_builder(self, builder: int) -> None:
        """BVH_HOST_SAH, BVH_GPU_PLOC, BVH_GPU_SAH or BVH_AUTO (the default:
        GPU_SAH from 2^20 triangles, else HOST_SAH) for scenes created from
        now on."""
        _check(library().cenote_context_set_bvh_builder(self._h, builder))

    def close(self) -> None:
        if self._h:
            library().cenote_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- probes -------------------------------------------------------------------

    def probe_sampler(self, pixel: int, dimension: int, count: int):
        pts = np.zeros((count, 2), np.float32)
        vals = np.zeros(count, np.float32)
        _check(library().cenote_probe_sampler(self._h, pixel, dimension, count, _ptr(pts), _ptr(vals)))
        return pts, vals

    def probe_bsdf(self, material, wo: np.ndarray, wi: np.ndarray, exiting: bool = False):
        wo = np.ascontiguousarray(wo, np.float32)
        wi = np.ascontiguousarray(wi, np.float32)
        n = len(wo)
        f = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        m = _c_material(material)
        _check(library().cenote_probe_bsdf(self._h, C.byref(m), _ptr(wo), _ptr(wi), n, int(exiting), _ptr(f), _ptr(pdf)))
        return f, pdf

    def probe_bsdf_sample(self, material, wo: np.ndarray, u: np.ndarray, exiting: bool = False):
        wo = np.ascontiguousarray(wo, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        n = len(wo)
        wi = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        lobe = np.zeros(n, np.uint32)
        m = _c_material(material)
        _check(library().cenote_probe_bsdf_sample(self._h, C.byref(m), _ptr(wo), _ptr(u), n, int(exiting), _ptr(wi),
                                                  _ptr(pdf), _ptr(lobe)))
        return wi, pdf, lobe


def env_tables_static(ctx: "Context", texels_ptr: int, width: int, height: int, marginal_ptr: int,
                      conditional_ptr: int, pdfs_ptr: int) -> float:
    """The environment tables into caller-owned device memory, with no device
    allocation inside the library (see cenote_env_tables_static in
    include/cenote_c.h for who needs that and its size limit). Returns the
    emitted power."""
    power = C.c_double()
    _check(library().cenote_env_tables_static(ctx.handle, texels_ptr, width, height, marginal_ptr, conditional_ptr,
                                              pdfs_ptr, C.byref(power)))
    return power.value


class TextureC(C.Structure):
    _fields_ = [("format", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32), ("pad", C.c_uint32),
                ("data", C.c_void_p)]


def texture_bytes(fmt: int, width: int, height: int) -> int:
    return int(library().cenote_texture_bytes(fmt, width, height))


def encode_texture(fmt: int, tex: scenes.Texture) -> scenes.Texture:
    """BC-encode an RGBA8 texture (the host prep step; no device needed)."""
    src = np.ascontiguousarray(tex.data, np.uint8)
    n = texture_bytes(fmt, tex.width, tex.height)
    if n == 0:
        raise CenoteError(-1, f"format {fmt} cannot hold a {tex.width}x{tex.height} texture")
    out = np.zeros(n, np.uint8)
    _check(library().cenote_texture_encode(fmt, _ptr(src), tex.width, tex.height, _ptr(out)))
    return scenes.Texture(fmt, tex.width, tex.height, out)


def encode_texture_float(fmt: int, tex: scenes.Texture) -> scenes.Texture:
    """BC6H-encode an RGBA32F texture (unsigned; the host prep step)."""
    src = np.ascontiguousarray(tex.data, np.float32)
    n = texture_bytes(fmt, tex.width, tex.height)
    if n == 0:
        raise CenoteError(-1, f"format {fmt} cannot hold a {tex.width}x{tex.height} texture")
    out = np.zeros(n, np.uint8)
    _check(library().cenote_texture_encode_float(fmt, _ptr(src), tex.width, tex.height, _ptr(out)))
    return scenes.Texture(fmt, tex.width, tex.height, out)


class Scene:
    """Scene::new: meshes, transforms and materials, a camera and an environment."""

    def __init__(self, ctx: Context, spec: SceneSpec):
        lib = library()
        self.ctx = ctx
        self.spec = spec
        self._keep = []
        objs = (Object * len(spec.objects))()
        for i, o in enumerate(spec.objects):
            m = o.mesh
            arrays = [np.ascontiguousarray(a) for a in (m.positions, m.normals, m.uvs, m.indices)]
            self._keep += arrays
            objs[i].positions, objs[i].normals, objs[i].uvs, objs[i].indices = [_ptr(a) for a in arrays]
            objs[i].vertex_count = len(m.positions)
            objs[i].triangle_count = len(m.indices)
            objs[i].transform[:] = [float(v) for v in np.asarray(o.transform, np.float32)]
            objs[i].material = _c_material(o.material)
            objs[i].camera_visible = 1 if o.camera_visible else 0
        env = spec.environment
        tex = np.ascontiguousarray(env.texels, np.float32)
        self._keep.append(tex)
        envc = EnvironmentC(env.width, env.height, _ptr(tex))
        deltas = (DeltaLightC * max(1, len(spec.delta_lights)))()
        for i, d in enumerate(spec.delta_lights):
            deltas[i].kind = d.kind
            deltas[i].anchor[:] = list(d.anchor)
            deltas[i].emission[:] = list(d.emission)
        cam = _c_camera(spec.camera)
        texs = (TextureC * max(1, len(spec.textures)))()
        for k, t in enumerate(spec.textures):
            data = np.ascontiguousarray(t.data)
            self._keep.append(data)
            texs[k].format, texs[k].width, texs[k].height = t.format, t.width, t.height
            texs[k].data = _ptr(data)
        h = C.c_void_p()
        _check(lib.cenote_scene_create_textured(ctx.handle, objs, len(spec.objects), C.byref(cam), C.byref(envc),
                                                deltas, len(spec.delta_lights), texs, len(spec.textures),
                                                C.byref(h)))
        self._h = h
        self._keep = None  # the library copied everything it needs

    @property
    def handle(self):
        return self._h

    def set_camera(self, cam: scenes.Camera) -> None:
        c = _c_camera(cam)
        _check(library().cenote_scene_set_camera(self._h, C.byref(c)))

    def add_delta_light(self, light: "scenes.DeltaLight") -> None:
        """Append a point or distant light; the light list and its alias
        table are rebuilt as if the scene had been created with it."""
        d = DeltaLightC()
        d.kind = light.kind
        d.anchor[:] = list(light.anchor)
        d.emission[:] = list(light.emission)
        _check(library().cenote_scene_add_delta_light(self._h, C.byref(d)))

    def prep_times_ms(self):
        out = np.zeros(3, np.float32)
        _check(library().cenote_scene_prep_times(self._h, _ptr(out)))
        return out

    def device_bytes(self) -> int:
        return int(library().cenote_scene_device_bytes(self._h))

    def bvh_builder(self) -> int:
        """The builder this scene's BVH came from (BVH_AUTO resolved)."""
        return int(library().cenote_scene_bvh_builder(self._h))

    def light_records(self) -> np.ndarray:
        n = C.c_uint32()
        _check(library().cenote_scene_light_records(self._h, None, C.byref(n)))
        out = np.zeros(n.value, LIGHT_RECORD_DTYPE)
        if n.value:
            _check(library().cenote_scene_light_records(self._h, _ptr(out), C.byref(n)))
        return out

    def env_tables(self):
        env = self.spec.environment
        w, h = env.width, env.height
        marginal = np.zeros(h + 1, np.float32)
        conditional = np.zeros(h * (w + 1), np.float32)
        pdfs = np.zeros(h * w, np.float32)
        power = C.c_double()
        sel = C.c_float()
        _check(library().cenote_scene_env_tables(self._h, _ptr(marginal), _ptr(conditional), _ptr(pdfs),
                                                 C.byref(power), C.byref(sel)))
        return marginal, conditional, pdfs, power.value, sel.value

    def probe_intersect(self, origins: np.ndarray, directions: np.ndarray, queued: bool = False):
        """Closest hits; `queued` walks them through the warp triangle queue."""
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(directions, np.float32)
        n = len(o)
        hits = np.zeros((n, 4), np.uint32)
        t = np.zeros(n, np.float32)
        fn = library().cenote_probe_intersect_queued if queued else library().cenote_probe_intersect
        _check(fn(self._h, _ptr(o), _ptr(d), n, _ptr(hits), _ptr(t)))
        return hits, t

    def probe_shadow(self, origins, directions, tmax, targets, queued: bool = False):
        """Shadow queries; `queued` walks them through the warp triangle queue."""
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(directions, np.float32)
        tm = np.ascontiguousarray(tmax, np.float32)
        tg = np.ascontiguousarray(targets, np.uint32)
        n = len(o)
        out = np.zeros(n, np.float32)
        fn = library().cenote_probe_shadow_queued if queued else library().cenote_probe_shadow
        _check(fn(self._h, _ptr(o), _ptr(d), _ptr(tm), _ptr(tg), n, _ptr(out)))
        return out

    def probe_env_sample(self, u: np.ndarray):
        u = np.ascontiguousarray(u, np.float32)
        n = len(u)
        d = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        rc = np.zeros((n, 2), np.uint32)
        _check(library().cenote_probe_env_sample(self._h, _ptr(u), n, _ptr(d), _ptr(pdf), _ptr(rc)))
        return d, pdf, rc

    def probe_texture(self, index: int, uv: np.ndarray, mode: int = 0) -> np.ndarray:
        """n taps of bindless slot `index`: 0 filtered texel, 1 sampleColor, 2 sampleScalar, 3 sampleNormal."""
        u = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
        out = np.zeros((len(u), 4), np.float32)
        _check(library().cenote_probe_texture(self._h, index, mode, _ptr(u), len(u), _ptr(out)))
        return out

    def probe_env_pdf(self, directions: np.ndarray):
        d = np.ascontiguousarray(directions, np.float32)
        out = np.zeros(len(d), np.float32)
        _check(library().cenote_probe_env_pdf(self._h, _ptr(d), len(d), _ptr(out)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().cenote_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Film:
    """The progressive film: running sums plus the sample count."""

    def __init__(self, ctx: Context, width: int, height: int):
        h = C.c_void_p()
        _check(library().cenote_film_create(ctx.handle, width, height, C.byref(h)))
        self._h = h
        self.ctx = ctx
        self.width, self.height = width, height

    @property
    def handle(self):
        return self._h

    @property
    def samples(self) -> int:
        return int(library().cenote_film_samples(self._h))

    def reset(self) -> None:
        _check(library().cenote_film_reset(self._h))

    def averages(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.zeros((self.height, self.width, 4), np.float32)
        _check(library().cenote_film_averages(self._h, _ptr(out), None, None, None))
        return out

    def all_averages(self) -> dict:
        """Film::averages (film.rs:183-191): beauty, albedo, normal (H, W, 4) and depth (H, W)."""
        out = {k: np.zeros((self.height, self.width, 4), np.float32) for k in ("beauty", "albedo", "normal")}
        out["depth"] = np.zeros((self.height, self.width), np.float32)
        _check(library().cenote_film_averages(self._h, _ptr(out["beauty"]), _ptr(out["albedo"]), _ptr(out["normal"]),
                                              _ptr(out["depth"])))
        return out

    def averages_into(self, ptr: int) -> None:
        """Resolve into caller memory at `ptr` (pinned host memory for speed)."""
        _check(library().cenote_film_averages(self._h, ptr, None, None, None))

    def tonemap(self, exposure_stops: float = 0.0) -> np.ndarray:
        """The display frame (tonemap.slang): uint8 (H, W, 4), sRGB-encoded."""
        out = np.zeros((self.height, self.width), np.uint32)
        _check(library().cenote_film_tonemap(self._h, exposure_stops, _ptr(out)))
        return out.view(np.uint8).reshape(self.height, self.width, 4)

    def tonemap_device(self, exposure_stops: float, ptr: int) -> None:
        """Write the display frame (H*W packed RGBA8 words) to device memory at
        `ptr`, ordered on the context's stream; returns without waiting."""
        _check(library().cenote_film_tonemap_device(self._h, exposure_stops, ptr))

    def set_sums(self, beauty_sum: np.ndarray, samples: int) -> None:
        """Resume from saved beauty sums (H, W, 4) holding `samples` samples."""
        s = np.ascontiguousarray(beauty_sum, np.float32)
        if s.shape != (self.height, self.width, 4):
            raise CenoteError(-1, f"sums of shape {s.shape} for a {self.width}x{self.height} film")
        _check(library().cenote_film_restore(self._h, _ptr(s), samples))

    def sums(self) -> np.ndarray:
        out = np.zeros((self.height, self.width, 4), np.float32)
        _check(library().cenote_film_sums(self._h, _ptr(out)))
        return out

    def device_sums(self) -> int:
        return int(library().cenote_film_device_sums(self._h) or 0)

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().cenote_film_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SORT_NONE, SORT_ALL, SORT_SECONDARY = 0, 1, 2


class Renderer:
    """Renderer::with_max_bounces + LightSampling: the wavefront engine."""

    def __init__(self, ctx: Context, max_bounces: int = 8, light_sampling: int = LIGHT_SAMPLING_MIS,
                 capacity: int = 0, samples_per_wave: int = 0, material_sort: int | None = None):
        h = C.c_void_p()
        _check(library().cenote_renderer_create(ctx.handle, max_bounces, light_sampling, capacity, C.byref(h)))
        self._h = h
        self.ctx = ctx
        if samples_per_wave:
            self.set_samples_per_wave(samples_per_wave)
        if material_sort is not None:
            self.set_material_sort(material_sort)

    @property
    def handle(self):
        return self._h

    def set_samples_per_wave(self, n: int) -> None:
        _check(library().cenote_renderer_set_samples_per_wave(self._h, n))

    def set_material_sort(self, mode: int) -> None:
        """SORT_NONE, SORT_ALL or SORT_SECONDARY: shade each bounce's paths in material order."""
        _check(library().cenote_renderer_set_material_sort(self._h, mode))

    def tuning(self) -> dict:
        t = TuningC()
        _check(library().cenote_renderer_get_tuning(self._h, C.byref(t)))
        return {name: getattr(t, name) for name, _ in TuningC._fields_}

    def set_tuning(self, material_sort: int, samples_per_wave: int = 0, refill_idle: int = 0,
                   top_nodes: int = 0, l2_window: int = 0, per_lane_triangles: int = 0, block_size: int = 0,
                   stack_depth: int = 0, sort_by_location: int = 0) -> None:
        t = TuningC(material_sort, samples_per_wave, refill_idle, top_nodes, l2_window, per_lane_triangles, 0.0,
                    block_size, stack_depth, sort_by_location)
        _check(library().cenote_renderer_set_tuning(self._h, C.byref(t)))

    def autotune(self, scene: Scene, width: int, height: int) -> dict:
        """Time the launch knobs on `scene` at width x height, keep the fastest and return it."""
        t = TuningC()
        _check(library().cenote_renderer_autotune(self._h, scene.handle, width, height, C.byref(t)))
        return {name: getattr(t, name) for name, _ in TuningC._fields_}

    def render(self, scene: Scene, width: int, height: int, sample: int = 0) -> np.ndarray:
        out = np.zeros((height, width, 4), np.float32)
        _check(library().cenote_render_once(self._h, scene.handle, width, height, sample, _ptr(out)))
        return out

    def accumulate(self, scene: Scene, film: Film, count: int = 1) -> None:
        _check(library().cenote_accumulate_n(self._h, scene.handle, film.handle, count))

    def accumulate_range(self, scene: Scene, film: Film, first_sample: int, count: int) -> None:
        """Accumulate samples first_sample .. first_sample + count - 1 (independent of the film's count)."""
        _check(library().cenote_accumulate_range(self._h, scene.handle, film.handle, first_sample, count))

    def set_guide(self, guide, fraction: float = 0.5, train_steps: int = 0, lr: float = 1e-2) -> None:
        """Guided sampling with a Guide (None detaches); train_steps Adam steps per wave."""
        self._guide = guide  # keep it alive while attached
        _check(library().cenote_renderer_set_guide(self._h, guide._h if guide else None, fraction, train_steps, lr))

    def set_profiling(self, flags: int) -> None:
        _check(library().cenote_renderer_set_profiling(self._h, flags))

    def stats(self) -> dict:
        s = Stats()
        _check(library().cenote_renderer_stats(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in Stats._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().cenote_renderer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- serving ---------------------------------------------------------------------

JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3

FRAME_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.POINTER(C.c_float), C.c_uint32,
                       C.c_uint32)


class ServerOptions(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("frame_spp", C.c_uint32), ("max_active", C.c_uint32),
                ("pool_paths", C.c_uint32), ("light_sampling", C.c_uint32), ("no_graphs", C.c_uint32)]


class JobStatus(C.Structure):
    _fields_ = [("state", C.c_uint32), ("samples", C.c_uint32), ("target", C.c_uint32), ("error", C.c_int32),
                ("submit_ms", C.c_double), ("admit_ms", C.c_double), ("first_frame_ms", C.c_double),
                ("done_ms", C.c_double)]


class ServerCounters(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("queued", C.c_uint64), ("active", C.c_uint64), ("samples", C.c_uint64),
                ("bytes_in_use", C.c_uint64), ("budget", C.c_uint64), ("wall_ms", C.c_double),
                ("waves", C.c_uint64), ("first_waves", C.c_uint64), ("wave_paths", C.c_uint64),
                ("busy_ms", C.c_double)]


class Server:
    """The serving loop (cenote_server_*): progressive jobs admitted by an HBM
    budget and traced together, job-tagged, in waves over `slots` lanes (1 or
    2; a path pool and a stream pair each). `on_frame(job, samples, target,
    rgba)` runs on the server thread after every frame_spp samples."""

    def __init__(self, ctx: Context, hbm_budget: int, slots: int = 0, frame_spp: int = 0, max_active: int = 0,
                 pool_paths: int = 0, light_sampling: int = LIGHT_SAMPLING_MIS, graphs: bool = True, on_frame=None):
        opt = ServerOptions(slots, frame_spp, max_active, pool_paths, light_sampling, 0 if graphs else 1)
        h = C.c_void_p()
        _check(library().cenote_server_create(ctx.handle, int(hbm_budget), C.byref(opt), C.byref(h)))
        self._h = h
        self.ctx = ctx
        self._sizes = {}
        self._on_frame = on_frame
        self._fn = FRAME_FN(self._frame) if on_frame else None

    def _frame(self, user, job, samples, target, rgba, w, h):
        img = np.ctypeslib.as_array(rgba, shape=(h, w, 4)).copy()
        self._on_frame(int(job), int(samples), int(target), img)

    def submit(self, scene: Scene, width: int, height: int, target_spp: int, max_bounces: int) -> int:
        job = C.c_uint64()
        _check(library().cenote_job_submit(self._h, scene.handle, width, height, target_spp, max_bounces,
                                           C.cast(self._fn, C.c_void_p) if self._fn else None, None, C.byref(job)))
        self._sizes[job.value] = (width, height)
        return job.value

    def poll(self, job: int) -> JobStatus:
        st = JobStatus()
        _check(library().cenote_job_poll(self._h, job, C.byref(st)))
        return st

    def wait(self, job: int, timeout_ms: float = 600000.0) -> None:
        _check(library().cenote_job_wait(self._h, job, timeout_ms))

    def result(self, job: int) -> np.ndarray:
        w, h = self._sizes[job]
        out = np.zeros((h, w, 4), np.float32)
        _check(library().cenote_job_result(self._h, job, _ptr(out)))
        return out

    def release(self, job: int) -> None:
        _check(library().cenote_job_release(self._h, job))
        self._sizes.pop(job, None)

    def stats(self) -> dict:
        st = ServerCounters()
        _check(library().cenote_server_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerCounters._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().cenote_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- the learned guide ---------------------------------------------------------------

GUIDE_IN, GUIDE_OUT, GUIDE_PARAMS = 96, 40, 17128


class Guide:
    """The directional guide's MLP (cenote_guide_*): tensor-core forward and
    training step over host arrays."""

    def __init__(self, ctx: Context, seed: int = 1):
        h = C.c_void_p()
        _check(library().cenote_guide_create(ctx.handle, seed, C.byref(h)))
        self._h = h
        self.ctx = ctx

    def params(self) -> np.ndarray:
        out = np.zeros(GUIDE_PARAMS, np.float32)
        _check(library().cenote_guide_params(self._h, _ptr(out)))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == GUIDE_PARAMS
        _check(library().cenote_guide_set_params(self._h, _ptr(p)))

    def forward(self, feats: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(feats, np.float32).reshape(-1, GUIDE_IN)
        out = np.zeros((len(x), GUIDE_OUT), np.float32)
        _check(library().cenote_guide_forward(self._h, _ptr(x), len(x), _ptr(out)))
        return out

    def train_step(self, feats, dirs, weights, lr: float = 0.0, grads: bool = False):
        x = np.ascontiguousarray(feats, np.float32).reshape(-1, GUIDE_IN)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        w = np.ascontiguousarray(weights, np.float32).reshape(-1)
        loss = np.zeros(1, np.float32)
        g = np.zeros(GUIDE_PARAMS, np.float32) if grads else None
        _check(library().cenote_guide_train_step(self._h, _ptr(x), _ptr(d), _ptr(w), len(x), lr, _ptr(loss),
                                                 _ptr(g) if grads else None))
        return (float(loss[0]), g) if grads else float(loss[0])

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().cenote_guide_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
