"""Headless command line, the `cenote-cli render` contract
(crates/cenote-cli/src/main.rs:30-65, 96-244):

    python -m cenote_b200.cli render [SCENE] [--spp N] [--width W] [--height H]
                                     [--depth D] [--out render.exr] [--frames K]

SCENE is a built-in workload (cornell, chart, textured, large, ceiling_box), a
scene file in the reference's change-set format (.ron, cenote_b200.scene_file)
or a pbrt-v4 file (.pbrt, the subset cenote_b200.pbrt imports). Unset flags take the scene's own settings.
Accumulates SPP samples and writes the linear averages as one multi-layer
EXR: beauty R/G/B/A, the denoiser guides albedo.R/G/B and normal.X/Y/Z, depth Z
(crates/cenote-cli/src/main.rs:196-216).
--png additionally writes the display frame the reference's viewer presents
(crates/cenote/shaders/tonemap.slang: exposure --exposure stops, ACES fit, sRGB)
as an 8-bit PNG, tonemapped on the device.
--frames repeats the render (profiling); --samples-per-wave fixes how many
samples of every pixel one wave carries; --tuning pins the launch knobs
(sort,samples_per_wave,refill,top_nodes,l2) and --autotune picks them on the
scene first; --stats prints the renderer's counters.
"""
from __future__ import annotations

import argparse
import json
import struct
import sys
import time
import zlib

import numpy as np

from . import Context, Film, Renderer, Scene, scenes
from .exr import write_aov_exr


def load_scene(name: str):
    if name.endswith(".pbrt"):
        from .pbrt import import_pbrt
        return import_pbrt(name)
    if name.endswith(".ron"):
        from .scene_file import load_scene_file
        return load_scene_file(name)
    if name in scenes.SCENES:
        return scenes.SCENES[name]()
    raise SystemExit(f"unknown scene {name!r}: use one of {sorted(scenes.SCENES)}, a .ron or a .pbrt file")


def write_png(path: str, rgba8: np.ndarray) -> None:
    """An 8-bit RGBA PNG (no filtering) from uint8 (H, W, 4)."""
    h, w = rgba8.shape[:2]
    raw = b"".join(b"\x00" + rgba8[y].tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
                chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))


def render(args) -> int:
    spec = load_scene(args.scene)
    width = args.width or spec.width
    height = args.height or spec.height
    spp = args.spp or spec.spp
    depth = args.depth or spec.max_bounces
    ctx = Context(args.device)
    t0 = time.perf_counter()
    scene = Scene(ctx, spec)
    prep = time.perf_counter() - t0
    renderer = Renderer(ctx, depth, samples_per_wave=args.samples_per_wave)
    if args.tuning:
        knobs = [int(x) for x in args.tuning.split(",")]
        if args.samples_per_wave and len(knobs) > 1:
            knobs[1] = args.samples_per_wave
        renderer.set_tuning(*knobs)
    elif args.autotune:
        renderer.autotune(scene, width, height)
    film = Film(ctx, width, height)
    t0 = time.perf_counter()
    for _ in range(max(1, args.frames)):
        film.reset()
        renderer.accumulate(scene, film, spp)
    dt = (time.perf_counter() - t0) / max(1, args.frames)
    if args.out:
        av = film.all_averages()
        write_aov_exr(args.out, av["beauty"], av["albedo"], av["normal"], av["depth"])
    if args.png:
        write_png(args.png, film.tonemap(args.exposure))
    st = renderer.stats()
    msg = (f"wrote {args.out} ({width}x{height}, {spp} spp, depth {depth}; layers: beauty, albedo, normal, Z) "
           f"in {dt * 1e3:.1f} ms/frame, "
           f"{width * height * spp / dt / 1e6:.1f} Msamples/s, prep {prep * 1e3:.1f} ms")
    print(msg, file=sys.stderr)
    if args.stats:
        print(json.dumps(st))
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="cenote-cli", description="cenote-b200: a B200 path tracer")
    sub = ap.add_subparsers(dest="command", required=True)
    r = sub.add_parser("render", help="render a scene to an EXR")
    r.add_argument("scene", nargs="?", default="chart")
    r.add_argument("--spp", type=int, default=0)
    r.add_argument("--width", type=int, default=0)
    r.add_argument("--height", type=int, default=0)
    r.add_argument("--depth", type=int, default=0)
    r.add_argument("--out", default="render.exr")
    r.add_argument("--frames", type=int, default=1)
    r.add_argument("--device", type=int, default=0)
    r.add_argument("--samples-per-wave", type=int, default=0, help="0 = automatic")
    r.add_argument("--stats", action="store_true")
    r.add_argument("--tuning", default="",
                   help="launch knobs: sort,samples_per_wave,refill,top_nodes,l2[,per_lane_triangles]")
    r.add_argument("--autotune", action="store_true", help="time the launch knobs on the scene first")
    r.add_argument("--png", default="", help="also write the tonemapped display frame here")
    r.add_argument("--exposure", type=float, default=0.0, help="display exposure in stops (--png)")
    args = ap.parse_args(argv)
    for v in (args.spp, args.width, args.height, args.samples_per_wave):
        if v < 0:
            ap.error("sizes must be positive")
    if args.depth and not 1 <= args.depth <= 255:
        ap.error("--depth must be in 1..=255")
    return render(args)


if __name__ == "__main__":
    sys.exit(main())
