"""Generate tests/golden/corpus_*.npz from the reference's pbrt corpus.

Each fixture holds the scene as cenote_b200.pbrt imports it (meshes,
materials, camera, settings; scenes.save_spec layout) and, as the extra
array `golden`, the linear RGB of the reference's own 64-spp render of that
scene (crates/cenote-pbrt/tests/golden/{name}.exr, written by
crates/cenote-pbrt/tests/corpus.rs:84-114 at the resolutions of
corpus.rs:29-33). The GPU test then needs neither the reference tree nor its
pbrt files at run time. A scene lit by an image sky stores the sky's
octahedral source texels (half floats, as the sky file holds them), its
orientation and scale instead of the resampled equirect, and the tests
rebuild the environment with cenote_b200.pbrt.sky_environment.

    python tests/golden/make_corpus.py REFERENCE_ROOT

REFERENCE_ROOT is the reference project's checkout (its tests/scenes and
crates/cenote-pbrt/tests/golden are read); CENOTE_REFERENCE_ROOT may give it
instead.
"""
from __future__ import annotations

import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from cenote_b200.exr import read_exr  # noqa: E402
from cenote_b200.pbrt import import_pbrt  # noqa: E402
from cenote_b200.scenes import Environment, save_spec  # noqa: E402

CORPUS = [("cornell-box", 256, 256), ("veach-mis", 320, 180), ("teapot-full", 320, 180)]


def main(root: str | None = None) -> None:
    import os
    root = root or os.environ.get("CENOTE_REFERENCE_ROOT")
    if not root:
        raise SystemExit("usage: make_corpus.py REFERENCE_ROOT (or set CENOTE_REFERENCE_ROOT)")
    ref = pathlib.Path(root)
    for name, w, h in CORPUS:
        spec = import_pbrt(str(ref / "tests/scenes" / name / "scene-v4.pbrt"), w, h)
        g = read_exr(ref / "crates/cenote-pbrt/tests/golden" / f"{name}.exr")
        golden = np.stack([g["R"], g["G"], g["B"]], -1).astype(np.float32)
        assert golden.shape == (h, w, 3), golden.shape
        out = HERE / f"corpus_{name.replace('-', '_')}.npz"
        extra = {}
        if spec.sky_source is not None:
            src, world_from_light, scale = spec.sky_source
            assert np.array_equal(src.astype(np.float16).astype(np.float32), src), "sky texels are not half floats"
            extra = dict(sky_octahedral=src.astype(np.float16), sky_world_from_light=world_from_light,
                         sky_scale=np.float32(scale))
            spec.environment = Environment.constant((0.0, 0.0, 0.0))  # rebuilt from the source on load
        save_spec(out, spec, golden=golden, warnings=np.array(list(spec.warnings), dtype=str), **extra)
        print(f"{out.name}: {len(spec.objects)} objects, {spec.triangle_count} triangles, "
              f"spp {spec.spp}, max_bounces {spec.max_bounces}, {out.stat().st_size} bytes")


if __name__ == "__main__":
    main(*sys.argv[1:])
