"""The kernels' BVH on the CPU: the library's wide-BVH builder and the device
traversal header (cenote_b200/csrc/traverse.cuh), compiled for the host
through tests/host/cuda_host_shim.h, must produce a well-formed tree (every
index in range, every triangle in exactly one leaf) and commit bit-identical
closest hits to the oracle's independent binary BVH on the same rays.

This validates traversal logic and memory safety before any GPU runs it; the
GPU tests repeat the comparison on the device."""
import pathlib
import subprocess

import numpy as np
import pytest

import oracle
from cenote_b200 import scenes

ROOT = pathlib.Path(__file__).resolve().parents[1]
CSRC = ROOT / "cenote_b200" / "csrc"
HOST = ROOT / "tests" / "host"


def cuda_include():
    import shutil
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return pathlib.Path(nvcc).resolve().parent.parent / "include"


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = tmp_path_factory.mktemp("host") / "traverse_host"
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{HOST}", f"-I{CSRC}", f"-I{cuda_include()}",
           "-include", str(HOST / "cuda_host_shim.h"), str(HOST / "traverse_host.cpp"), str(CSRC / "bvh_build.cpp"),
           "-o", str(out), "-lpthread"]
    subprocess.run(cmd, check=True)
    return out


def world_triangles(spec):
    """World-space corners in the library's f32 operation order (glam's
    transform_point3: ((x·p.x + y·p.y) + z·p.z) + w)."""
    out = []
    for inst, o in enumerate(spec.objects):
        m = np.asarray(o.transform, np.float32).reshape(3, 4)
        p = o.mesh.positions.astype(np.float32)
        w = np.empty_like(p)
        for r in range(3):
            w[:, r] = ((m[r, 0] * p[:, 0] + m[r, 1] * p[:, 1]) + m[r, 2] * p[:, 2]) + m[r, 3]
        c = w[o.mesh.indices]  # (T, 3, 3)
        ids = np.zeros((len(c), 3), np.uint32)
        ids[:, 0] = inst
        ids[:, 1] = np.arange(len(c))
        ids[:, 2] = 0xFF | 0x100
        out.append((c.reshape(-1, 9), ids))
    return np.concatenate([c for c, _ in out]), np.concatenate([i for _, i in out])


def random_rays(spec, n, seed):
    rng = np.random.default_rng(seed)
    tris, _ = world_triangles(spec)
    pts = tris.reshape(-1, 3)
    lo, hi = pts.min(0), pts.max(0)
    org = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    d = rng.normal(size=(n, 3))
    # A few axis-aligned and exactly-zero components to exercise the slab edge cases.
    d[: n // 16, 1] = 0.0
    d[n // 16: n // 8, :2] = 0.0
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return org, d


def run_harness(harness, tmp_path, tris, ids, org, d, lanes=None):
    tb = tmp_path / "tris.bin"
    with open(tb, "wb") as f:
        f.write(np.uint32(len(tris)).tobytes())
        rec = np.concatenate([tris.view(np.uint32), ids], axis=1).astype(np.uint32)
        f.write(rec.tobytes())
    rb = tmp_path / "rays.bin"
    with open(rb, "wb") as f:
        f.write(np.uint32(len(org)).tobytes())
        f.write(np.concatenate([org, d], axis=1).astype(np.float32).tobytes())
    hb = tmp_path / "hits.bin"
    import os
    env = dict(os.environ)
    if lanes is not None:
        env["CN_HOST_LANES"] = str(lanes)
    r = subprocess.run([str(harness), str(tb), str(rb), str(hb)], capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    h = np.fromfile(hb, np.uint32).reshape(-1, 5)
    return h[:, :4], h[:, 4].view(np.float32), r.stdout


@pytest.mark.parametrize("lanes", [None, 1], ids=["random-lanes", "lone-lane"])
@pytest.mark.parametrize("name", ["cornell", "chart"])
def test_wide_bvh_matches_oracle_hits(harness, tmp_path, name, lanes):
    spec = scenes.cornell() if name == "cornell" else scenes.chart(env_size=(8, 4))
    tris, ids = world_triangles(spec)
    org, d = random_rays(spec, 20000, seed=1)
    hits, t, log = run_harness(harness, tmp_path, tris, ids, org, d, lanes)
    ref_hits, ref_t = oracle.OracleScene(spec).intersect(org, d)
    assert np.array_equal(hits, ref_hits), log
    assert np.array_equal(t.view(np.uint32), ref_t.view(np.uint32))
    assert (hits[:, 0] != 0xFFFFFFFF).mean() > 0.3


def test_wide_bvh_random_soup(harness, tmp_path):
    """A dense random triangle soup: many overlapping boxes, deep trees. Above
    65,536 triangles, so the root splits by binned SAH and the subtrees by the
    exact sweep."""
    rng = np.random.default_rng(7)
    n = 80000
    c = rng.random((n, 1, 3)) * 10.0 + rng.normal(scale=0.05, size=(n, 3, 3))
    tris = c.astype(np.float32).reshape(n, 9)
    ids = np.zeros((n, 3), np.uint32)
    ids[:, 1] = np.arange(n)
    ids[:, 2] = 0x1FF
    org = (rng.random((5000, 3)) * 10.0).astype(np.float32)
    d = rng.normal(size=(5000, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    hits, t, _ = run_harness(harness, tmp_path, tris, ids, org, d)
    # Brute force on the CPU with the oracle's watertight test, via a one-object scene.
    mesh = scenes.Mesh(tris.reshape(-1, 3), np.tile([0, 1, 0], (3 * n, 1)).astype(np.float32),
                       np.zeros((3 * n, 2), np.float32), np.arange(3 * n, dtype=np.uint32).reshape(n, 3))
    spec = scenes.SceneSpec("soup", [scenes.Object(mesh, scenes.rows(np.eye(4)), scenes.matte((0.5, 0.5, 0.5)))],
                            scenes.Camera((0, 0, 20), (5, 5, 5)), scenes.Environment.constant((0, 0, 0)), 8, 8, 1, 1)
    ref_hits, ref_t = oracle.OracleScene(spec).intersect(org, d)
    assert np.array_equal(hits, ref_hits)
    assert np.array_equal(t.view(np.uint32), ref_t.view(np.uint32))


def test_degenerate_inputs(harness, tmp_path):
    """One triangle; coincident centroids (few, and more than the binned
    split's 65,536-triangle threshold); a flat (zero-extent) axis."""
    one = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32)
    same = np.tile(one, (40, 1))
    many = np.tile(one, (70000, 1))
    flat = np.random.default_rng(3).random((500, 9)).astype(np.float32)
    flat[:, 2::3] = 0.25
    for tris in (one, same, many, flat):
        ids = np.zeros((len(tris), 3), np.uint32)
        ids[:, 1] = np.arange(len(tris))
        ids[:, 2] = 0x1FF
        org = np.array([[0.2, 0.2, 1.0], [0.2, 0.2, -1.0], [5, 5, 5]], np.float32)
        d = np.array([[0, 0, -1], [0, 0, 1], [0, 0, 1]], np.float32)
        hits, t, _ = run_harness(harness, tmp_path, tris, ids, org, d)
        assert hits[2, 0] == 0xFFFFFFFF
        if tris is not flat:  # every copy hit at the same t: the lowest primitive wins
            assert hits[0, 0] == 0 and hits[0, 1] == 0 and t[0] == np.float32(1.0)


def camera_rays(spec, width, height):
    """Pinhole rays through pixel centres from the scene camera (float64 basis
    rounded to f32: a traversal workload, not the renderer's raygen)."""
    cam = spec.camera
    p = np.asarray(cam.position, np.float64)
    f = np.asarray(cam.look_at, np.float64) - p
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(cam.up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    th = np.tan(np.radians(cam.vfov_degrees) / 2)
    ys, xs = np.mgrid[0:height, 0:width]
    sx = ((xs + 0.5) / width * 2 - 1) * th * width / height
    sy = (1 - (ys + 0.5) / height * 2) * th
    d = f + sx.reshape(-1, 1) * r + sy.reshape(-1, 1) * u
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return np.broadcast_to(p, d.shape).astype(np.float32), d


def test_tree_quality_chart(harness, tmp_path):
    """Camera rays through the material chart: hits equal the oracle's, and the
    tree stays as cheap to walk as the SAH-swept, cost-optimally collapsed
    build makes it: 4.99 wide nodes and 3.85 triangles per ray here (the
    greedily collapsed 32-bin tree needed 6.01 and 4.54); the bounds leave
    about 5 %."""
    spec = scenes.chart(env_size=(8, 4))
    tris, ids = world_triangles(spec)
    org, d = camera_rays(spec, 160, 90)
    hits, t, log = run_harness(harness, tmp_path, tris, ids, org, d)
    ref_hits, ref_t = oracle.OracleScene(spec).intersect(org, d)
    assert np.array_equal(hits, ref_hits), log
    assert np.array_equal(t.view(np.uint32), ref_t.view(np.uint32))
    words = log.split()
    visits = float(words[words.index("visits/ray") + 1])
    tests = float(words[words.index("tests/ray") + 1])
    assert visits < 5.25 and tests < 4.05, log


def test_nested_triangles_keep_the_tree_shallow(harness, tmp_path):
    """Nested triangles of geometrically growing size: at every level the
    SAH's cheapest split peels the largest triangle off, which without a
    bound makes a binary chain as deep as the input. Past 48 SAH levels the
    builder splits at the object median, so the wide tree stays well inside
    the traversal stack and the walk still finds the oracle's hits."""
    n = 300
    k = np.arange(n, dtype=np.float64)
    s = 1.3 ** k
    base = np.array([[-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0]])
    tris = (base[None] * s[:, None, None]).astype(np.float64)
    tris[:, :, 0] += 0.1 * s[:, None]  # distinct centroids, ordered by size
    tris[:, :, 2] = -1e-3 * k[:, None]  # layered in depth: a ray down -z meets the smallest first
    tris = tris.astype(np.float32).reshape(n, 9)
    ids = np.zeros((n, 3), np.uint32)
    ids[:, 1] = np.arange(n)
    ids[:, 2] = 0x1FF
    rng = np.random.default_rng(5)
    org = np.zeros((4000, 3), np.float32)
    org[:, :2] = (rng.normal(size=(4000, 2)) * np.exp(rng.uniform(0, 40, (4000, 1)))).astype(np.float32)
    org[:, 2] = 1.0
    # Steep rays (z their dominant axis): every triangle's corners then sit
    # at one depth along the ray's axis and the FP32 hit distance has no
    # cancellation, whatever the triangle's size.
    d = np.tile(np.array([0, 0, -1], np.float32), (4000, 1))
    d[::2, :2] = rng.uniform(-0.5, 0.5, (2000, 2)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    hits, t, log = run_harness(harness, tmp_path, tris, ids, org, d)
    stack = int(log.split("stack ")[1].split()[0])
    assert stack < 16, log
    mesh = scenes.Mesh(tris.reshape(-1, 3), np.tile([0, 0, 1], (3 * n, 1)).astype(np.float32),
                       np.zeros((3 * n, 2), np.float32), np.arange(3 * n, dtype=np.uint32).reshape(n, 3))
    spec = scenes.SceneSpec("nested", [scenes.Object(mesh, scenes.rows(np.eye(4)), scenes.matte((0.5, 0.5, 0.5)))],
                            scenes.Camera((0, 0, 20), (0, 0, 0)), scenes.Environment.constant((0, 0, 0)), 8, 8, 1, 1)
    ref_hits, ref_t = oracle.OracleScene(spec).intersect(org, d)
    assert np.array_equal(hits, ref_hits)
    assert np.array_equal(t.view(np.uint32), ref_t.view(np.uint32))
    assert (hits[:, 0] != 0xFFFFFFFF).mean() > 0.3
