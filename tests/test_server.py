"""The serving loop: admission by HBM budget, progressive frames, concurrency.

The serving API (cenote_server_*, cenote_job_*) has no counterpart in the
reference, whose Session renders one view at a time
(crates/cenote/src/render/session.rs:416); the properties tested are the
serving contract: a job's result is bitwise the same alone and in any mix,
a frame comes every frame_spp samples, admission respects the budget, and
failures surface as status codes.
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

from cenote_b200 import CenoteError, Film, Renderer, Scene, Server, scenes
from cenote_b200 import JOB_DONE

GIB = 1 << 30


def standalone(ctx, scene, w, h, spp, bounces):
    r = Renderer(ctx, bounces)
    f = Film(ctx, w, h)
    r.accumulate(scene, f, spp)
    return f.averages()


@pytest.fixture(scope="module")
def scene_set(ctx):
    return {
        "cornell": Scene(ctx, scenes.cornell(64, 64, 8, 6)),
        "chart": Scene(ctx, scenes.chart(96, 54, 6, 6, env_size=(256, 128))),
        "textured": Scene(ctx, scenes.textured(80, 45, 4, 5, size=32)),
    }


JOBS = [("cornell", 64, 64, 8, 6), ("chart", 96, 54, 6, 6), ("textured", 80, 45, 5, 5), ("cornell", 48, 40, 1, 8),
        ("chart", 64, 64, 9, 4), ("cornell", 33, 17, 4, 3)]


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
def test_jobs_match_standalone_renders_bitwise(ctx, scene_set, graphs):
    server = Server(ctx, 8 * GIB, slots=2, pool_paths=1 << 18, graphs=graphs)
    ids = [server.submit(scene_set[n], w, h, spp, b) for n, w, h, spp, b in JOBS]
    for j in ids:
        server.wait(j, 120000.0)
    for j, (n, w, h, spp, b) in zip(ids, JOBS):
        got = server.result(j)
        ref = standalone(ctx, scene_set[n], w, h, spp, b)
        assert np.array_equal(got, ref), (n, w, h, spp)
        st = server.poll(j)
        assert st.state == JOB_DONE and st.samples == spp
        assert 0 <= st.submit_ms <= st.admit_ms <= st.first_frame_ms <= st.done_ms
    stats = server.stats()
    assert stats["completed"] == len(JOBS) and stats["failed"] == 0 and stats["queued"] == 0
    assert stats["samples"] == sum(w * h * spp for _, w, h, spp, _ in JOBS)
    for j in ids:
        server.release(j)
    server.close()


@pytest.mark.gpu
def test_progressive_frames_every_frame_spp(ctx, scene_set):
    frames = {}
    lock = threading.Lock()

    def on_frame(job, samples, target, rgba):
        with lock:
            frames.setdefault(job, []).append((samples, target, rgba))

    server = Server(ctx, 8 * GIB, slots=2, frame_spp=4, pool_paths=1 << 18, on_frame=on_frame)
    a = server.submit(scene_set["cornell"], 40, 40, 10, 6)
    b = server.submit(scene_set["chart"], 32, 24, 4, 6)
    server.wait(a)
    server.wait(b)
    assert [s for s, _, _ in frames[a]] == [4, 8, 10]
    assert [s for s, _, _ in frames[b]] == [4]
    # Each frame is the running average: alpha is exactly 1, and the last is the result.
    for s, t, img in frames[a]:
        assert t == 10 and (img[..., 3] == 1.0).all()
    assert np.array_equal(frames[a][-1][2], server.result(a))
    # The 8-spp frame equals a standalone 8-spp render.
    assert np.array_equal(frames[a][1][2], standalone(ctx, scene_set["cornell"], 40, 40, 8, 6))
    server.close()


@pytest.mark.gpu
def test_admission_respects_the_budget(ctx, scene_set):
    """The budget holds the path pool, each resident scene's device bytes
    (BVH, triangles, records, textures, environment tables) once, and every
    admitted job's film: room for two 128x128 jobs of one scene at a time."""
    pool_paths = 1 << 16
    probe = Server(ctx, 8 * GIB, pool_paths=pool_paths)
    pool_bytes = probe.stats()["bytes_in_use"]
    probe.close()
    scene_bytes = scene_set["cornell"].device_bytes()
    job_bytes = 128 * 128 * 32
    budget = pool_bytes + scene_bytes + 2 * job_bytes + 100
    server = Server(ctx, budget, pool_paths=pool_paths)
    ids = [server.submit(scene_set["cornell"], 128, 128, 2, 4) for _ in range(5)]
    peak = 0
    done = set()
    while len(done) < len(ids):
        st = server.stats()
        peak = max(peak, st["active"])
        assert st["bytes_in_use"] <= budget
        for j in ids:
            if server.poll(j).state == JOB_DONE:
                done.add(j)
    assert peak == 2
    with pytest.raises(CenoteError) as e:
        server.submit(scene_set["cornell"], 200, 200, 1, 4)  # could never fit
    assert e.value.code == -8
    server.close()


@pytest.mark.gpu
def test_jobs_of_many_scenes_share_waves_and_match(ctx, scene_set):
    """Twenty-four jobs of three scenes and two bounce counts submitted at
    once, one wave in flight and two: each job's result is bitwise its
    standalone render, whatever it shared its waves with."""
    rng = np.random.default_rng(4)
    jobs = []
    for k in range(24):
        n = ["cornell", "chart", "textured"][k % 3]
        w, h = [(32, 32), (40, 24), (17, 33)][rng.integers(3)]
        jobs.append((n, w, h, int(rng.integers(1, 13)), [4, 6][k % 2]))
    for depth in (1, 2):
        server = Server(ctx, 8 * GIB, slots=depth, frame_spp=4, pool_paths=1 << 14)
        ids = [server.submit(scene_set[n], w, h, spp, b) for n, w, h, spp, b in jobs]
        for j in ids:
            server.wait(j, 120000.0)
        for j, (n, w, h, spp, b) in zip(ids, jobs):
            assert np.array_equal(server.result(j), standalone(ctx, scene_set[n], w, h, spp, b)), (n, w, h, spp, b)
        server.close()


@pytest.mark.gpu
def test_server_rejects_bad_requests(ctx, scene_set):
    with pytest.raises(CenoteError) as e:
        Server(ctx, 1 << 20, pool_paths=1 << 20)  # the pool alone exceeds the budget
    assert e.value.code == -8
    server = Server(ctx, 4 * GIB, slots=1, pool_paths=1 << 16)
    for args in [(0, 8, 1, 4), (8, 8, 0, 4), (8, 8, 1, 0), (8, 8, 1, 256)]:
        with pytest.raises(CenoteError) as e:
            server.submit(scene_set["cornell"], *args)
        assert e.value.code == -1
    with pytest.raises(CenoteError):
        server.poll(12345)
    j = server.submit(scene_set["cornell"], 16, 16, 40, 4)
    with pytest.raises(CenoteError):
        server.release(j)  # still running
    server.wait(j)
    server.release(j)
    server.close()
