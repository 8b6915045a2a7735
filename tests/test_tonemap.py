"""The headless display transform (cenote_film_tonemap) against the oracle.

The reference checks its tonemap kernel against a CPU mirror of the same
transform on six synthetic averages at exposure 0.5, allowing one quantisation
step (crates/cenote/src/render/tonemap.rs:164-207); the same fixture and
tolerance pin the oracle here (float64 restatement) and the CUDA kernel (GPU).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import tonemap as T

# crates/cenote/src/render/tonemap.rs:176-183: black, mid grey, white, a hot
# highlight, a negative channel, a saturated red.
FIXTURE = np.array([[0.0, 0.0, 0.0, 1.0], [0.18, 0.18, 0.18, 1.0], [1.0, 1.0, 1.0, 1.0], [10.0, 2.0, 0.5, 1.0],
                    [-0.5, 0.2, 0.2, 1.0], [1.0, 0.1, 0.05, 1.0]], np.float32)


def tonemap64(avg, stops):
    """The transform in float64 with half-away-from-zero rounding (the
    reference's Rust mirror rounds that way)."""
    v = avg[..., :3].astype(np.float64) * 2.0 ** stops
    v = T.ACES_INPUT.astype(np.float64) @ (T.SRGB_FROM_ACESCG.astype(np.float64) @ v.T)
    v = v.T
    fit = (v * (v + 0.0245786) - 0.000090537) / (v * (0.983729 * v + 0.4329510) + 0.238081)
    d = np.clip((T.ACES_OUTPUT.astype(np.float64) @ fit.T).T, 0, 1)
    e = np.where(d <= 0.0031308, 12.92 * d, 1.055 * np.power(d, 1 / 2.4) - 0.055)
    return np.floor(np.clip(e, 0, 1) * 255 + 0.5).astype(np.int32)


def test_oracle_matches_the_known_answer_fixture():
    got = T.tonemap(FIXTURE, 0.5).astype(np.int32)
    ref = tonemap64(FIXTURE, 0.5)
    assert np.abs(got[:, :3] - ref).max() <= 1
    assert (got[:, 3] == 255).all()
    assert (got[0, :3] == 0).all()  # black stays black
    # A negative channel comes out finite; Hill's rational fit rises again
    # below zero, so the reference saturates it rather than clamping it to 0.
    assert got[4, 0] == 255
    assert got[2, 0] == got[2, 1] == got[2, 2]  # white stays neutral
    assert got[3, 0] == 255 and got[3, 2] < 255  # the highlight is compressed, not clipped everywhere


def test_oracle_is_monotonic_in_exposure():
    grey = np.full((1, 4), 0.18, np.float32)
    vals = [int(T.tonemap(grey, s)[0, 0]) for s in np.linspace(-8, 8, 33)]
    assert vals == sorted(vals) and vals[0] < 10 and vals[-1] == 255


def test_oracle_matches_float64_on_random_averages():
    rng = np.random.default_rng(3)
    avg = np.exp(rng.normal(-1.5, 2.0, (4096, 4))).astype(np.float32)
    for stops in (-2.0, 0.0, 1.25):
        d = np.abs(T.tonemap(avg, stops)[:, :3].astype(np.int32) - tonemap64(avg, stops))
        assert d.max() <= 1 and (d > 0).mean() < 0.01


def test_cli_png_writer_round_trips(tmp_path):
    from cenote_b200.cli import write_png
    from cenote_b200.scene_file import read_png

    rng = np.random.default_rng(2)
    img = rng.integers(0, 256, (7, 13, 4), dtype=np.uint8)
    write_png(str(tmp_path / "f.png"), img)
    back = read_png(str(tmp_path / "f.png"))
    assert back.shape[:2] == (7, 13)
    got = back if back.dtype == np.uint8 else np.rint(np.asarray(back) * 255).astype(np.uint8)
    assert np.array_equal(got[..., :4], img)


# ---- the CUDA kernel -------------------------------------------------------------------


def film_with(ctx, avg):
    """A film whose average is `avg`: one sample of a constant-emission
    furnace cannot produce arbitrary pixels, so the sums are written directly."""
    from cenote_b200 import Film

    h, w = avg.shape[:2]
    f = Film(ctx, w, h)
    f.set_sums(avg.astype(np.float32), samples=1)
    return f


@pytest.mark.gpu
def test_gpu_tonemap_matches_the_known_answer_fixture(ctx):
    f = film_with(ctx, FIXTURE.reshape(1, 6, 4))
    got = f.tonemap(0.5).reshape(6, 4).astype(np.int32)
    assert np.abs(got[:, :3] - tonemap64(FIXTURE, 0.5)).max() <= 1
    assert (got[:, 3] == 255).all()


@pytest.mark.gpu
@pytest.mark.parametrize("stops", [-3.0, 0.0, 0.5, 2.0])
def test_gpu_tonemap_matches_the_oracle_on_a_render(ctx, stops):
    from cenote_b200 import Film, Renderer, Scene, scenes

    spec = scenes.cornell(96, 64, 16, 6)
    f = Film(ctx, spec.width, spec.height)
    Renderer(ctx, 6).accumulate(Scene(ctx, spec), f, 16)
    got = f.tonemap(stops).astype(np.int32)
    ref = T.tonemap(f.averages(), stops).astype(np.int32)
    d = np.abs(got - ref)
    assert d.max() <= 1 and (d > 0).mean() < 0.01


@pytest.mark.gpu
def test_gpu_tonemap_into_device_memory(ctx):
    import torch

    rng = np.random.default_rng(9)
    avg = np.exp(rng.normal(-1.0, 2.0, (33, 47, 4))).astype(np.float32)
    f = film_with(ctx, avg)
    out = torch.zeros((33, 47), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()  # the zero fill ran on torch's stream, not the context's
    f.tonemap_device(1.0, out.data_ptr())
    ctx.synchronize()
    got = out.cpu().numpy().view(np.uint8).reshape(33, 47, 4).astype(np.int32)
    d = np.abs(got - T.tonemap(avg, 1.0).astype(np.int32))
    assert d.max() <= 1 and (d > 0).mean() < 0.01


@pytest.mark.gpu
def test_gpu_tonemap_of_an_empty_film_is_an_error(ctx):
    from cenote_b200 import CenoteError, Film

    with pytest.raises(CenoteError):
        Film(ctx, 8, 8).tonemap(0.0)
