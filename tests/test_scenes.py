"""The procedural inputs: solids restated from crates/cenote/src/scene/shapes.rs
(its own tests, :145-202) and the named workloads' sizes."""
import numpy as np
import pytest

from cenote_b200 import scenes


@pytest.mark.parametrize("n", [0, 1, 2])
def test_icosphere_counts_follow_the_subdivision_formula(n):
    m = scenes.icosphere(n)
    assert m.triangle_count == 20 * 4 ** n
    assert len(m.positions) == 10 * 4 ** n + 2


def test_icosphere_vertices_lie_on_the_unit_sphere():
    m = scenes.icosphere(2)
    assert np.allclose(np.linalg.norm(m.positions, axis=1), 1.0, atol=1e-6)
    assert np.array_equal(m.normals, m.positions)


def test_winding_is_counter_clockwise_outward():
    m = scenes.icosphere(1)
    a, b, c = (m.positions[m.indices[:, k]] for k in range(3))
    assert np.all(np.einsum("ij,ij->i", np.cross(b - a, c - a), a + b + c) > 0)
    p = scenes.ground_plane(5.0)
    a, b, c = (p.positions[p.indices[:, k]] for k in range(3))
    assert np.all(np.cross(b - a, c - a)[:, 1] > 0)
    bx = scenes.box(1.0, 2.0, 0.5)
    a, b, c = (bx.positions[bx.indices[:, k]] for k in range(3))
    n = np.cross(b - a, c - a)
    assert np.all(np.einsum("ij,ij->i", n, (a + b + c) / 3) > 0)


def test_indices_stay_in_bounds():
    m = scenes.icosphere(2)
    assert m.indices.max() < len(m.positions)


def test_workload_sizes():
    c = scenes.cornell()
    assert (c.width, c.height, c.spp, c.max_bounces) == (256, 256, 16, 8)
    assert c.triangle_count == 36
    ch = scenes.chart(env_size=(64, 32))
    assert (ch.width, ch.height, ch.spp, ch.max_bounces) == (1280, 720, 64, 12)
    assert ch.triangle_count == 25 * 1280 + 2 + 2
    assert scenes.MATERIAL_DTYPE.itemsize == 144


def test_sky_has_its_sun():
    env = scenes.sky_hdri(256, 128)
    lum = env.texels[..., :3].mean(-1)
    r, c = np.unravel_index(np.argmax(lum), lum.shape)
    elevation = 90.0 - (r + 0.5) / 128 * 180.0
    assert abs(elevation - 35.0) < 1.5
    assert lum.max() > 1e3
