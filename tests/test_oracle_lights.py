"""The oracle's restatement of the GI cache's per-light visibility rays (gi_light,
gi_cache.wgsl:2054-2077; gi_light_affects :2028-2036; gi_light_direction :1977-1983), pinned by
the properties the WGSL states: which lights reach a cell (colour, facing, range, spot cone), the
ray toward each (from the cell's offset origin, the one its gather rays use; tmax the light's
distance, 1e20 for a directional light), and the visibility words over a scene with an occluder."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from renderlab_b200 import api as A
from renderlab_b200 import scenes as S


def _cells(points, normal=(0.0, 1.0, 0.0), edge=0.5):
    p = np.asarray(points, np.float32).reshape(-1, 3)
    c = np.zeros((len(p), 8), np.uint32)
    c[:, 0:3] = p.view(np.uint32)
    c[:, 3] = np.float32(edge).view(np.uint32)
    c[:, 4] = S.pack_normal(np.tile(np.asarray(normal, np.float32), (len(p), 1)))
    return c


def _light(kind, pos=(0, 0, 0), rng=0.0, travel=(0, -1, 0), outer=0.0, rgb=(1, 1, 1)):
    f = np.zeros(20, np.float32)
    f[0:3], f[3] = pos, rng
    f[4:7], f[7] = travel, outer
    f[8:11] = rgb
    w = f.view(np.uint32).copy()
    w[12] = kind
    return w


def _scene():
    """A 20 x 20 ground at y = 0 and a 2 x 2 occluder at y = 2 over the origin (GI layout)."""
    quad = lambda y, h: np.array([[-h, y, -h], [h, y, -h], [h, y, h], [-h, y, h]], np.float32)
    pos = np.concatenate([quad(0.0, 10.0), quad(2.0, 1.0)])
    idx = np.array([0, 2, 1, 0, 3, 2, 4, 6, 5, 4, 7, 6], np.uint32)
    return A.pack_scene(A.LAYOUT_GI, [A.Blas(pos, idx)], S.identity_instances(1))


def test_which_lights_reach_a_cell():
    cells = _cells([(0.0, 0.0, 0.0), (6.0, 0.0, 0.0)])
    lights = np.stack([
        _light(1, pos=(0, 5, 0), rng=100.0),                 # point above: reaches both
        _light(1, pos=(0, -5, 0), rng=100.0),                # below the surface: faces away
        _light(1, pos=(0, 5, 0), rng=1.0),                   # out of range
        _light(1, pos=(0, 5, 0), rng=100.0, rgb=(0, 0, 0)),  # black
        _light(0, travel=(0, -1, 0)),                        # directional, straight down
        _light(2, pos=(0, 5, 0), rng=100.0, travel=(0, -1, 0), outer=0.9),  # spot: cone cos 0.9
        _light(1, pos=(0, 5, 0), rng=0.0),                   # range 0: unlimited
    ])
    rays, affects = O.gi_light_rays(cells, lights)
    assert affects.tolist() == [[True, False, False, False, True, True, True],
                                [True, False, False, False, True, False, True]]
    r = rays.reshape(2, len(lights), 8)
    np.testing.assert_allclose(r[0, 0, 4:7], [0, 1, 0], atol=1e-7)    # toward the point light
    assert r[0, 0, 3] == 0.0 and abs(r[0, 0, 7] - 5.0) < 1e-5          # tmin 0, tmax its distance
    assert r[1, 4, 7] == np.float32(1e20) and np.array_equal(r[1, 4, 4:7], [0, 1, 0])
    np.testing.assert_allclose(np.linalg.norm(r[1, 0, 4:7]), 1.0, rtol=1e-6)


def test_light_rays_start_where_the_gather_rays_start():
    cells = _cells([(3.25, 0.0, -7.5), (100.0, 50.0, 1e4)], normal=(0.3, 0.9, 0.3), edge=0.25)
    lights = np.stack([_light(1, pos=(0, 100, 0), rng=0.0)])
    rays, _ = O.gi_light_rays(cells, lights)
    gather = O.gi_cell_rays(cells).reshape(2, 64, 8)
    assert np.array_equal(rays[:, 0:4].view(np.uint32), gather[:, 0, 0:4].view(np.uint32))


def test_visibility_words_over_an_occluder():
    words = _scene()
    cells = _cells([(0.0, 0.0, 0.0), (5.0, 0.0, 5.0)])
    lights = np.stack([_light(1, pos=(0, 5, 0), rng=100.0), _light(0, travel=(0, -1, 0)),
                       _light(1, pos=(0, -5, 0), rng=100.0)])
    bits = O.gi_light_bits(words, cells, lights)
    # the occluder hides both lights from the cell under it; the other cell sees them; nothing
    # reaches either from below the ground
    assert bits[:, 0].tolist() == [0b000, 0b011]


def test_visibility_words_pack_past_32_lights():
    words = _scene()
    cells = _cells([(5.0, 0.0, 5.0), (0.0, 0.0, 0.0)])
    lights = np.stack([_light(1, pos=(0, 5, 0), rng=100.0, rgb=(1, 1, 1) if l % 3 else (0, 0, 0)) for l in range(40)])
    bits = O.gi_light_bits(words, cells, lights)
    want = sum(1 << l for l in range(32) if l % 3)
    assert bits.shape == (2, 2)
    assert int(bits[0, 0]) == want and int(bits[0, 1]) == sum(1 << (l - 32) for l in range(32, 40) if l % 3)
    assert not bits[1].any()
