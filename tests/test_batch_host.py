"""CPU tests of the multi-scene batch host side: the heterogeneous scene
generator, the batch structures, the block sort key with its scene prefix, and
the admission-size estimate."""

import ctypes as C

import numpy as np

from oracle import oracle as O
from tessera_b200 import scenes
from tessera_b200._abi import MAT_FLUID, TmpmBatchOptions
from tessera_b200.batch import home_blocks, scene_bytes


def test_batch_options_layout():
    assert C.sizeof(TmpmBatchOptions) == 4 + 4 + 4 + 4 + 8


def test_heterogeneous_batch_distribution():
    scs = scenes.batch_scenes(256)
    n = np.array([s.info["particles"] for s in scs])
    res = np.array([s.info["resolution"] for s in scs])
    assert n.min() >= 4096 and n.max() <= 262144
    assert res.min() >= 32 and res.max() <= 128
    assert np.all(n == 8 * (res // 4) ** 3)  # a quarter of the domain side at 8 particles per cell
    assert 10e6 < n.sum() < 20e6
    fluids = sum(s.info["material"] == "fluid" for s in scs)
    assert 80 < fluids < 176
    youngs = [s.info["young"] for s in scs if s.info["material"] == "elastic"]
    assert min(youngs) >= 1e3 and max(youngs) <= 1e5
    # same seed, same batch
    again = scenes.batch_scenes(4)
    assert np.array_equal(again[2].particles.position, scs[2].particles.position)


def test_every_batch_scene_is_under_its_cfl_bound():
    for sc in scenes.batch_scenes(256)[::8]:
        p = sc.particles
        density = p.mass[0] / p.rest_volume[0]
        bound = O.timestep_bound(int(p.material[0]), p.material_params[0], density, (0.0, 0.0, 0.0),
                                 sc.params.cell_width)
        assert sc.dt <= bound, (sc.name, bound)
        assert np.all(p.position > 0.0) and np.all(p.position < 1.0)
        if p.material[0] == MAT_FLUID:
            assert p.material_params[0][0] == 1e4


def test_scene_prefix_orders_scenes_before_blocks():
    rng = np.random.default_rng(0)
    cells = rng.integers(-600, 600, size=(1000, 3)).astype(np.int32)
    k0 = O.block_morton_keys(cells, scene=0)
    k1 = O.block_morton_keys(cells, scene=1)
    k255 = O.block_morton_keys(cells, scene=255)
    assert k0.max() < (1 << 21) and k1.min() >= (1 << 21)
    assert np.array_equal(k1 - k0, np.full_like(k0, 1 << 21))
    assert k255.max() < 0x3FFFFFFF  # the removed-scene key sorts after every live key
    # the Morton part depends on block coordinates modulo 128 only
    assert np.array_equal(O.block_morton_keys(cells + 512), k0)


def test_admission_estimate_grows_with_particles_and_blocks():
    sc = scenes.batch_scene(7, cells=8)
    hb = home_blocks(sc.particles.position, sc.params.cell_width)
    assert 8 ** 3 // 64 <= hb <= 4 * 8 ** 3 // 64 + 64
    b = scene_bytes(sc.particles.count, hb)
    assert b > sc.particles.count * 27 * 4 * 2
    assert scene_bytes(2 * sc.particles.count, hb) > b
    assert scene_bytes(sc.particles.count, 2 * hb) > b
