"""CPU tests of the C ABI: the library loads, exports every declared entry point,
and its host-side validation answers before any device work."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from tessera_b200 import _native
from tessera_b200._abi import (
    MAT_ELASTIC, MAT_FLUID, TMPM_ERR_INVALID_INPUT, TMPM_ERR_MPM_INVALID_INPUT, ParticleArrays,
    TmpmObstacle, TmpmParams, TmpmParticleArrays, TmpmSessionOptions, density_particles, make_params,
)
from tessera_b200.session import Session, TesseraError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tmpm.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tmpm_[a-z0-9_]+)\s*\(", text)))


def exported_symbols():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True, text=True, check=True)
    return sorted({line.split()[-1] for line in out.stdout.splitlines() if line.split()[-1].startswith("tmpm_")})


def test_library_loads_and_exports_every_declared_symbol():
    L = _native.lib()
    assert "sm_100a" in _native.version()
    declared = declared_symbols()
    assert len(declared) >= 25
    exported = exported_symbols()
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    for name in declared:
        assert hasattr(L, name)


def test_struct_layouts_match_header():
    # sizes follow the C declarations on LP64
    assert C.sizeof(TmpmParams) == 8 + 24 + 8 + 4 + 4 + 24 + 24
    assert C.sizeof(TmpmParticleArrays) == 8 * 18
    assert C.sizeof(TmpmObstacle) == 16 + 24 + 32 + 24 + 24 + 8 + 24 + 72 + 8 + 8
    assert C.sizeof(TmpmSessionOptions) == 32


def test_launch_shapes_are_listed_without_a_device():
    from tessera_b200 import _native

    shapes = _native.launch_shapes()
    assert shapes[0] == (256, 4, 4)  # the default: 256 particles per CTA, 4 CTAs per SM, 4^3-cell blocks
    assert len(shapes) == 6 and len(set(shapes)) == 6
    for threads, ctas, edge in shapes:
        assert threads % 32 == 0 and threads * ctas <= 2048  # whole warps; within an SM's thread slots
        assert edge in (4, 8)
    assert [s[:2] for s in shapes[:3]] == [s[:2] for s in shapes[3:]]  # each CTA shape with both block edges
    t = C.c_uint32(0)
    assert _native.lib().tmpm_launch_shape_info(len(shapes), C.byref(t), None, None) != 0


def _one_particle(material=MAT_ELASTIC, params=(2000.0, 0.2)):
    return density_particles([(0.5, 0.5, 0.5)], 0.04, 1000.0, material, params)


def test_invalid_params_rejected_before_device_work():
    # MpmParams::validate (world.rs:51-65) -> Reference(InvalidInput)
    bad = make_params(0.0)
    with pytest.raises(TesseraError) as e:
        Session(bad, _one_particle(), 1e-4)
    assert e.value.status == TMPM_ERR_MPM_INVALID_INPUT


def test_invalid_particle_rejected_before_device_work():
    p = _one_particle()
    p.mass[0] = 0.0
    with pytest.raises(TesseraError) as e:
        Session(make_params(0.1), p, 1e-4)
    assert e.value.status == TMPM_ERR_MPM_INVALID_INPUT


def test_substep_above_cfl_bound_is_invalid_input():
    # validate_resident_world rejects substep_dt > stable_timestep (gpu.rs:664-677)
    p = _one_particle(MAT_FLUID, (2000.0, 7.0, 0.1, 0.25))
    with pytest.raises(TesseraError) as e:
        Session(make_params(0.1, max_substep=1e-3), p, 2e-3)
    assert e.value.status == TMPM_ERR_INVALID_INPUT
    with pytest.raises(TesseraError) as e:
        Session(make_params(0.1), p, float("nan"))
    assert e.value.status == TMPM_ERR_INVALID_INPUT


def test_invalid_obstacle_rejected_before_device_work():
    from tessera_b200._abi import Obstacle
    with pytest.raises(TesseraError) as e:
        Session(make_params(0.1), _one_particle(), 1e-4, obstacles=[Obstacle.sphere((0, 0, 0), -1.0)])
    assert e.value.status == TMPM_ERR_MPM_INVALID_INPUT


def test_particle_arrays_roundtrip_layout():
    p = density_particles(np.random.default_rng(0).uniform(size=(7, 3)), 0.01, 10.0, MAT_ELASTIC, (1e3, 0.2))
    c = p.as_c()
    assert c.count == 7
    assert C.cast(c.position, C.POINTER(C.c_double))[3] == p.position[1, 0]
    q = ParticleArrays.concat([p, p])
    assert q.count == 14 and np.array_equal(q.position[7:], p.position)
