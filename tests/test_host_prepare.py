"""CPU tests of scene preparation (validation and f32 packing into host memory,
`tmpm_scene_prepare`; no device work): the parallel packing pass runs in
contiguous chunks on the library's host worker pool, and its results must not
depend on how many host threads there are, nor on which chunk a rejected
particle falls in (the reported error is the first in world order, as the
reference's serial pass over the particles reports it, gpu.rs:1091-1357)."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

from tessera_b200 import scenes
from tessera_b200.batch import PreparedScene
from tessera_b200.session import TesseraError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# prepared sizes of two scenes, printed as JSON by a fresh process (the host
# thread count is read once per process)
SIZES = """
import json, sys
sys.path.insert(0, {root!r})
from tessera_b200 import scenes
from tessera_b200.batch import PreparedScene
out = []
for sc in (scenes.dam_break(scale=0.3), scenes.batch_scene(7, cells=24)):
    p = PreparedScene(sc.params, sc.particles, sc.dt)
    out.append([p.count, p.device_bytes()])
    p.close()
print(json.dumps(out))
"""


def sizes_with_threads(threads: int):
    env = dict(os.environ, TMPM_HOST_THREADS=str(threads))
    r = subprocess.run([sys.executable, "-c", SIZES.format(root=ROOT)], env=env, capture_output=True, text=True,
                       timeout=300, check=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_prepared_sizes_do_not_depend_on_host_threads():
    """Particle count and device footprint (rows plus the block pool sized from
    the distinct occupied blocks, a union over the chunks) agree for 1, 3 and 8
    host threads."""
    runs = [sizes_with_threads(t) for t in (1, 3, 8)]
    assert runs[0] == runs[1] == runs[2], runs
    assert all(count > 0 and size > 0 for count, size in runs[0])


def prepare_error(particles, params, dt) -> str:
    with pytest.raises(TesseraError) as err:
        PreparedScene(params, particles, dt)
    return str(err.value)


@pytest.mark.parametrize("early_first", [True, False])
def test_first_rejected_particle_in_world_order_is_reported(early_first):
    """Two particles the f32 packing rejects for different reasons, one near
    the start of the world and one near its end (in different chunks of the
    parallel pass): the error of the one that comes first is reported."""
    sc = scenes.dam_break(scale=0.3)
    p = sc.particles.copy()
    n = p.count
    a, b = (10, n - 10) if early_first else (n - 10, 10)
    # not representable in f32 (the force is outside the CFL bound and the MPM checks)
    force = np.zeros((n, 3)) if p.force is None else np.array(p.force, dtype=np.float64)
    force[a] = (1e39, 0.0, 0.0)
    p.force = force
    # a radius that underflows f32 to zero (positive in f64, so the MPM checks pass)
    p.radius = np.array(p.radius, dtype=np.float64)
    p.radius[b] = 1e-50
    msg = prepare_error(p, sc.params, sc.dt)
    if early_first:
        assert "particle state not representable in f32" in msg, msg
    else:
        assert "particle radius or damping invalid" in msg, msg
