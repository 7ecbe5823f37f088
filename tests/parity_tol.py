"""Relative FP32 tolerances for particle state, device (f32) against the f64 oracle.

Each quantity's largest per-particle error (Euclidean norm for vectors,
Frobenius norm for matrices) is divided by the scale that quantity lives on,
so one bound holds across scenes of different cell widths and speeds:

  position  max |dx|           / h                     (in cells)
  velocity  max |dv|           / max |v|
  affine C  max |dC|_F         / max(max |C|_F, max |v| / h)
  F         max |dF|_F         / max |F|_F

C is a velocity gradient across a cell, so its natural scale is |v| / h: the
floor keeps the bound meaningful where C itself is round-off (a block in free
fall has C = 0 exactly in f64).
"""

import numpy as np

# one to a few substeps (the per-substep bound) and after long runs (bounded drift)
PER_SUBSTEP = dict(position=1e-4, velocity=1e-4, affine=1e-3, deformation=1e-5)


def _mat_norm(a):
    return np.linalg.norm(np.asarray(a).reshape(-1, 9), axis=1)


def rel_errors(expected, actual, h):
    vmax = np.linalg.norm(expected.velocity, axis=1).max()
    cscale = max(_mat_norm(expected.affine).max(), vmax / h)
    return dict(
        position=np.linalg.norm(expected.position - actual.position, axis=1).max() / h,
        velocity=np.linalg.norm(expected.velocity - actual.velocity, axis=1).max() / max(vmax, 1e-30),
        affine=_mat_norm(expected.affine - actual.affine).max() / max(cscale, 1e-30),
        deformation=_mat_norm(expected.deformation - actual.deformation).max() / _mat_norm(expected.deformation).max(),
    )


def assert_rel_close(expected, actual, h, tol=PER_SUBSTEP, label=""):
    err = rel_errors(expected, actual, h)
    print(f"PARITY {label} " + " ".join(f"{k}={v:.3e}" for k, v in err.items()))
    bad = {k: (err[k], tol[k]) for k in tol if not err[k] <= tol[k]}
    assert not bad, f"{label}: relative error above tolerance {bad}"
    return err


def _cell_keys(cells):
    c = np.asarray(cells, dtype=np.int64) + (1 << 20)
    return (c[:, 0] << 42) | (c[:, 1] << 21) | c[:, 2]


def assert_grid_close(cells, mm, keys, vals, tol_mass=1e-5, tol_momentum=1e-5, label=""):
    """Device P2G nodes (cells, float4 mass+momentum) against the oracle's
    (keys, vals): every node within `tol` of the largest node value of that
    quantity.  A node present on one side only counts as zero on the other:
    the device lists nodes whose mass is non-zero after the fixed-point
    accumulation, so a node that only the far tail of a weight reaches (mass
    below one quantum) can be absent there; the bound covers it like any
    other node."""
    kd, ko = _cell_keys(cells), _cell_keys(keys[:, :3])
    union = np.union1d(kd, ko)
    dev = np.zeros((len(union), 4))
    ref = np.zeros((len(union), 4))
    dev[np.searchsorted(union, kd)] = np.asarray(mm, dtype=np.float64)
    ref[np.searchsorted(union, ko)] = vals[:, :4]
    dm = np.abs(dev[:, 0] - ref[:, 0]).max() / ref[:, 0].max()
    pscale = np.abs(ref[:, 1:]).max()
    dp = np.abs(dev[:, 1:] - ref[:, 1:]).max() / pscale if pscale > 0 else np.abs(dev[:, 1:]).max()
    only = len(union) - min(len(kd), len(ko))
    print(f"GRID {label} nodes={len(ko)} device={len(kd)} one-sided={only} mass={dm:.3e} momentum={dp:.3e}")
    assert dm < tol_mass and dp < tol_momentum, (label, dm, dp)
    # one-sided nodes are few (weight tails below one quantum)
    assert only <= 1e-4 * len(ko) + 8, (label, only)
    return dm, dp
