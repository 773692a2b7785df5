"""Multi-tick diagnostics of a fluid state: the quantities long runs are compared on.

mass (sum of fluid particle masses), kinetic energy (1/2 sum m |v|^2), centre of mass and
free-surface height (95th percentile of fluid y), all over the fluid prefix and computed in
float64 from the float32 state, plus the fraction of fluid particles outside a box.
"""
from __future__ import annotations

import numpy as np


def quantities(pos: np.ndarray, vel: np.ndarray, n_fluid: int, mass: float, box=None) -> dict:
    p = np.asarray(pos, np.float64)[:n_fluid]
    v = np.asarray(vel, np.float64)[:n_fluid]
    m = float(np.float32(mass))
    out = {
        "mass": m * n_fluid,
        "kinetic_energy": 0.5 * m * float(np.sum(v * v)),
        "com": (p.mean(axis=0) if n_fluid else np.zeros(3)).tolist(),
        "surface_height": float(np.percentile(p[:, 1], 95)) if n_fluid else 0.0,
        "max_speed": float(np.sqrt(np.max(np.sum(v * v, axis=1)))) if n_fluid else 0.0,
    }
    if box is not None:
        lo, hi = np.asarray(box[0], np.float64), np.asarray(box[1], np.float64)
        outside = np.any((p < lo) | (p > hi), axis=1)
        out["escaped_fraction"] = float(outside.mean()) if n_fluid else 0.0
    return out
