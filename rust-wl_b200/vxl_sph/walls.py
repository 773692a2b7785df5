"""Host side of the provider walls for any ProviderColliders (voxel terrain, meshes, splats,
SDFs): the contact tables the device reads every substep of a tick.

This follows the reference's GPU tier: once per tick the stepper reads the fluid positions
back from the device, queries the providers on the host, and uploads two sparse tables
(crates/vxl-phys-gpu/src/pipeline/stepper.rs:118-137, gather_in in
crates/vxl-phys-gpu/src/pipeline/walls.rs:164-215):

  mirror     contacts_point(bid, p, h), planes with 0 < sdf < h   (wall_planes_in's rule)
  projection contacts_point_boundary(bid, p, h), planes with sdf < h

with sdf = (p - point) . normal in float32, at most 8 planes per particle over all
providers, a provider skipped when p lies outside its bounds grown by h.

A provider set here is any object with the reference trait's methods
(crates/vxl-phys-core/src/interop.rs:166-223):
  bounds(bid) -> ((x, y, z), (x, y, z)) or None
  contacts_point(bid, p, probe) -> list of (point (3,), outward normal (3,))
  contacts_point_boundary(bid, p, probe) -> same (optional; defaults to contacts_point)
"""
from __future__ import annotations

import numpy as np

F = np.float32
MIRROR, PROJECT = 0, 1
MAX_PLANES = 8


def _sdf(p, point, normal):
    # (p - point).dot(normal), float32 left to right (crates/vxl-phys-core/src/math.rs)
    d = (np.asarray(p, F) - np.asarray(point, F)).astype(F)
    n = np.asarray(normal, F)
    return F(F(F(d[0] * n[0]) + F(d[1] * n[1])) + F(d[2] * n[2]))


def gather_contacts(boundaries, h: float, ps: np.ndarray, providers, side: int):
    """(ids, start, planes) of one side for fluid positions ps (n, 3) float32."""
    h = F(h)
    ids, start, planes = [], [0], []
    query_name = "contacts_point" if side == MIRROR else "contacts_point_boundary"
    for i, p in enumerate(np.asarray(ps, F)):
        np_ = 0
        for bid in boundaries:
            bb = providers.bounds(bid)
            if bb is not None:
                lo, hi = (np.asarray(x, F) for x in bb)
                if (p[0] < lo[0] - h or p[0] > hi[0] + h or p[1] < lo[1] - h or p[1] > hi[1] + h
                        or p[2] < lo[2] - h or p[2] > hi[2] + h):
                    continue
            query = getattr(providers, query_name, None) or providers.contacts_point
            for point, normal in query(bid, p, h):
                sdf = _sdf(p, point, normal)
                keep = (F(0) < sdf < h) if side == MIRROR else (sdf < h)
                if keep and np_ < MAX_PLANES:
                    planes.append(np.concatenate([np.asarray(point, F), np.asarray(normal, F)]))
                    np_ += 1
        if np_:
            ids.append(i)
            start.append(len(planes))
    planes_arr = np.asarray(planes, F).reshape(-1, 6)
    return np.asarray(ids, np.uint32), np.asarray(start, np.uint32), planes_arr
