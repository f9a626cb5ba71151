"""ORACLE -- test infrastructure only.

NumPy restatement of the co-translation exit tunnel,
crates/dynamics/src/cotranslate.rs:135-154 (CylindricalTunnel::add_force):
atoms whose projection on the axis lies in [0, length] and whose distance d
from the axis exceeds the radius get -k (d - radius) along the outward
radial unit vector; the direction is used as given.
"""
from __future__ import annotations

import numpy as np


def tunnel_forces(xyz, origin, direction, radius, length, k):
    xyz = np.asarray(xyz, dtype=np.float64)
    o = np.asarray(origin, dtype=np.float64)
    d = np.asarray(direction, dtype=np.float64)
    r = xyz - o
    along = r @ d
    perp = r - np.outer(along, d)
    dist = np.linalg.norm(perp, axis=1)
    f = np.zeros_like(xyz)
    m = (along >= 0.0) & (along <= length) & (dist > radius)
    f[m] = -(perp[m] / dist[m, None]) * (k * (dist[m] - radius))[:, None]
    return f
