"""ORACLE -- test infrastructure only.

NumPy float64 restatement of the learned-Born-radius inputs defined in
include/origami_gpu.h: the 64 environment descriptors (16 Gaussian shells x
4 element classes, partner-radius weighted, cosine cutoff at 12 A) as
x = log(1 + D) followed by the 16 self features (class one-hot, rho~, HCT
scale, rho~/R_cfa, log R_cfa, 0, log(rho~/R_cfa), zeros), and the
Coulomb-field radius in its
pairwise (Hawkins-Cramer-Truhlar) form 1/R_cfa = max(1/rho~_i - sum_j fc
I_HCT, 1/30).
These are this project's definitions (the reference has no learned radii).
"""
from __future__ import annotations

import numpy as np

CLASS_OF_ELEMENT = np.array([3, 0, 1, 2, 1, 0])  # H, C, N, O, P, S -> C/S 0, N/P 1, O 2, H 3
MU = 1.5 + 0.7 * np.arange(16)
SIGMA = 0.7
CUTOFF = 12.0


def hct(r, rti, sj):
    """HCT pairwise descreening integral (standard closed form)."""
    out = np.zeros_like(r)
    ok = rti < r + sj
    l = np.maximum(rti, np.abs(r - sj))
    u = r + sj
    with np.errstate(divide="ignore", invalid="ignore"):
        t = 0.5 * (1 / l - 1 / u + 0.25 * r * (1 / u**2 - 1 / l**2) + 0.5 / r * np.log(l / u)
                   + 0.25 * sj**2 / r * (1 / l**2 - 1 / u**2))
        t = t + np.where(rti < sj - r, 2.0 * (1 / rti - 1 / l), 0.0)
    return np.where(ok, t, 0.0)


def descriptors(xyz: np.ndarray, element: np.ndarray, rho: np.ndarray, rho_tilde: np.ndarray,
                srho: np.ndarray):
    xyz = np.asarray(xyz, dtype=np.float64)
    n = xyz.shape[0]
    cls = CLASS_OF_ELEMENT[np.asarray(element)]
    r = np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=2)
    mask = (r < CUTOFF) & ~np.eye(n, dtype=bool)
    fc = np.where(mask, 0.5 * (np.cos(np.pi * r / CUTOFF) + 1.0), 0.0)
    w = fc * np.asarray(rho)[None, :]
    d = np.zeros((n, 64))
    for s in range(16):
        g = w * np.exp(-(r - MU[s]) ** 2 / (2 * SIGMA * SIGMA))
        for c in range(4):
            d[:, 16 * c + s] = (g * (cls == c)[None, :]).sum(1)
    rti = np.asarray(rho_tilde)[:, None]
    sj = np.asarray(srho)[None, :]
    rr = np.where(mask, r, 1.0)
    cfa = np.where(mask, fc * hct(rr, rti + 0 * rr, sj + 0 * rr), 0.0).sum(1)
    rt = np.asarray(rho_tilde, dtype=np.float64)
    rcfa = 1.0 / np.maximum(1.0 / rt - cfa, 1.0 / 30.0)
    selfx = np.zeros((n, 16))
    selfx[np.arange(n), cls] = 1.0
    selfx[:, 4] = rt
    selfx[:, 5] = np.asarray(srho) / rt
    selfx[:, 6] = rt / rcfa
    selfx[:, 7] = np.log(rcfa)
    selfx[:, 9] = np.log(rt / rcfa)
    return np.concatenate([np.log1p(d), selfx], axis=1), rcfa
