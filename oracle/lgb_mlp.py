"""ORACLE -- test infrastructure only.

NumPy restatement of the learned-Born-radius network and its loss
gradient, with the tensor-core kernels' rounding points: every GEMM operand
is rounded to bfloat16 (round to nearest even) and products accumulate in
float64 here (float32 on the GPU); bias adds, SiLU, the 128 -> 1 head and
the loss stay in float32/float64.  The network has no counterpart in the
reference (it is this project's addition), so the oracle restates the
definition in include/origami_gpu.h rather than reference code.
"""
from __future__ import annotations

import numpy as np

HIDDEN, N_INPUT = 128, 80
N_SELF = N_INPUT - 64
N_PARAMS = HIDDEN * N_INPUT + HIDDEN + 2 * (HIDDEN * HIDDEN + HIDDEN) + HIDDEN + 1 + N_SELF


def bf16(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unpack(p: np.ndarray) -> dict:
    p = np.asarray(p, dtype=np.float64)
    o, d = 0, {}
    for name, shape in (("W1", (HIDDEN, N_INPUT)), ("b1", (HIDDEN,)), ("W2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
                        ("W3", (HIDDEN, HIDDEN)), ("b3", (HIDDEN,)), ("w4", (HIDDEN,)), ("b4", (1,)),
                        ("v", (N_SELF,))):
        n = int(np.prod(shape))
        d[name] = p[o:o + n].reshape(shape)
        o += n
    return d


def forward(p: np.ndarray, x: np.ndarray) -> dict:
    w = unpack(p)
    z1 = bf16(x) @ bf16(w["W1"]).T + w["b1"]
    h1 = silu(z1)
    z2 = bf16(h1) @ bf16(w["W2"]).T + w["b2"]
    h2 = silu(z2)
    z3 = bf16(h2) @ bf16(w["W3"]).T + w["b3"]
    h3 = silu(z3)
    y = h3 @ w["w4"] + w["b4"][0] + np.asarray(x, np.float64)[:, 64:] @ w["v"]
    return {"x": x, "z1": z1, "h1": h1, "z2": z2, "h2": h2, "z3": z3, "h3": h3, "y": y}


def loss_and_gradient(p: np.ndarray, x: np.ndarray, t: np.ndarray) -> tuple[float, np.ndarray]:
    w = unpack(p)
    f = forward(p, x)
    b = x.shape[0]
    d = f["y"] - t
    loss = float(np.mean(d * d))
    dy = 2.0 * d / b
    g = {"w4": dy @ f["h3"], "b4": np.array([dy.sum()]), "v": dy @ np.asarray(x, np.float64)[:, 64:]}
    dz3 = dy[:, None] * w["w4"][None, :] * silu_grad(f["z3"])
    g["b3"] = dz3.sum(0)
    g["W3"] = bf16(dz3).T @ bf16(f["h2"])
    dz2 = (bf16(dz3) @ bf16(w["W3"])) * silu_grad(f["z2"])
    g["b2"] = dz2.sum(0)
    g["W2"] = bf16(dz2).T @ bf16(f["h1"])
    dz1 = (bf16(dz2) @ bf16(w["W2"])) * silu_grad(f["z1"])
    g["b1"] = dz1.sum(0)
    g["W1"] = bf16(dz1).T @ bf16(x)
    flat = np.concatenate([g[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4", "v")])
    return loss, flat
