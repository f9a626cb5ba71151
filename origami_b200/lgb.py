"""Learned Born radii: the Python face of the og_lgb_* entries.

The network maps an atom's 80 inputs (64 environment descriptors and 16
features of the atom itself) to y = log(R_plainGB / R_cfa); see
include/origami_gpu.h for the inputs, the Coulomb-field baseline R_cfa and
the parameter layout.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi as F
from . import _check, lib

N_PARAMS = F.LGB_N_PARAMS
N_INPUT = F.LGB_N_INPUT
HIDDEN = 128

# offsets into the flat parameter vector (W row-major, out x in)
OFF_W1 = 0
OFF_B1 = OFF_W1 + HIDDEN * N_INPUT
OFF_W2 = OFF_B1 + HIDDEN
OFF_B2 = OFF_W2 + HIDDEN * HIDDEN
OFF_W3 = OFF_B2 + HIDDEN
OFF_B3 = OFF_W3 + HIDDEN * HIDDEN
OFF_W4 = OFF_B3 + HIDDEN
OFF_B4 = OFF_W4 + HIDDEN
OFF_V = OFF_B4 + 1
N_SELF = N_INPUT - 64
assert OFF_V + N_SELF == N_PARAMS


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(F.c_float_p)


def unpack(params: np.ndarray) -> dict:
    p = np.asarray(params, dtype=np.float32)
    return {
        "W1": p[OFF_W1:OFF_B1].reshape(HIDDEN, N_INPUT), "b1": p[OFF_B1:OFF_W2],
        "W2": p[OFF_W2:OFF_B2].reshape(HIDDEN, HIDDEN), "b2": p[OFF_B2:OFF_W3],
        "W3": p[OFF_W3:OFF_B3].reshape(HIDDEN, HIDDEN), "b3": p[OFF_B3:OFF_W4],
        "w4": p[OFF_W4:OFF_B4], "b4": p[OFF_B4:OFF_V], "v": p[OFF_V:N_PARAMS],
    }


def init_params(seed: int = 0) -> np.ndarray:
    p = np.empty(N_PARAMS, dtype=np.float32)
    _check(lib().og_lgb_init_params(seed & 0xFFFFFFFFFFFFFFFF, _fptr(p)))
    return p


def loss_and_gradient(x: np.ndarray, target: np.ndarray, params: np.ndarray) -> tuple[float, np.ndarray]:
    x = np.ascontiguousarray(x, dtype=np.float32)
    t = np.ascontiguousarray(target, dtype=np.float32)
    p = np.ascontiguousarray(params, dtype=np.float32)
    g = np.empty(N_PARAMS, dtype=np.float32)
    loss = C.c_double()
    _check(lib().og_lgb_loss_and_gradient(_fptr(x), _fptr(t), x.shape[0], _fptr(p), C.byref(loss), _fptr(g)))
    return loss.value, g


def train(x: np.ndarray, target: np.ndarray, params: np.ndarray, steps: int, batch: int = 8192,
          lr: float = 1e-3, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Adam on the GPU; returns (trained parameters, per-step batch loss)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    t = np.ascontiguousarray(target, dtype=np.float32)
    p = np.array(params, dtype=np.float32, copy=True)
    hist = np.empty(max(steps, 1), dtype=np.float32)
    _check(lib().og_lgb_train(_fptr(x), _fptr(t), x.shape[0], steps, batch, lr, seed & 0xFFFFFFFFFFFFFFFF,
                              _fptr(p), _fptr(hist)))
    return p, hist[:steps]


# ------------------------------------------------------------ engine hooks

def samples(engine, sys: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """(x [n_atoms x 80], target [n_atoms]) of one system (sys = -1: all
    systems, concatenated) at the current positions."""
    n = sum(engine._n_atoms) if sys == -1 else engine._n_atoms[sys]
    x = np.empty((n, N_INPUT), dtype=np.float32)
    t = np.empty(n, dtype=np.float32)
    _check(lib().og_lgb_samples(engine._h, sys, _fptr(x), _fptr(t)))
    return x, t


def set_params(engine, params: np.ndarray) -> None:
    p = np.ascontiguousarray(params, dtype=np.float32)
    _check(lib().og_lgb_set_params(engine._h, _fptr(p)))


def set_judge(engine, interval_steps: int = 500, tolerance: float = 1e-3) -> None:
    _check(lib().og_lgb_set_judge(engine._h, interval_steps, tolerance))


def status(engine) -> dict:
    active, judged, err = C.c_int32(), C.c_int32(), C.c_double()
    _check(lib().og_lgb_status(engine._h, C.byref(active), C.byref(judged), C.byref(err)))
    return {"active": bool(active.value), "judged": judged.value, "last_error": err.value}


def judge(engine) -> float:
    err = C.c_double()
    _check(lib().og_lgb_judge(engine._h, C.byref(err)))
    return err.value
