"""CPU check of the product's reverse-mode PowerSasa term gradients
(origami_b200/csrc/engine/sasa_geom.h, the math the GPU force kernel runs)
against the oracle's forward-mode directional derivatives, one tangent per
(role, axis), on random cap geometries: agreement to 1e-9 relative."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, dp, oracle

SHIM_SRC = os.path.join(ROOT, "tests", "sasa_geom_shim.cpp")
SHIM_SO = os.path.join(ROOT, "tests", "_build", "libsasa_geom_shim.so")
HEADER = os.path.join(ROOT, "origami_b200", "csrc", "engine", "sasa_geom.h")


@pytest.fixture(scope="module")
def shim():
    stale = not os.path.exists(SHIM_SO) or any(os.path.getmtime(SHIM_SO) < os.path.getmtime(s)
                                                for s in (SHIM_SRC, HEADER))
    if stale:
        os.makedirs(os.path.dirname(SHIM_SO), exist_ok=True)
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
        subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-o", SHIM_SO, SHIM_SRC], check=True)
    lib = C.CDLL(SHIM_SO)
    d = C.POINTER(C.c_double)
    lib.shim_arc_gradient.argtypes = [d, d, C.c_int, C.c_int, C.c_double, C.c_int, d]
    lib.shim_vertex_gradient.argtypes = [d, d, C.c_int, d]
    o = oracle()
    o.orc_arc_term_jvps.argtypes = [d, d, C.c_int, C.c_int, C.c_double, C.c_int, d]
    o.orc_vertex_term_jvps.argtypes = [d, d, C.c_int, d]
    return lib


RADII = [2.6, 2.92, 2.95, 3.1, 3.2]


def random_centres(rng, n):
    p = np.zeros((n, 3))
    for k in range(1, n):
        v = rng.normal(size=3)
        p[k] = v / np.linalg.norm(v) * rng.uniform(1.0, 5.5)
    return p


def test_arc_term_gradient_matches_directional_derivatives(shim):
    rng = np.random.default_rng(7)
    o = oracle()
    checked = 0
    for _ in range(3000):
        p = np.ascontiguousarray(random_centres(rng, 4))
        r = np.ascontiguousarray(rng.choice(RADII, 4))
        ss, se = (int(s) for s in rng.choice([-1, 1], 2))
        theta = float(rng.uniform(-2 * np.pi, 0))
        vertexed = int(rng.integers(0, 4) > 0)
        want, got = np.zeros(12), np.zeros(12)
        o.orc_arc_term_jvps(dp(p), dp(r), ss, se, theta, vertexed, dp(want))
        shim.shim_arc_gradient(dp(p), dp(r), ss, se, theta, vertexed, dp(got))
        scale = max(np.abs(want).max(), 1e-3)
        assert np.abs(got - want).max() <= 1e-9 * scale, (p, r, ss, se, vertexed, got, want)
        checked += np.abs(want).max() > 0
    assert checked > 2000


def test_vertex_term_gradient_matches_directional_derivatives(shim):
    rng = np.random.default_rng(8)
    o = oracle()
    nonzero = 0
    for _ in range(3000):
        p = np.ascontiguousarray(random_centres(rng, 3))
        r = np.ascontiguousarray(rng.choice(RADII, 3))
        sign = int(rng.choice([-1, 1]))
        want, got = np.zeros(9), np.zeros(9)
        o.orc_vertex_term_jvps(dp(p), dp(r), sign, dp(want))
        shim.shim_vertex_gradient(dp(p), dp(r), sign, dp(got))
        scale = max(np.abs(want).max(), 1e-3)
        assert np.abs(got - want).max() <= 1e-9 * scale, (p, r, sign, got, want)
        nonzero += np.abs(want).max() > 0
    assert nonzero > 500
