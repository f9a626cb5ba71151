"""Shared test fixtures.

The oracle (oracle/oracle.cpp, a CPU FP64 restatement of origami's force and
integrator code) is the checker for every parity test; it is built on demand
with `make -C oracle`.  GPU tests are marked `gpu` and call the product only
through the C ABI (origami_b200/liborigami_b200.so).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
# Every device buffer starts as NaN in the tests, so a kernel that reads a
# buffer before writing it fails a parity test instead of passing by luck.
os.environ.setdefault("OG_DEBUG_POISON", "1")

from origami_b200 import _ffi as F  # noqa: E402

ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liborigami_oracle.so")
LIB_SO = os.path.join(ROOT, "origami_b200", "liborigami_b200.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


_oracle = None


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        srcs = [os.path.join(ROOT, "oracle", s) for s in ("oracle.cpp", "powersasa.cpp")]
        if not os.path.exists(ORACLE_SO) or any(os.path.getmtime(ORACLE_SO) < os.path.getmtime(s) for s in srcs):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
        o = C.CDLL(ORACLE_SO)
        dp, ip = F.c_double_p, F.c_int32_p
        tp = C.POINTER(F.og_topology)
        o.orc_bonded_energy.argtypes = [tp, dp, dp]
        o.orc_bonded_energy.restype = None
        o.orc_nonbonded_energy.argtypes = [tp, dp, C.c_double, dp]
        o.orc_nonbonded_energy.restype = C.c_int
        o.orc_born_integrals.argtypes = [tp, dp, C.c_double, dp]
        o.orc_born_integrals.restype = None
        o.orc_born_radii.argtypes = [tp, dp, C.c_double, dp]
        o.orc_born_radii.restype = C.c_int
        o.orc_gb_energy.argtypes = [tp, dp, C.c_double, dp]
        o.orc_gb_energy.restype = C.c_int
        o.orc_total_force.argtypes = [tp, dp, C.c_double, C.c_double, C.c_double, dp]
        o.orc_total_force.restype = None
        o.orc_bonded_forces.argtypes = [tp, dp, dp]
        o.orc_bonded_forces.restype = None
        o.orc_potential_energy.argtypes = [tp, dp, C.c_double, C.c_double, dp]
        o.orc_potential_energy.restype = C.c_double
        o.orc_exclusion_matrix.argtypes = [C.c_int, C.c_int, ip, C.POINTER(C.c_int8)]
        o.orc_exclusion_matrix.restype = None
        o.orc_engine_normals.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, dp]
        o.orc_engine_normals.restype = None
        o.orc_baoab.argtypes = [tp, dp, dp, dp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_uint64,
                                C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double]
        o.orc_baoab.restype = C.c_int
        o.orc_shake.argtypes = [dp, dp, dp, C.c_int, ip, dp, C.c_double, C.c_int]
        o.orc_shake.restype = C.c_int
        o.orc_sasa_radius.argtypes = [C.c_int]
        o.orc_sasa_radius.restype = C.c_double
        o.orc_sasa_gamma.argtypes = [C.c_int, C.c_double]
        o.orc_sasa_gamma.restype = C.c_double
        o.orc_sasa_areas.argtypes = [C.c_int, dp, dp, dp]
        o.orc_sasa_areas.restype = None
        o.orc_sasa_forces.argtypes = [C.c_int, dp, dp, dp, dp]
        o.orc_sasa_forces.restype = None
        o.orc_sasa_forces_tangent_one_root.argtypes = [C.c_int, dp, dp, dp, dp]
        o.orc_sasa_forces_tangent_one_root.restype = None
        o.orc_shrake_rupley_areas.argtypes = [C.c_int, dp, dp, C.c_int, dp]
        o.orc_shrake_rupley_areas.restype = None
        _oracle = o
    return _oracle


def dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(F.c_double_p)


INF = 1e300  # the ABI's "no cutoff"


class Orc:
    """Thin numpy wrappers around the oracle for one chain."""

    def __init__(self, chain):
        self.chain = chain
        self.tp = chain.topology_ptr()
        self.o = oracle()

    def xyz(self, x=None):
        return np.ascontiguousarray(self.chain.positions if x is None else x, dtype=np.float64)

    def total_force(self, x=None, nb=10.0, born=20.0, gb=10.0):
        x = self.xyz(x)
        f = np.zeros_like(x)
        self.o.orc_total_force(self.tp, dp(x), nb, born, gb, dp(f))
        return f

    def bonded_force(self, x=None):
        x = self.xyz(x)
        f = np.zeros_like(x)
        self.o.orc_bonded_forces(self.tp, dp(x), dp(f))
        return f

    def energy_terms(self, x=None, nb=10.0, born=20.0):
        x = self.xyz(x)
        t = np.zeros(9)
        tot = self.o.orc_potential_energy(self.tp, dp(x), nb, born, dp(t))
        d = dict(zip(("bond", "angle", "dihedral", "improper", "lj", "coulomb", "gb", "gb_self", "gb_pair"), t))
        d["total"] = tot
        return d

    def born_integrals(self, x=None, born=20.0):
        x = self.xyz(x)
        r = np.zeros(x.shape[0])
        self.o.orc_born_integrals(self.tp, dp(x), born, dp(r))
        return r

    def born_radii(self, x=None, born=20.0):
        x = self.xyz(x)
        r = np.zeros(x.shape[0])
        self.o.orc_born_radii(self.tp, dp(x), born, dp(r))
        return r


@pytest.fixture(scope="session")
def origami():
    import origami_b200
    origami_b200.lib()
    return origami_b200


@pytest.fixture(scope="session")
def gpu_available():
    return have_gpu()


# The reference's known answers (tests/golden/known_answers.json, written by
# tests/golden/make_known_answers.py from the reference's tests, constants
# and README, each value with its source line).
_KNOWN = None


def known(key: str):
    global _KNOWN
    if _KNOWN is None:
        import json
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "known_answers.json")) as f:
            _KNOWN = json.load(f)
    return _KNOWN[key]["value"]


_HOST_GOLDEN = None


def host_golden() -> dict:
    """tests/golden/host_model.npz by case: {case: {array: value}} (the
    independent host-model oracle's output, tests/golden/make_host_golden.py)."""
    global _HOST_GOLDEN
    if _HOST_GOLDEN is None:
        z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "host_model.npz"))
        out = {}
        for key in z.files:
            case, name = key.split("/", 1)
            out.setdefault(case, {})[name] = z[key]
        _HOST_GOLDEN = out
    return _HOST_GOLDEN


class GoldenSystem:
    """An og_topology over the golden (oracle-built) arrays of one case, with
    the case's coordinates: what Orc needs, without the product's host model."""

    TOPO_FIELDS = ("charge", "rmin_half", "epsilon", "rmin_half_14", "epsilon_14", "gb_rho", "gb_scale", "mass")

    def __init__(self, case: dict, positions=None):
        self.case = case
        self._keep = {}

        def arr(name, dt):
            a = np.ascontiguousarray(case["topo_" + name], dtype=dt)
            self._keep[name] = a
            return a

        t = F.og_topology()
        t.n_atoms = int(case["counts"].sum())
        for f in self.TOPO_FIELDS:
            setattr(t, f, arr(f, np.float64).ctypes.data_as(F.c_double_p))
        t.element = arr("element", np.int32).ctypes.data_as(F.c_int32_p)
        i32 = lambda n: arr(n, np.int32).ctypes.data_as(F.c_int32_p)  # noqa: E731
        f64 = lambda n: arr(n, np.float64).ctypes.data_as(F.c_double_p)  # noqa: E731
        t.n_bonds, t.bond_atoms, t.bond_k, t.bond_r0 = len(case["topo_bond_k"]), i32("bonds"), f64("bond_k"), f64("bond_r0")
        t.n_angles, t.angle_atoms = len(case["topo_angle_k"]), i32("angles")
        t.angle_k, t.angle_theta0 = f64("angle_k"), f64("angle_theta0")
        t.n_dihedrals = len(case["topo_dihedral_term_start"]) - 1
        t.dihedral_atoms, t.dihedral_term_start = i32("dihedrals"), i32("dihedral_term_start")
        t.n_dihedral_terms = len(case["topo_term_k"])
        t.term_k, t.term_n, t.term_delta = f64("term_k"), i32("term_n"), f64("term_delta")
        t.n_impropers, t.improper_atoms = len(case["topo_improper_k"]), i32("impropers")
        t.improper_k, t.improper_psi0 = f64("improper_k"), f64("improper_psi0")
        t.n_exclusions, t.exclusion_atoms = len(case["topo_exclusion_kind"]), i32("exclusions")
        t.exclusion_kind = arr("exclusion_kind", np.int8).ctypes.data_as(F.c_int8_p)
        t.n_constraints, t.constraint_atoms = len(case["topo_constraint_length"]), i32("constraints")
        t.constraint_length = f64("constraint_length")
        self.topo = t
        self.positions = np.array(case["xyz"] if positions is None else positions, dtype=np.float64).reshape(-1, 3)
        self.n_atoms = t.n_atoms

    def topology_ptr(self):
        return C.pointer(self.topo)


def ch2_tangent_cluster(c_sq=5e-10):
    """A carbon with two hydrogens at 1.111 A (a CH2 group under SHAKE) whose
    H-C-H angle puts the two H caps on the carbon sphere in the PowerSasa
    tangent band, 0 < c_sq <= 1e-9: for equal caps of cosine c with axes at
    cos sigma, c_sq = 1 - 2 c^2 / (1 + sigma), solved for sigma.  The three
    spheres then nearly share one point, so the circles on each H sphere are
    in the band too.  An oxygen adds a generic cap.  Returns (xyz, elements)."""
    import math
    o = oracle()
    rc, rh = o.orc_sasa_radius(1), o.orc_sasa_radius(0)
    d = 1.111
    c = (d * d + rc * rc - rh * rh) / (2.0 * d * rc)
    th = math.acos(2.0 * c * c / (1.0 - c_sq) - 1.0)
    x = np.array([[0.0, 0.0, 0.0], [d, 0.0, 0.0], [d * math.cos(th), d * math.sin(th), 0.0], [-1.3, -0.9, 2.1]])
    return x, np.array([1, 0, 0, 3])
