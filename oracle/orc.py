"""ctypes bindings of the CPU oracle (oracle/_build/liborigami_oracle.so) that
need nothing from the product package -- test infrastructure.

The benchmark's CPU arms (the reference arm and the same-process CPU
baseline) time the oracle through this module, so they load the oracle's
library and no other native code.  The og_topology layout is restated from
include/origami_gpu.h (the oracle is compiled against that header); a system
is given as the arrays of a fixture (tests/golden/*.npz, keys "topo_<field>").
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_build", "liborigami_oracle.so")

dptr_t = C.POINTER(C.c_double)
iptr_t = C.POINTER(C.c_int32)
bptr_t = C.POINTER(C.c_int8)
INF = 1e300  # "no cutoff"


class Topology(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32),
        ("charge", dptr_t), ("rmin_half", dptr_t), ("epsilon", dptr_t), ("rmin_half_14", dptr_t),
        ("epsilon_14", dptr_t), ("gb_rho", dptr_t), ("gb_scale", dptr_t), ("mass", dptr_t), ("element", iptr_t),
        ("n_bonds", C.c_int32), ("bond_atoms", iptr_t), ("bond_k", dptr_t), ("bond_r0", dptr_t),
        ("n_angles", C.c_int32), ("angle_atoms", iptr_t), ("angle_k", dptr_t), ("angle_theta0", dptr_t),
        ("n_dihedrals", C.c_int32), ("dihedral_atoms", iptr_t), ("dihedral_term_start", iptr_t),
        ("n_dihedral_terms", C.c_int32), ("term_k", dptr_t), ("term_n", iptr_t), ("term_delta", dptr_t),
        ("n_impropers", C.c_int32), ("improper_atoms", iptr_t), ("improper_k", dptr_t), ("improper_psi0", dptr_t),
        ("n_exclusions", C.c_int32), ("exclusion_atoms", iptr_t), ("exclusion_kind", bptr_t),
        ("n_constraints", C.c_int32), ("constraint_atoms", iptr_t), ("constraint_length", dptr_t),
    ]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        srcs = [os.path.join(HERE, s) for s in ("oracle.cpp", "powersasa.cpp")]
        if not os.path.exists(SO) or any(os.path.getmtime(SO) < os.path.getmtime(s) for s in srcs):
            subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
        o = C.CDLL(SO)
        tp = C.POINTER(Topology)
        o.orc_total_force.argtypes = [tp, dptr_t, C.c_double, C.c_double, C.c_double, dptr_t]
        o.orc_total_force.restype = None
        o.orc_potential_energy.argtypes = [tp, dptr_t, C.c_double, C.c_double, dptr_t]
        o.orc_potential_energy.restype = C.c_double
        o.orc_baoab.argtypes = [tp, dptr_t, dptr_t, dptr_t, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                C.c_uint64, C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double]
        o.orc_baoab.restype = C.c_int
        o.orc_sasa_radius.argtypes = [C.c_int]
        o.orc_sasa_radius.restype = C.c_double
        o.orc_sasa_gamma.argtypes = [C.c_int, C.c_double]
        o.orc_sasa_gamma.restype = C.c_double
        o.orc_sasa_forces.argtypes = [C.c_int, dptr_t, dptr_t, dptr_t, dptr_t]
        o.orc_sasa_forces.restype = None
        _lib = o
    return _lib


def dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(dptr_t)


class System:
    """One system for the oracle: an og_topology over fixture arrays."""

    F64 = ("charge", "rmin_half", "epsilon", "rmin_half_14", "epsilon_14", "gb_rho", "gb_scale", "mass")

    def __init__(self, arrays: dict):
        keep = {}

        def arr(name, dt):
            a = np.ascontiguousarray(arrays["topo_" + name], dtype=dt)
            keep[name] = a
            return a

        t = Topology()
        t.n_atoms = len(arrays["topo_charge"])
        for f in self.F64:
            setattr(t, f, arr(f, np.float64).ctypes.data_as(dptr_t))
        t.element = arr("element", np.int32).ctypes.data_as(iptr_t)
        i32 = lambda n: arr(n, np.int32).ctypes.data_as(iptr_t)  # noqa: E731
        f64 = lambda n: arr(n, np.float64).ctypes.data_as(dptr_t)  # noqa: E731
        t.n_bonds, t.bond_atoms = len(arrays["topo_bond_k"]), i32("bonds")
        t.bond_k, t.bond_r0 = f64("bond_k"), f64("bond_r0")
        t.n_angles, t.angle_atoms = len(arrays["topo_angle_k"]), i32("angles")
        t.angle_k, t.angle_theta0 = f64("angle_k"), f64("angle_theta0")
        t.n_dihedrals = len(arrays["topo_dihedral_term_start"]) - 1
        t.dihedral_atoms, t.dihedral_term_start = i32("dihedrals"), i32("dihedral_term_start")
        t.n_dihedral_terms = len(arrays["topo_term_k"])
        t.term_k, t.term_n, t.term_delta = f64("term_k"), i32("term_n"), f64("term_delta")
        t.n_impropers, t.improper_atoms = len(arrays["topo_improper_k"]), i32("impropers")
        t.improper_k, t.improper_psi0 = f64("improper_k"), f64("improper_psi0")
        t.n_exclusions, t.exclusion_atoms = len(arrays["topo_exclusion_kind"]), i32("exclusions")
        t.exclusion_kind = arr("exclusion_kind", np.int8).ctypes.data_as(bptr_t)
        t.n_constraints, t.constraint_atoms = len(arrays["topo_constraint_length"]), i32("constraints")
        t.constraint_length = f64("constraint_length")
        self._keep = keep
        self.topo = t
        self.tp = C.pointer(t)
        self.n_atoms = t.n_atoms
        self.element = keep["element"]

    def total_force(self, x: np.ndarray, nb=INF, born=INF, gb=INF) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        f = np.zeros_like(x)
        lib().orc_total_force(self.tp, dp(x), nb, born, gb, dp(f))
        return f

    def sasa_params(self, gamma_scale: float):
        o = lib()
        rad = np.array([o.orc_sasa_radius(int(e)) for e in self.element])
        gam = np.array([o.orc_sasa_gamma(int(e), gamma_scale) for e in self.element])
        return rad, gam


def load_fixture(path: str) -> dict:
    z = np.load(path)
    return {k: z[k] for k in z.files}
