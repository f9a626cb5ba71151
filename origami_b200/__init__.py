"""origami_b200: B200-native force-and-integrate engine for origami's MD hot path.

The product is the C ABI in include/origami_gpu.h, implemented by
``liborigami_b200.so`` (host C++ + sm_100a CUDA, built by
``python -m origami_b200.build``).  This module is the thin Python host on top
of it, mirroring origami's Rust API for the hot path:

    Chain.build / build_extended_chain     geom/src/builder.rs:50-90
    Chain.topology()                        geom/src/topology_graph.rs:134 + ForceScratch params
    Engine.total_force                      energy/src/forces.rs:78 total_force_with_scratch
    Engine.energies                         dynamics/src/remd.rs:529 potential_energy
    run_langevin                            dynamics/src/langevin.rs:128
    run_remd                                dynamics/src/remd.rs:136

Loading fails loudly when the library is missing; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import _ffi as F

__all__ = [
    "OrigamiError", "lib", "Chain", "Engine", "Params", "build_extended_chain",
    "run_langevin", "run_remd", "LangevinOptions", "RemdOptions", "Xoshiro256pp",
]

_PKG = os.path.dirname(os.path.abspath(__file__))
# ORIGAMI_B200_LIB selects another build of the library (tuning sweeps).
LIB_PATH = os.environ.get("ORIGAMI_B200_LIB") or os.path.join(_PKG, "liborigami_b200.so")
DATA_DIR = os.path.join(_PKG, "data")

BOLTZMANN_KJ_PER_MOL_K = 8.314_462_618e-3   # dynamics/src/langevin.rs:44
ACCEL_FACTOR = 1.0e-4                        # dynamics/src/langevin.rs:47


class OrigamiError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{F.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """The loaded C library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OrigamiError(F.OG_OK - 1, f"{LIB_PATH} missing: run `python -m origami_b200.build`")
        l = C.CDLL(LIB_PATH)
        F.declare(l)
        st = l.og_set_data_dir(DATA_DIR.encode())
        if st != F.OG_OK:
            raise OrigamiError(st, l.og_last_error().decode())
        _lib = l
    return _lib


def _check(st: int) -> None:
    if st != F.OG_OK:
        raise OrigamiError(st, lib().og_last_error().decode())


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(F.c_double_p)


# --------------------------------------------------------------- host model

class Chain:
    """An all-atom chain built by the library's NeRF builder (owns an og_chain)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    @classmethod
    def build(cls, sequence: str, phi: float = math.nan, psi: float = math.nan,
              omega: float = math.nan) -> "Chain":
        h = C.c_void_p()
        _check(lib().og_chain_build(sequence.encode(), phi, psi, omega, C.byref(h)))
        return cls(h)

    @classmethod
    def from_structure(cls, residues: str, atoms_per_residue, names, xyz, elements=None,
                       chains: str | None = None) -> "Chain":
        """A chain from a structure held by the caller (og_chain_from_structure):
        one-letter residue codes, atom counts per residue, atom names in
        wwPDB v3.3 form, positions (n x 3) and optionally element codes
        (0 H .. 5 S) and one chain id per residue."""
        counts = np.ascontiguousarray(atoms_per_residue, dtype=np.int32)
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        if len(residues) != counts.shape[0] or int(counts.sum()) != x.shape[0] or len(names) != x.shape[0]:
            raise ValueError("residue, count, name and position arrays disagree")
        name_buf = b"".join(n.encode()[:8].ljust(8, b"\0") for n in names)
        el = None
        if elements is not None:
            el = np.ascontiguousarray(elements, dtype=np.int32)
        h = C.c_void_p()
        _check(lib().og_chain_from_structure(
            len(residues), residues.encode(), None if chains is None else chains.encode(),
            counts.ctypes.data_as(F.c_int32_p), name_buf,
            None if el is None else el.ctypes.data_as(F.c_int32_p), _dptr(x), C.byref(h)))
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.og_chain_free(h)
            self._h = None

    def append(self, residue: str, phi: float = math.nan, psi: float = math.nan, omega: float = math.nan) -> None:
        _check(lib().og_chain_append(self._h, residue.encode()[:1], phi, psi, omega))

    @property
    def n_atoms(self) -> int:
        n = C.c_int32()
        _check(lib().og_chain_n_atoms(self._h, C.byref(n)))
        return n.value

    @property
    def n_residues(self) -> int:
        n = C.c_int32()
        _check(lib().og_chain_n_residues(self._h, C.byref(n)))
        return n.value

    @property
    def positions(self) -> np.ndarray:
        x = np.empty((self.n_atoms, 3))
        _check(lib().og_chain_get_positions(self._h, _dptr(x)))
        return x

    @positions.setter
    def positions(self, xyz: np.ndarray) -> None:
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        if x.shape[0] != self.n_atoms:
            raise ValueError("position array has the wrong number of atoms")
        _check(lib().og_chain_set_positions(self._h, _dptr(x)))

    def write_pdb(self, path: str, xyz: np.ndarray | None = None, title: str = "") -> None:
        """One-model PDB of the chain (io/src/pdb.rs write_pdb); xyz defaults
        to the chain's own positions."""
        ptr = None
        if xyz is not None:
            x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
            if x.shape[0] != self.n_atoms:
                raise ValueError("position array has the wrong number of atoms")
            ptr = _dptr(x)
        _check(lib().og_pdb_write(self._h, ptr, title.encode(), os.fsencode(path)))

    def topology_ptr(self) -> C.POINTER(F.og_topology):
        p = C.POINTER(F.og_topology)()
        _check(lib().og_chain_topology(self._h, C.byref(p)))
        return p

    def topology(self) -> "Topology":
        return Topology.from_struct(self.topology_ptr().contents)

    def atom_info(self, i: int) -> tuple[int, int, str]:
        r, t = C.c_int32(), C.c_int32()
        name = C.create_string_buffer(8)
        _check(lib().og_chain_atom_info(self._h, i, C.byref(r), C.byref(t), name))
        return r.value, t.value, name.value.decode()

    def missing_params(self) -> int:
        m = C.c_int32()
        _check(lib().og_chain_missing_params(self._h, C.byref(m)))
        return m.value


def build_extended_chain(sequence: str) -> Chain:
    """geom::build_extended_chain: phi -120, psi 140, omega 180 degrees."""
    return Chain.build(sequence)


def topology_extends(base, grown) -> tuple[bool, str]:
    """Whether `grown` (Chain or Topology) extends `base` so that an engine
    system built from base can take it by Engine.append_atoms, and if not,
    why (og_topology_extends; host only)."""
    keep = []

    def ptr(t):
        if isinstance(t, Chain):
            return t.topology_ptr()
        s = t.to_struct()
        keep.append(s)
        return C.pointer(s)

    ok = C.c_int32()
    _check(lib().og_topology_extends(ptr(base), ptr(grown), C.byref(ok)))
    return bool(ok.value), ("" if ok.value else lib().og_last_error().decode())


@dataclass
class Topology:
    """NumPy copy of an og_topology (per-atom params, term lists, exclusions)."""
    charge: np.ndarray
    rmin_half: np.ndarray
    epsilon: np.ndarray
    rmin_half_14: np.ndarray
    epsilon_14: np.ndarray
    gb_rho: np.ndarray
    gb_scale: np.ndarray
    mass: np.ndarray
    element: np.ndarray
    bonds: np.ndarray
    bond_k: np.ndarray
    bond_r0: np.ndarray
    angles: np.ndarray
    angle_k: np.ndarray
    angle_theta0: np.ndarray
    dihedrals: np.ndarray
    dihedral_term_start: np.ndarray
    term_k: np.ndarray
    term_n: np.ndarray
    term_delta: np.ndarray
    impropers: np.ndarray
    improper_k: np.ndarray
    improper_psi0: np.ndarray
    exclusions: np.ndarray
    exclusion_kind: np.ndarray
    constraints: np.ndarray
    constraint_length: np.ndarray
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_atoms(self) -> int:
        return int(self.charge.shape[0])

    @staticmethod
    def from_struct(t: F.og_topology) -> "Topology":
        def arr(p, n, dt=np.float64, w=1):
            if n == 0:
                return np.zeros((0, w) if w > 1 else (0,), dtype=dt)
            a = np.ctypeslib.as_array(p, (n * w,)).astype(dt, copy=True)
            return a.reshape(n, w) if w > 1 else a
        n = t.n_atoms
        return Topology(
            charge=arr(t.charge, n), rmin_half=arr(t.rmin_half, n), epsilon=arr(t.epsilon, n),
            rmin_half_14=arr(t.rmin_half_14, n), epsilon_14=arr(t.epsilon_14, n),
            gb_rho=arr(t.gb_rho, n), gb_scale=arr(t.gb_scale, n), mass=arr(t.mass, n),
            element=arr(t.element, n, np.int32),
            bonds=arr(t.bond_atoms, t.n_bonds, np.int32, 2), bond_k=arr(t.bond_k, t.n_bonds),
            bond_r0=arr(t.bond_r0, t.n_bonds),
            angles=arr(t.angle_atoms, t.n_angles, np.int32, 3), angle_k=arr(t.angle_k, t.n_angles),
            angle_theta0=arr(t.angle_theta0, t.n_angles),
            dihedrals=arr(t.dihedral_atoms, t.n_dihedrals, np.int32, 4),
            dihedral_term_start=arr(t.dihedral_term_start, t.n_dihedrals + 1, np.int32),
            term_k=arr(t.term_k, t.n_dihedral_terms), term_n=arr(t.term_n, t.n_dihedral_terms, np.int32),
            term_delta=arr(t.term_delta, t.n_dihedral_terms),
            impropers=arr(t.improper_atoms, t.n_impropers, np.int32, 4),
            improper_k=arr(t.improper_k, t.n_impropers), improper_psi0=arr(t.improper_psi0, t.n_impropers),
            exclusions=arr(t.exclusion_atoms, t.n_exclusions, np.int32, 2),
            exclusion_kind=arr(t.exclusion_kind, t.n_exclusions, np.int8),
            constraints=arr(t.constraint_atoms, t.n_constraints, np.int32, 2),
            constraint_length=arr(t.constraint_length, t.n_constraints),
        )

    def to_struct(self) -> F.og_topology:
        """An og_topology pointing into this object's arrays (kept alive by self)."""
        def p(a, ct):
            a = np.ascontiguousarray(a)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(ct))
        t = F.og_topology()
        t.n_atoms = self.n_atoms
        for name in ("charge", "rmin_half", "epsilon", "rmin_half_14", "epsilon_14", "gb_rho", "gb_scale", "mass"):
            setattr(t, name, p(getattr(self, name).astype(np.float64), C.c_double))
        t.element = p(self.element.astype(np.int32), C.c_int32)
        t.n_bonds = len(self.bond_k); t.bond_atoms = p(self.bonds.astype(np.int32), C.c_int32)
        t.bond_k = p(self.bond_k, C.c_double); t.bond_r0 = p(self.bond_r0, C.c_double)
        t.n_angles = len(self.angle_k); t.angle_atoms = p(self.angles.astype(np.int32), C.c_int32)
        t.angle_k = p(self.angle_k, C.c_double); t.angle_theta0 = p(self.angle_theta0, C.c_double)
        t.n_dihedrals = len(self.dihedrals); t.dihedral_atoms = p(self.dihedrals.astype(np.int32), C.c_int32)
        t.dihedral_term_start = p(self.dihedral_term_start.astype(np.int32), C.c_int32)
        t.n_dihedral_terms = len(self.term_k); t.term_k = p(self.term_k, C.c_double)
        t.term_n = p(self.term_n.astype(np.int32), C.c_int32); t.term_delta = p(self.term_delta, C.c_double)
        t.n_impropers = len(self.improper_k); t.improper_atoms = p(self.impropers.astype(np.int32), C.c_int32)
        t.improper_k = p(self.improper_k, C.c_double); t.improper_psi0 = p(self.improper_psi0, C.c_double)
        t.n_exclusions = len(self.exclusion_kind)
        t.exclusion_atoms = p(self.exclusions.astype(np.int32), C.c_int32)
        t.exclusion_kind = p(self.exclusion_kind.astype(np.int8), C.c_int8)
        t.n_constraints = len(self.constraint_length)
        t.constraint_atoms = p(self.constraints.astype(np.int32), C.c_int32)
        t.constraint_length = p(self.constraint_length, C.c_double)
        return t


# ------------------------------------------------------------------- engine

NO_CUTOFF = math.inf


@dataclass
class Params:
    """og_params; defaults are origami's integrator-path values."""
    nb_cutoff: float = 10.0
    born_cutoff: float = 20.0
    gb_force_cutoff: float = 10.0
    dt_fs: float = 1.0
    friction_ps_inv: float = 1.0
    constrain_h_bonds: bool = False
    shake_max_iters: int = 64
    shake_tol_sq: float = 1e-6
    include_sasa: bool = False
    sasa_gamma_scale: float = 1.0
    born_mode: int = 0
    seed: int = 0

    @staticmethod
    def all_pairs(**kw) -> "Params":
        """No cutoffs anywhere (bare Coulomb, all-pairs Born and GB)."""
        return Params(nb_cutoff=NO_CUTOFF, born_cutoff=NO_CUTOFF, gb_force_cutoff=NO_CUTOFF, **kw)

    def to_struct(self) -> F.og_params:
        c = lambda v: 1e300 if math.isinf(v) else float(v)  # noqa: E731
        return F.og_params(c(self.nb_cutoff), c(self.born_cutoff), c(self.gb_force_cutoff), self.dt_fs,
                           self.friction_ps_inv, int(self.constrain_h_bonds), self.shake_max_iters,
                           self.shake_tol_sq, int(self.include_sasa), self.sasa_gamma_scale, self.born_mode,
                           self.seed & 0xFFFFFFFFFFFFFFFF)


ENERGY_TERMS = ("bond", "angle", "dihedral", "improper", "lj", "coulomb", "gb", "gb_self", "gb_pair", "sasa", "total")


class Engine:
    """A set of systems on one GPU (owns an og_engine)."""

    def __init__(self, params: Params | None = None):
        self.params = params or Params()
        h = C.c_void_p()
        _check(lib().og_engine_create(C.byref(self.params.to_struct()), C.byref(h)))
        self._h = h
        self._n_atoms: list[int] = []
        self._temps: list[float] = []
        self._finalized = False

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().og_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_system(self, topo, xyz: np.ndarray, temperature_k: float = 310.0) -> int:
        if isinstance(topo, Chain):
            tp = topo.topology_ptr()
        elif isinstance(topo, Topology):
            tp = C.pointer(topo.to_struct())
        else:
            tp = topo
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        idx = C.c_int32()
        _check(lib().og_engine_add_system(self._h, tp, _dptr(x), float(temperature_k), C.byref(idx)))
        self._n_atoms.append(x.shape[0])
        self._temps.append(float(temperature_k))
        return idx.value

    def finalize(self) -> "Engine":
        _check(lib().og_engine_finalize(self._h))
        self._finalized = True
        return self

    def append_atoms(self, sys: int, grown, xyz_new: np.ndarray, v_new: np.ndarray | None = None) -> None:
        """Grow system `sys` (the last) in place to the topology `grown`
        (a Chain after Chain.append, or a Topology) that extends it; xyz_new
        and v_new (None = zero) hold the new atoms only (og_engine_append_atoms)."""
        tp = grown.topology_ptr() if isinstance(grown, Chain) else C.pointer(grown.to_struct())
        x = np.ascontiguousarray(xyz_new, dtype=np.float64).reshape(-1, 3)
        vp = None
        if v_new is not None:
            v = np.ascontiguousarray(v_new, dtype=np.float64).reshape(-1, 3)
            if v.shape != x.shape:
                raise ValueError("velocity and position arrays differ in shape")
            vp = _dptr(v)
        if self._n_atoms[sys] + x.shape[0] != tp.contents.n_atoms:
            raise ValueError("xyz_new must hold exactly the new atoms")
        _check(lib().og_engine_append_atoms(self._h, sys, tp, _dptr(x), vp))
        self._n_atoms[sys] += x.shape[0]

    @property
    def n_systems(self) -> int:
        return len(self._n_atoms)

    def n_atoms(self, sys: int = 0) -> int:
        return self._n_atoms[sys]

    def temperature(self, sys: int) -> float:
        return self._temps[sys]

    def set_stream(self, cuda_stream_ptr: int | None) -> None:
        _check(lib().og_engine_set_stream(self._h, C.c_void_p(cuda_stream_ptr or 0)))

    def synchronize(self) -> None:
        _check(lib().og_engine_synchronize(self._h))

    def positions(self, sys: int = 0) -> np.ndarray:
        x = np.empty((self._n_atoms[sys], 3))
        _check(lib().og_get_positions(self._h, sys, _dptr(x)))
        return x

    def set_positions(self, sys: int, xyz: np.ndarray) -> None:
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        _check(lib().og_set_positions(self._h, sys, _dptr(x)))

    def velocities(self, sys: int = 0) -> np.ndarray:
        v = np.empty((self._n_atoms[sys], 3))
        _check(lib().og_get_velocities(self._h, sys, _dptr(v)))
        return v

    def set_velocities(self, sys: int, v: np.ndarray) -> None:
        a = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        _check(lib().og_set_velocities(self._h, sys, _dptr(a)))

    def init_velocities(self, sys: int, seed: int, remove_com: bool = True) -> None:
        _check(lib().og_init_velocities(self._h, sys, seed & 0xFFFFFFFFFFFFFFFF, int(remove_com)))

    def set_temperature(self, sys: int, t: float) -> None:
        _check(lib().og_set_temperature(self._h, sys, float(t)))
        self._temps[sys] = float(t)

    def total_force(self, sys: int = 0) -> np.ndarray:
        """Forces of every system at the current positions; returns system `sys` (kJ/mol/A)."""
        f = np.empty((self._n_atoms[sys], 3))
        _check(lib().og_compute_forces(self._h, sys, _dptr(f)))
        return f

    def born_radii(self, sys: int = 0) -> np.ndarray:
        r = np.empty(self._n_atoms[sys])
        _check(lib().og_get_born_radii(self._h, sys, _dptr(r)))
        return r

    def born_integrals(self, sys: int = 0) -> np.ndarray:
        """Descreening integrals of the last force evaluation (1/A)."""
        r = np.empty(self._n_atoms[sys])
        _check(lib().og_get_born_integrals(self._h, sys, _dptr(r)))
        return r

    def sasa_areas(self, sys: int = 0, method: str = "powersasa", n_dots: int = 960) -> np.ndarray:
        """Per-atom accessible area (A^2): "powersasa" (analytical, as
        powersasa_energy) or "shrake_rupley" with n_dots test points (as
        sasa_per_atom_with_dots)."""
        codes = {"powersasa": 0, "shrake_rupley": 1}
        if method not in codes:
            raise ValueError(f"unknown SASA method {method!r}")
        r = np.empty(self._n_atoms[sys])
        _check(lib().og_compute_sasa(self._h, sys, codes[method], n_dots, _dptr(r)))
        return r

    # ---- whole-engine state and checkpoints
    STATE_PARTS = ("positions", "velocities", "forces_fixed", "steps", "shake_failures", "status", "temperature")

    def counts(self) -> tuple[int, int]:
        """(real atoms over all systems, systems)."""
        n, s = C.c_int64(), C.c_int32()
        _check(lib().og_engine_counts(self._h, C.byref(n), C.byref(s)))
        return n.value, s.value

    def state_buffers(self, alloc=np.empty) -> dict:
        """Arrays shaped for og_state (alloc(shape, dtype) makes each one, e.g.
        page-locked memory)."""
        n, s = self.counts()
        return {"positions": alloc((n, 3), np.float64), "velocities": alloc((n, 3), np.float64),
                "forces_fixed": alloc((n, 3), np.int64), "steps": alloc((s,), np.int64),
                "shake_failures": alloc((s,), np.int64), "status": alloc((s,), np.int32),
                "temperature": alloc((s,), np.float64)}

    @staticmethod
    def _state_struct(d: dict) -> F.og_state:
        st = F.og_state()
        types = {"positions": (np.float64, F.c_double_p), "velocities": (np.float64, F.c_double_p),
                 "forces_fixed": (np.int64, C.POINTER(C.c_int64)), "steps": (np.int64, C.POINTER(C.c_int64)),
                 "shake_failures": (np.int64, C.POINTER(C.c_int64)), "status": (np.int32, F.c_int32_p),
                 "temperature": (np.float64, F.c_double_p)}
        for k, (dt, pt) in types.items():
            a = d.get(k)
            if a is None:
                continue
            if a.dtype != dt or not a.flags["C_CONTIGUOUS"]:
                raise ValueError(f"state part {k!r} must be a C-contiguous {np.dtype(dt).name} array")
            setattr(st, k, a.ctypes.data_as(pt))
        return st

    def get_state(self, out: dict | None = None, parts=STATE_PARTS) -> dict:
        """The dynamic state of every system (og_get_state): filled into `out`
        (e.g. page-locked arrays from state_buffers) or new arrays."""
        d = out if out is not None else {k: v for k, v in self.state_buffers().items() if k in parts}
        st = self._state_struct({k: d[k] for k in parts if k in d})
        _check(lib().og_get_state(self._h, C.byref(st)))
        return d

    def set_state(self, state: dict) -> None:
        """Restores any subset of a state taken with get_state (og_set_state)."""
        st = self._state_struct(state)
        _check(lib().og_set_state(self._h, C.byref(st)))
        if state.get("temperature") is not None:
            self._temps = [float(t) for t in state["temperature"]]

    def save_checkpoint(self, path: str) -> None:
        _check(lib().og_save_checkpoint(self._h, os.fsencode(path)))

    def load_checkpoint(self, path: str) -> None:
        _check(lib().og_load_checkpoint(self._h, os.fsencode(path)))
        self._temps = [float(t) for t in self.get_state(parts=("temperature",))["temperature"]]

    def energies(self, sys: int = 0) -> dict:
        e = F.og_energies()
        _check(lib().og_compute_energies(self._h, sys, C.byref(e)))
        d = {k: getattr(e, k) for k in ENERGY_TERMS}
        d["born_clamped"] = e.born_clamped
        d["nb_pairs"] = e.nb_pairs
        return d

    def all_energies(self) -> list[dict]:
        arr = (F.og_energies * self.n_systems)()
        _check(lib().og_compute_energies(self._h, -1, arr))
        return [{k: getattr(e, k) for k in ENERGY_TERMS} for e in arr]

    def step(self, n_steps: int = 1, check: bool = True) -> int:
        st = lib().og_step(self._h, int(n_steps))
        if check:
            _check(st)
        return st

    def stats(self, sys: int = 0) -> dict:
        steps, fails, div = C.c_int64(), C.c_int64(), C.c_int32()
        _check(lib().og_system_stats(self._h, sys, C.byref(steps), C.byref(fails), C.byref(div)))
        return {"steps": steps.value, "shake_failures": fails.value, "diverged": bool(div.value)}

    def kinetic(self, sys: int = 0) -> tuple[float, float]:
        ke, t = C.c_double(), C.c_double()
        _check(lib().og_kinetic(self._h, sys, C.byref(ke), C.byref(t)))
        return ke.value, t.value

    def remd_swap(self, parity: int, uniforms: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        acc = np.zeros(max(self.n_systems - 1, 1), dtype=np.int32)
        _check(lib().og_remd_swap(self._h, parity, _dptr(u), acc.ctypes.data_as(F.c_int32_p)))
        return acc[: self.n_systems - 1]

    def remd_run(self, n_rounds: int, steps_per_swap: int, seed: int) -> dict:
        """Device-side parallel tempering rounds (og_remd_run): cumulative
        attempts / accepts per temperature pair and the system at each
        temperature slot."""
        n = self.n_systems
        att = np.zeros(max(n - 1, 1), dtype=np.int64)
        acc = np.zeros(max(n - 1, 1), dtype=np.int64)
        slots = np.zeros(n, dtype=np.int32)
        _check(lib().og_remd_run(self._h, n_rounds, steps_per_swap, seed & 0xFFFFFFFFFFFFFFFF,
                                 att.ctypes.data_as(C.POINTER(C.c_int64)), acc.ctypes.data_as(C.POINTER(C.c_int64)),
                                 slots.ctypes.data_as(F.c_int32_p)))
        return {"attempts": att[: n - 1], "accepts": acc[: n - 1], "sys_of_slot": slots}

    def profile(self, on: bool = True) -> None:
        _check(lib().og_profile_enable(self._h, int(on)))

    def autotune(self, cache_path: str | None = None) -> dict:
        """Times the pair passes' launch variants on this engine's systems and
        keeps the fastest (og_engine_autotune); the choice is cached in the
        JSON file cache_path when given."""
        r = F.og_autotune_result()
        _check(lib().og_engine_autotune(self._h, None if cache_path is None else os.fsencode(cache_path),
                                        C.byref(r)))
        return {k: getattr(r, k) for k, _ in F.og_autotune_result._fields_}

    def set_pair_launch(self, pass_: str, shape: int, persistent: bool, chunk: int = 16) -> None:
        """Sets one pair pass's launch variant ("born" or "force") by hand."""
        _check(lib().og_engine_set_pair_launch(self._h, {"born": 0, "force": 1}[pass_], shape, int(persistent),
                                               chunk))

    def profile_read(self) -> dict:
        buf = (F.og_kernel_time * 64)()
        n = C.c_int32()
        _check(lib().og_profile_read(self._h, buf, 64, C.byref(n)))
        return {buf[k].name.decode(): (buf[k].ms, buf[k].launches) for k in range(n.value)}


# ------------------------------------------------------------------ drivers

class Trajectory:
    """Multi-MODEL PDB trajectory (io/src/pdb.rs write_pdb_trajectory): one
    MODEL block per frame, from host coordinates (write) or from an engine
    system's device positions (capture: queued on the engine's stream into
    page-locked memory; written after the next capture or at close)."""

    def __init__(self, chain: Chain, path: str, title: str = ""):
        h = C.c_void_p()
        _check(lib().og_trajectory_open(chain._h, title.encode(), os.fsencode(path), C.byref(h)))
        self._h = h
        self.n_atoms = chain.n_atoms

    def write(self, xyz: np.ndarray) -> None:
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        if x.shape[0] != self.n_atoms:
            raise ValueError("position array has the wrong number of atoms")
        _check(lib().og_trajectory_write(self._h, _dptr(x)))

    def capture(self, engine: "Engine", sys: int = 0) -> None:
        _check(lib().og_trajectory_capture(self._h, engine._h, sys))

    def close(self) -> None:
        if getattr(self, "_h", None):
            h, self._h = self._h, None
            _check(lib().og_trajectory_close(h))

    def __enter__(self) -> "Trajectory":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Xoshiro256pp:
    """xoshiro256++ with SplitMix64 seeding and cached Box-Muller (dynamics/src/rng.rs)."""

    M = 0xFFFFFFFFFFFFFFFF

    def __init__(self, seed: int):
        sm = seed & self.M
        self.s = []
        for _ in range(4):
            sm = (sm + 0x9E3779B97F4A7C15) & self.M
            z = sm
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.M
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.M
            self.s.append(z ^ (z >> 31))
        self.spare = None

    @staticmethod
    def _rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & Xoshiro256pp.M

    def next_u64(self) -> int:
        s = self.s
        result = (self._rotl((s[0] + s[3]) & self.M, 23) + s[0]) & self.M
        t = (s[1] << 17) & self.M
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t
        s[3] = self._rotl(s[3], 45)
        return result

    def next_f64(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / (1 << 53))

    def gaussian(self) -> float:
        if self.spare is not None:
            g, self.spare = self.spare, None
            return g
        u1 = self.next_f64()
        while u1 <= 0.0:
            u1 = self.next_f64()
        u2 = self.next_f64()
        r = math.sqrt(-2.0 * math.log(u1))
        th = 2.0 * math.pi * u2
        self.spare = r * math.sin(th)
        return r * math.cos(th)


@dataclass
class LangevinOptions:
    """dynamics/src/langevin.rs:52-95."""
    dt_fs: float = 1.0
    temperature_k: float = 310.0
    friction_ps_inv: float = 1.0
    steps: int = 1000
    save_every: int = 10
    seed: int = 0
    randomise_initial_velocities: bool = True
    include_sasa: bool = False
    constrain_h_bonds: bool = False


def run_langevin(chain: Chain, opts: LangevinOptions, callback=None, params: Params | None = None) -> dict:
    """BAOAB Langevin trajectory of one chain on the GPU (dynamics/src/langevin.rs:128).

    The chain's positions are updated in place.  `callback(step, time_fs, T_inst, positions)`
    receives every save_every-th frame including step 0.  O-step noise comes
    from the engine's counter-based generator (not origami's sequential
    xoshiro stream); initial velocities use origami's xoshiro stream exactly.
    """
    p = params or Params()
    p.dt_fs, p.friction_ps_inv = opts.dt_fs, opts.friction_ps_inv
    p.constrain_h_bonds, p.include_sasa, p.seed = opts.constrain_h_bonds, opts.include_sasa, opts.seed
    eng = Engine(p)
    eng.add_system(chain, chain.positions, opts.temperature_k)
    eng.finalize()
    if opts.randomise_initial_velocities:
        eng.init_velocities(0, opts.seed, remove_com=True)
    n = chain.n_atoms
    dof = 3.0 * n
    temps = []
    if callback and opts.save_every > 0:
        _, t0 = eng.kinetic(0)
        callback(0, 0.0, t0, eng.positions(0))
    done, diverged = 0, False
    chunk = opts.save_every if opts.save_every > 0 else opts.steps
    while done < opts.steps:
        k = min(chunk, opts.steps - done)
        st = eng.step(k, check=False)
        done += k
        if st != F.OG_OK:
            diverged = True
            break
        _, t_inst = eng.kinetic(0)
        temps.append(t_inst)
        if callback and opts.save_every > 0 and done % opts.save_every == 0:
            callback(done, done * opts.dt_fs, t_inst, eng.positions(0))
    chain.positions = eng.positions(0)
    ke, _ = eng.kinetic(0)
    stats = eng.stats(0)
    t = np.array(temps) if temps else np.zeros(1)
    return {
        "steps_run": stats["steps"],
        "temperature_mean_k": float(t.mean()),
        "temperature_stddev_k": float(t.std()),
        "equipartition_ratio": ke / (0.5 * dof * BOLTZMANN_KJ_PER_MOL_K * opts.temperature_k),
        "final_kinetic_energy_kj_mol": ke,
        "atoms_count": n,
        "diverged": diverged or stats["diverged"],
        "shake_failures": stats["shake_failures"],
    }


@dataclass
class RemdOptions:
    """dynamics/src/remd.rs:50-89."""
    temperatures_k: list = field(default_factory=lambda: [300.0, 350.0, 400.0, 450.0])
    dt_fs: float = 1.0
    friction_ps_inv: float = 2.0
    total_time_fs: float = 2000.0
    swap_interval_fs: float = 200.0
    save_every: int = 100
    seed: int = 0
    include_sasa: bool = False
    constrain_h_bonds: bool = False
    # swap decisions on the device (og_remd_run: temperature labels exchanged,
    # counter-based uniforms) instead of host Metropolis with origami's swap
    # RNG stream; not with include_sasa
    device_swaps: bool = False


def run_remd(chain: Chain, opts: RemdOptions, callback=None, params: Params | None = None) -> dict:
    """Parallel tempering on one GPU (dynamics/src/remd.rs:136): every replica
    is a system of one engine; swaps follow origami's odd/even schedule,
    Metropolis rule and swap-RNG seed (seed + 0xDEADBEEF), or with
    opts.device_swaps run as device rounds (og_remd_run)."""
    temps = sorted(opts.temperatures_k)
    p = params or Params()
    p.dt_fs, p.friction_ps_inv = opts.dt_fs, opts.friction_ps_inv
    p.constrain_h_bonds, p.include_sasa, p.seed = opts.constrain_h_bonds, opts.include_sasa, opts.seed
    eng = Engine(p)
    x0 = chain.positions
    for t in temps:
        eng.add_system(chain, x0, t)
    eng.finalize()
    for i in range(len(temps)):
        eng.init_velocities(i, (opts.seed + i * 0xC0FFEE) & Xoshiro256pp.M, remove_com=False)
    steps_per_swap = max(1, round(opts.swap_interval_fs / opts.dt_fs))
    total_steps = round(opts.total_time_fs / opts.dt_fs)
    n_rounds = -(-total_steps // steps_per_swap)
    if opts.device_swaps:
        if callback is not None or total_steps % steps_per_swap:
            raise ValueError("device swaps run whole rounds without a frame callback")
        r = eng.remd_run(n_rounds, steps_per_swap, (opts.seed + 0xDEADBEEF) & Xoshiro256pp.M)
        energies = eng.all_energies()
        slot_of = {int(sy): k for k, sy in enumerate(r["sys_of_slot"])}
        order = [int(sy) for sy in r["sys_of_slot"]]
        att, acc = r["attempts"], r["accepts"]
        return {
            "n_replicas": len(temps), "atoms_count": chain.n_atoms,
            "swap_attempts": att.tolist(), "swap_accepts": acc.tolist(),
            "acceptance_ratios": [a / t if t else 0.0 for a, t in zip(acc, att)],
            "sys_of_slot": order,
            "per_replica": [
                {"temperature_k": temps[k], "system": order[k],
                 "final_kinetic_energy_kj_mol": eng.kinetic(order[k])[0],
                 "final_potential_energy_kj_mol": energies[order[k]]["total"], **eng.stats(order[k])}
                for k in range(len(temps))],
            "slot_of_system": slot_of,
        }
    swap_rng = Xoshiro256pp((opts.seed + 0xDEADBEEF) & Xoshiro256pp.M)
    n_pairs = max(len(temps) - 1, 0)
    attempts = np.zeros(n_pairs, dtype=np.int64)
    accepts = np.zeros(n_pairs, dtype=np.int64)
    done = 0
    for rnd in range(n_rounds):
        k = min(steps_per_swap, total_steps - done)
        if k <= 0:
            break
        eng.step(k, check=False)
        done += k
        parity = rnd % 2
        u = np.zeros(max(n_pairs, 1))
        div = [eng.stats(i)["diverged"] for i in range(len(temps))]
        for pi in range(parity, n_pairs, 2):
            if div[pi] or div[pi + 1]:
                continue
            attempts[pi] += 1
            u[pi] = swap_rng.next_f64()
        if n_pairs:
            acc = eng.remd_swap(parity, u)
            accepts += acc
        if callback:
            for i in range(len(temps)):
                callback(i, temps[i], done, eng.positions(i))
    energies = eng.all_energies()
    return {
        "n_replicas": len(temps),
        "atoms_count": chain.n_atoms,
        "swap_attempts": attempts.tolist(),
        "swap_accepts": accepts.tolist(),
        "acceptance_ratios": [a / t if t else 0.0 for a, t in zip(accepts, attempts)],
        "per_replica": [
            {"temperature_k": temps[i], "final_kinetic_energy_kj_mol": eng.kinetic(i)[0],
             "final_potential_energy_kj_mol": energies[i]["total"], **eng.stats(i)}
            for i in range(len(temps))
        ],
    }
