"""ctypes declarations of the C ABI in include/origami_gpu.h.

Only declarations live here; origami_b200/__init__.py loads the library and
builds the Python interface on top.
"""
from __future__ import annotations

import ctypes as C

c_double_p = C.POINTER(C.c_double)
c_int32_p = C.POINTER(C.c_int32)
c_int8_p = C.POINTER(C.c_int8)
c_float_p = C.POINTER(C.c_float)

OG_OK = 0
LGB_N_PARAMS = 43537  # OG_LGB_N_PARAMS
LGB_N_INPUT = 80      # OG_LGB_N_INPUT
STATUS_NAMES = {
    0: "OG_OK", 1: "OG_E_BADARG", 2: "OG_E_NONFINITE", 3: "OG_E_SHAKE", 4: "OG_E_TIMEOUT",
    5: "OG_E_CUDA", 6: "OG_E_NOMEM", 7: "OG_E_STATE", 8: "OG_E_DATA", 9: "OG_E_UNSUPPORTED", 10: "OG_E_IO",
}


class og_topology(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32),
        ("charge", c_double_p), ("rmin_half", c_double_p), ("epsilon", c_double_p),
        ("rmin_half_14", c_double_p), ("epsilon_14", c_double_p),
        ("gb_rho", c_double_p), ("gb_scale", c_double_p), ("mass", c_double_p),
        ("element", c_int32_p),
        ("n_bonds", C.c_int32), ("bond_atoms", c_int32_p), ("bond_k", c_double_p), ("bond_r0", c_double_p),
        ("n_angles", C.c_int32), ("angle_atoms", c_int32_p), ("angle_k", c_double_p), ("angle_theta0", c_double_p),
        ("n_dihedrals", C.c_int32), ("dihedral_atoms", c_int32_p), ("dihedral_term_start", c_int32_p),
        ("n_dihedral_terms", C.c_int32), ("term_k", c_double_p), ("term_n", c_int32_p), ("term_delta", c_double_p),
        ("n_impropers", C.c_int32), ("improper_atoms", c_int32_p), ("improper_k", c_double_p),
        ("improper_psi0", c_double_p),
        ("n_exclusions", C.c_int32), ("exclusion_atoms", c_int32_p), ("exclusion_kind", c_int8_p),
        ("n_constraints", C.c_int32), ("constraint_atoms", c_int32_p), ("constraint_length", c_double_p),
    ]


class og_params(C.Structure):
    _fields_ = [
        ("nb_cutoff", C.c_double), ("born_cutoff", C.c_double), ("gb_force_cutoff", C.c_double),
        ("dt_fs", C.c_double), ("friction_ps_inv", C.c_double),
        ("constrain_h_bonds", C.c_int32), ("shake_max_iters", C.c_int32), ("shake_tol_sq", C.c_double),
        ("include_sasa", C.c_int32), ("sasa_gamma_scale", C.c_double),
        ("born_mode", C.c_int32), ("seed", C.c_uint64),
    ]


class og_energies(C.Structure):
    _fields_ = [
        ("bond", C.c_double), ("angle", C.c_double), ("dihedral", C.c_double), ("improper", C.c_double),
        ("lj", C.c_double), ("coulomb", C.c_double),
        ("gb", C.c_double), ("gb_self", C.c_double), ("gb_pair", C.c_double),
        ("sasa", C.c_double), ("total", C.c_double),
        ("born_clamped", C.c_int32), ("nb_pairs", C.c_int32),
    ]


class og_autotune_result(C.Structure):
    _fields_ = [
        ("born_shape", C.c_int32), ("born_persistent", C.c_int32), ("born_chunk", C.c_int32),
        ("force_shape", C.c_int32), ("force_persistent", C.c_int32), ("force_chunk", C.c_int32),
        ("born_ms", C.c_double), ("force_ms", C.c_double),
        ("born_ms_default", C.c_double), ("force_ms_default", C.c_double),
        ("from_cache", C.c_int32),
    ]


class og_kernel_time(C.Structure):
    _fields_ = [("name", C.c_char_p), ("ms", C.c_double), ("launches", C.c_int64)]


class og_state(C.Structure):
    _fields_ = [
        ("positions", c_double_p), ("velocities", c_double_p), ("forces_fixed", C.POINTER(C.c_int64)),
        ("steps", C.POINTER(C.c_int64)), ("shake_failures", C.POINTER(C.c_int64)), ("status", c_int32_p),
        ("temperature", c_double_p),
    ]


# (name, restype, argtypes) of every exported symbol.
SIGNATURES = [
    ("og_engine_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_int64), c_int32_p]),
    ("og_set_tunnel", C.c_int, [C.c_void_p, c_double_p, c_double_p, C.c_double, C.c_double, C.c_double]),
    ("og_get_state", C.c_int, [C.c_void_p, C.POINTER(og_state)]),
    ("og_set_state", C.c_int, [C.c_void_p, C.POINTER(og_state)]),
    ("og_save_checkpoint", C.c_int, [C.c_void_p, C.c_char_p]),
    ("og_load_checkpoint", C.c_int, [C.c_void_p, C.c_char_p]),
    ("og_pdb_write", C.c_int, [C.c_void_p, c_double_p, C.c_char_p, C.c_char_p]),
    ("og_trajectory_open", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    ("og_trajectory_write", C.c_int, [C.c_void_p, c_double_p]),
    ("og_trajectory_capture", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    ("og_trajectory_close", C.c_int, [C.c_void_p]),
    ("og_last_error", C.c_char_p, []),
    ("og_status_string", C.c_char_p, [C.c_int]),
    ("og_version", C.c_char_p, []),
    ("og_set_data_dir", C.c_int, [C.c_char_p]),
    ("og_chain_build", C.c_int, [C.c_char_p, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_void_p)]),
    ("og_chain_append", C.c_int, [C.c_void_p, C.c_char, C.c_double, C.c_double, C.c_double]),
    ("og_chain_from_structure", C.c_int, [C.c_int32, C.c_char_p, C.c_char_p, c_int32_p, C.c_char_p, c_int32_p,
                                          c_double_p, C.POINTER(C.c_void_p)]),
    ("og_chain_n_atoms", C.c_int, [C.c_void_p, c_int32_p]),
    ("og_chain_n_residues", C.c_int, [C.c_void_p, c_int32_p]),
    ("og_chain_topology", C.c_int, [C.c_void_p, C.POINTER(C.POINTER(og_topology))]),
    ("og_chain_get_positions", C.c_int, [C.c_void_p, c_double_p]),
    ("og_chain_set_positions", C.c_int, [C.c_void_p, c_double_p]),
    ("og_chain_atom_info", C.c_int, [C.c_void_p, C.c_int32, c_int32_p, c_int32_p, C.c_char_p]),
    ("og_chain_missing_params", C.c_int, [C.c_void_p, c_int32_p]),
    ("og_chain_free", None, [C.c_void_p]),
    ("og_params_default", None, [C.POINTER(og_params)]),
    ("og_engine_create", C.c_int, [C.POINTER(og_params), C.POINTER(C.c_void_p)]),
    ("og_engine_add_system", C.c_int, [C.c_void_p, C.POINTER(og_topology), c_double_p, C.c_double, c_int32_p]),
    ("og_engine_finalize", C.c_int, [C.c_void_p]),
    ("og_engine_append_atoms", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(og_topology), c_double_p, c_double_p]),
    ("og_topology_extends", C.c_int, [C.POINTER(og_topology), C.POINTER(og_topology), c_int32_p]),
    ("og_engine_n_systems", C.c_int, [C.c_void_p, c_int32_p]),
    ("og_engine_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("og_engine_synchronize", C.c_int, [C.c_void_p]),
    ("og_engine_destroy", None, [C.c_void_p]),
    ("og_set_positions", C.c_int, [C.c_void_p, C.c_int32, c_double_p]),
    ("og_get_positions", C.c_int, [C.c_void_p, C.c_int32, c_double_p]),
    ("og_set_velocities", C.c_int, [C.c_void_p, C.c_int32, c_double_p]),
    ("og_get_velocities", C.c_int, [C.c_void_p, C.c_int32, c_double_p]),
    ("og_init_velocities", C.c_int, [C.c_void_p, C.c_int32, C.c_uint64, C.c_int32]),
    ("og_set_temperature", C.c_int, [C.c_void_p, C.c_int32, C.c_double]),
    ("og_compute_forces", C.c_int, [C.c_void_p, C.c_int32, c_double_p]),
    ("og_compute_energies", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(og_energies)]),
    ("og_get_born_radii", C.c_int, [C.c_void_p, C.c_int32, c_double_p]),
    ("og_get_born_integrals", C.c_int, [C.c_void_p, C.c_int32, c_double_p]),
    ("og_step", C.c_int, [C.c_void_p, C.c_int32]),
    ("og_system_stats", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64), c_int32_p]),
    ("og_kinetic", C.c_int, [C.c_void_p, C.c_int32, c_double_p, c_double_p]),
    ("og_remd_swap", C.c_int, [C.c_void_p, C.c_int32, c_double_p, c_int32_p]),
    ("og_compute_sasa", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, c_double_p]),
    ("og_profile_enable", C.c_int, [C.c_void_p, C.c_int32]),
    ("og_remd_run", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(C.c_int64),
                              C.POINTER(C.c_int64), c_int32_p]),
    ("og_engine_autotune", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(og_autotune_result)]),
    ("og_engine_set_pair_launch", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    ("og_profile_read", C.c_int, [C.c_void_p, C.POINTER(og_kernel_time), C.c_int32, c_int32_p]),
    ("og_measure_fp32_peak", C.c_int, [c_double_p]),
    ("og_gb_energy_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_double,
                                       C.c_void_p, C.c_void_p]),
    ("og_tc_gemm", C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                             C.c_int64, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                             C.c_int32, C.c_void_p]),
    ("og_lgb_init_params", C.c_int, [C.c_uint64, c_float_p]),
    ("og_lgb_train", C.c_int, [c_float_p, c_float_p, C.c_int64, C.c_int32, C.c_int32, C.c_double, C.c_uint64,
                               c_float_p, c_float_p]),
    ("og_lgb_loss_and_gradient", C.c_int, [c_float_p, c_float_p, C.c_int64, c_float_p, c_double_p, c_float_p]),
    ("og_lgb_samples", C.c_int, [C.c_void_p, C.c_int32, c_float_p, c_float_p]),
    ("og_lgb_set_params", C.c_int, [C.c_void_p, c_float_p]),
    ("og_lgb_set_judge", C.c_int, [C.c_void_p, C.c_int32, C.c_double]),
    ("og_lgb_status", C.c_int, [C.c_void_p, c_int32_p, c_int32_p, c_double_p]),
    ("og_lgb_judge", C.c_int, [C.c_void_p, c_double_p]),
]


def declare(lib: C.CDLL, names: set[str] | None = None) -> C.CDLL:
    """Attach restype/argtypes for every symbol in SIGNATURES present in lib."""
    for name, res, args in SIGNATURES:
        if names is not None and name not in names:
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
