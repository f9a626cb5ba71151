/*
 * origami_gpu.h -- C ABI of the B200 force-and-integrate engine for origami's
 * implicit-solvent MD hot path.
 *
 * origami (Rust) evaluates forces through
 *   energy::total_force_with_scratch(&Structure, &TopologyGraph, &ForceField,
 *        cutoff_a, include_sasa, &mut ForceScratch, &mut Vec<Vec3>)
 *        -- crates/energy/src/forces.rs:78-128
 * with per-atom caches built by ForceScratch::new (crates/energy/src/scratch.rs:143),
 * energies through bonded_energy / nonbonded_energy / gb_energy
 * (crates/energy/src/bonded.rs:34, nonbonded.rs:97, gb.rs:146), and steps with
 * BAOAB + SHAKE inside run_langevin / run_remd / run_cotranslate
 * (crates/dynamics/src/langevin.rs:128, remd.rs:136, cotranslate.rs:174).
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions (all entry points):
 *   - plain C types only; every pointer is borrowed for the duration of the
 *     call; the engine owns its device memory.
 *   - positions in Angstrom, velocities in Angstrom/fs, forces in kJ/mol/A,
 *     energies in kJ/mol, masses in Da, temperatures in K, times in fs --
 *     origami's unit system (crates/dynamics/src/langevin.rs:19-34).
 *   - coordinate arrays are interleaved xyz, 3*n_atoms doubles, in origami's
 *     atom order (residue order, then template order inside a residue).
 *   - every function returns an og_status; nothing aborts the process.
 *   - an engine is not thread safe; calls on one engine are stream ordered.
 */
#ifndef ORIGAMI_GPU_H
#define ORIGAMI_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum og_status {
  OG_OK = 0,
  OG_E_BADARG = 1,     /* invalid argument (null pointer, size, index) */
  OG_E_NONFINITE = 2,  /* a velocity or force became NaN/Inf (langevin.rs:316-319 "diverged") */
  OG_E_SHAKE = 3,      /* SHAKE did not converge within max iterations (shake.rs:86-125) */
  OG_E_TIMEOUT = 4,    /* a bounded device wait gave up */
  OG_E_CUDA = 5,       /* CUDA runtime error (see og_last_error) */
  OG_E_NOMEM = 6,      /* device or host allocation failed */
  OG_E_STATE = 7,      /* call not valid in the engine's current state */
  OG_E_DATA = 8,       /* force-field / template table missing or malformed */
  OG_E_UNSUPPORTED = 9, /* feature not built into this library */
  OG_E_IO = 10          /* a file could not be opened, read or written */
} og_status;

/* Human-readable text of the most recent error on this thread. */
const char* og_last_error(void);
const char* og_status_string(int status);
/* Library version string, e.g. "origami-b200 0.1 (sm_100a)". */
const char* og_version(void);

/* -------------------------------------------------------------- topology
 * Flat description of one molecular system: what origami's ForceScratch
 * caches per atom (scratch.rs:35-133 -- charges, CHARMM LJ params incl. 1-4,
 * GB rho / HCT scale) plus the TopologyGraph term lists with their force-field
 * parameters already resolved (forcefield.rs:84-158 lookups) and the 1-2/1-3
 * exclusion and 1-4 pair list (scratch.rs:233-251 rebuild_exclusions; graph
 * predicates geom/src/topology_graph.rs:81-112).  Terms whose parameters are
 * missing from the force field are simply absent, which is what the
 * reference's `let Some(p) = ... else { continue }` skips do.
 * Parameter units are CHARMM's (kcal/mol, Angstrom, degrees); the engine
 * converts at the leaves exactly where origami does (units.rs).
 */
typedef struct og_topology {
  int32_t n_atoms;
  const double* charge;        /* e */
  const double* rmin_half;     /* LJ Rmin/2, A */
  const double* epsilon;       /* LJ epsilon, kcal/mol (positive) */
  const double* rmin_half_14;  /* 1-4 Rmin/2 (equals rmin_half when the FF has none) */
  const double* epsilon_14;    /* 1-4 epsilon */
  const double* gb_rho;        /* intrinsic Born radius rho, A (gb.rs:58-68) */
  const double* gb_scale;      /* HCT descreening scale (gb.rs:73-83) */
  const double* mass;          /* Da (element.rs:27-37) */
  const int32_t* element;      /* 0 H, 1 C, 2 N, 3 O, 4 P, 5 S */

  int32_t n_bonds;
  const int32_t* bond_atoms;   /* 2 per bond, a < b, sorted (topology_graph.rs:252) */
  const double* bond_k;        /* kcal/mol/A^2, V = K (r - r0)^2 */
  const double* bond_r0;       /* A */

  int32_t n_angles;
  const int32_t* angle_atoms;  /* 3 per angle, central atom in the middle */
  const double* angle_k;       /* kcal/mol/rad^2 */
  const double* angle_theta0;  /* degrees */

  int32_t n_dihedrals;
  const int32_t* dihedral_atoms;      /* 4 per dihedral, canonical (b < c) */
  const int32_t* dihedral_term_start; /* n_dihedrals + 1 offsets into the term arrays */
  int32_t n_dihedral_terms;
  const double* term_k;               /* kcal/mol */
  const int32_t* term_n;              /* multiplicity */
  const double* term_delta;           /* degrees */

  int32_t n_impropers;
  const int32_t* improper_atoms; /* 4 per improper, central atom first */
  const double* improper_k;      /* kcal/mol/rad^2 */
  const double* improper_psi0;   /* degrees */

  int32_t n_exclusions;
  const int32_t* exclusion_atoms; /* 2 per pair, i < j, sorted */
  const int8_t* exclusion_kind;   /* 1 = excluded (1-2 or 1-3), 2 = 1-4 pair */

  int32_t n_constraints;            /* X-H bonds (shake.rs:47-76), bond order */
  const int32_t* constraint_atoms;  /* 2 per constraint */
  const double* constraint_length;  /* A (force-field r0) */
} og_topology;

/* ------------------------------------------------- host model (sequence ->
 * system).  Restates origami's chain builder and topology graph so callers
 * without a structure of their own can build one:
 *   build_extended_chain / build_chain / append_residue  geom/src/builder.rs:50-90
 *   build_topology_graph                                  geom/src/topology_graph.rs:134
 *   ForceScratch::rebuild_params (per-atom params)        energy/src/scratch.rs:196
 *   build_h_bond_constraints                              dynamics/src/shake.rs:47
 * The force-field and template tables are read from the data directory next
 * to the shared library (override with og_set_data_dir).
 */
typedef struct og_chain og_chain;

og_status og_set_data_dir(const char* path);
/* One-letter sequence; phi/psi/omega in radians (NAN = origami's defaults
 * phi -120 deg, psi 140 deg, omega 180 deg). */
og_status og_chain_build(const char* sequence, double phi, double psi, double omega, og_chain** out);
/* Appends one residue at the C terminus (cotranslate.rs:204 append_residue). */
og_status og_chain_append(og_chain* chain, char residue, double phi, double psi, double omega);
/* A chain from a structure the caller already holds: origami's
 * geom::Structure (geom/src/structure.rs), residues in order, each with its
 * chain id and its atoms' names, elements and positions -- what read_pdb
 * (io/src/pdb_read.rs:167) returns and what the CLI's energy / minimize /
 * dynamics commands score.  residues: n_residues one-letter codes; chains:
 * one chain id per residue (NULL = all 'A'; the peptide bond C(i-1)-N(i) is
 * made only inside a chain, topology_graph.rs:199-209); atoms_per_residue:
 * n_residues counts; names: 8 bytes per atom, NUL-padded wwPDB v3.3 names
 * as the residue templates use them; elements: 0 H, 1 C, 2 N, 3 O, 4 P, 5 S
 * per atom (NULL = from the name's first letter, pdb_read.rs:452-462); xyz:
 * 3 doubles per atom.  Atom order is kept as given.  An atom the force field
 * cannot type is OG_E_DATA (ForceScratch::rebuild_params panics there,
 * scratch.rs:202-205). */
og_status og_chain_from_structure(int32_t n_residues, const char* residues, const char* chains,
                                  const int32_t* atoms_per_residue, const char* names, const int32_t* elements,
                                  const double* xyz, og_chain** out);
og_status og_chain_n_atoms(const og_chain* chain, int32_t* n_atoms);
og_status og_chain_n_residues(const og_chain* chain, int32_t* n_residues);
/* Topology arrays stay valid until the chain is modified or freed. */
og_status og_chain_topology(og_chain* chain, const og_topology** topo);
og_status og_chain_get_positions(const og_chain* chain, double* xyz);
og_status og_chain_set_positions(og_chain* chain, const double* xyz);
/* Per-atom metadata: residue index, CHARMM atom-type index (chem atom_type.rs
 * declaration order), and the atom name into a caller buffer (<= 8 chars + NUL). */
og_status og_chain_atom_info(const og_chain* chain, int32_t atom, int32_t* residue,
                             int32_t* atom_type, char name[8]);
/* Counts of bonded tuples the force field could not parameterise
 * (bonded.rs:21-23 missing_count; nonbonded.rs:92). */
og_status og_chain_missing_params(const og_chain* chain, int32_t* missing);
void og_chain_free(og_chain* chain);

/* ------------------------------------------------------------------ engine */
typedef struct og_params {
  /* Cutoffs in A.  origami's integrator path uses 10 (LJ + reaction-field
   * Coulomb, forces_nonbonded.rs:125), 20 (Born descreening, gb.rs:40) and 10
   * (GB pair force, forces_gb.rs:33).  A value <= 0 or >= 1e30 means "no
   * cutoff": all pairs, bare Coulomb (the reaction field's Rc -> infinity limit). */
  double nb_cutoff;
  double born_cutoff;
  double gb_force_cutoff;
  /* Integrator (LangevinOptions, langevin.rs:52-95). */
  double dt_fs;
  double friction_ps_inv;
  int32_t constrain_h_bonds;  /* SHAKE X-H bonds, tol 1e-6 A^2, 64 iterations */
  int32_t shake_max_iters;    /* 0 -> 64 */
  double shake_tol_sq;        /* 0 -> 1e-6 */
  /* Analytical PowerSasa hydrophobic term: forces as
   * add_sasa_forces_analytical_with_scratch (powersasa/analytical.rs:451),
   * energy sum gamma_i A_i as powersasa_energy (powersasa/mod.rs:55).  gamma =
   * 0.005 kcal/mol/A^2 on C and S times sasa_gamma_scale (the reference's
   * ORIGAMI_SASA_GAMMA_SCALE, analytical.rs:607), applied to the energy as
   * well as the force so the two stay consistent (the reference scales the
   * force only).  An atom's arrangement may hold up to 254 cutting spheres,
   * 254 circle transitions per batch and 128 exposed arcs; beyond that the
   * step returns OG_E_UNSUPPORTED (the reference has no limit). */
  int32_t include_sasa;
  double sasa_gamma_scale;
  /* Born radii: 0 = plain OBC-II descreening pass, 1 = learned radii. */
  int32_t born_mode;
  uint64_t seed;
} og_params;

/* Fills origami's defaults (10/20/10 A cutoffs, dt 1 fs, gamma 1 ps^-1, no
 * SHAKE, no SASA, plain Born radii, seed 0). */
void og_params_default(og_params* p);

typedef struct og_energies {
  double bond, angle, dihedral, improper;  /* bonded.rs BondedBreakdown */
  double lj, coulomb;                      /* nonbonded.rs NonbondedBreakdown */
  double gb, gb_self, gb_pair;             /* gb.rs GbBreakdown */
  double sasa;                             /* sum gamma_i A_i (include_sasa) */
  double total;
  int32_t born_clamped;                    /* gb.rs GbBreakdown::clamped_count */
  int32_t nb_pairs;                        /* pairs inside the LJ/Coulomb cutoff */
} og_energies;

typedef struct og_engine og_engine;

/* Creates an engine on the current CUDA device.  Systems are added, then the
 * engine is finalised (device upload, tile lists), then stepped. */
og_status og_engine_create(const og_params* params, og_engine** out);
/* Adds one system (a replica or an independent chain).  xyz = initial
 * positions; temperature for its heat bath.  The topology is copied. */
og_status og_engine_add_system(og_engine* e, const og_topology* topo, const double* xyz,
                               double temperature_k, int32_t* system_index);
og_status og_engine_finalize(og_engine* e);
/* Co-translational growth in place: replaces the per-slice rebuild of
 * run_slice (cotranslate.rs:318-319, ForceScratch::new, scratch.rs:196-251).
 * System `sys` -- the engine's last -- takes the atoms and terms that
 * `grown` adds to its topology (the topology of the same chain after
 * og_chain_append; og_topology_extends states the rule).  xyz_new holds
 * the new atoms' positions, v_new their velocities (NULL = zero), 3 doubles
 * per new atom.  Only the new atoms' data crosses to the device: their
 * parameters, the exclusion-mask blocks and rows their exclusions reach,
 * their bonded terms and SHAKE clusters (appended), the system's atom count
 * and degrees of freedom; the existing atoms' positions, velocities and the
 * step count stay on the device.  Device arrays grow by half again when
 * full; the step graph is re-captured at the next og_step.  The force and
 * energy results equal those of an engine built from `grown` (forces bit
 * for bit).  OG_E_BADARG when `grown` does not extend the system or `sys`
 * is not the last system; the engine is then unchanged.  After any other
 * error (a failed device allocation or copy) the engine is to be destroyed. */
og_status og_engine_append_atoms(og_engine* e, int32_t sys, const og_topology* grown, const double* xyz_new,
                                 const double* v_new);
/* Host-only check (no GPU): *extends = 1 when `grown` extends `base` --
 * more atoms; the first base->n_atoms with bit-identical parameters; in
 * each term list (bonds, angles, dihedrals with their terms, impropers,
 * exclusions, constraints) the records among those atoms equal to base's
 * records, in base's order -- else 0, with the reason in og_last_error. */
og_status og_topology_extends(const og_topology* base, const og_topology* grown, int32_t* extends);
og_status og_engine_n_systems(const og_engine* e, int32_t* n);
/* Runs kernels on this CUDA stream (cudaStream_t as void*; NULL = the
 * engine's own stream). */
og_status og_engine_set_stream(og_engine* e, void* cuda_stream);
og_status og_engine_synchronize(og_engine* e);
void og_engine_destroy(og_engine* e);

/* Positions / velocities of one system, host arrays of 3*n_atoms doubles. */
og_status og_set_positions(og_engine* e, int32_t sys, const double* xyz);
og_status og_get_positions(og_engine* e, int32_t sys, double* xyz);
og_status og_set_velocities(og_engine* e, int32_t sys, const double* v);
og_status og_get_velocities(og_engine* e, int32_t sys, double* v);
/* Draw Maxwell-Boltzmann velocities at the system's temperature with
 * origami's own generator: xoshiro256++ seeded by SplitMix64 from `seed`,
 * Box-Muller gaussians drawn x, y, z per atom in atom order (rng.rs:18-98,
 * langevin.rs:487-513).  remove_com = 1 subtracts the centre-of-mass velocity
 * as run_langevin does; 0 leaves it, as run_remd does with seed
 * base + i * 0xC0FFEE for replica i (remd.rs:209-212). */
og_status og_init_velocities(og_engine* e, int32_t sys, uint64_t seed, int32_t remove_com);
og_status og_set_temperature(og_engine* e, int32_t sys, double temperature_k);

/* External potential of co-translational folding (cotranslate.rs:119-154
 * CylindricalTunnel): every real atom of every system whose projection on
 * the axis origin + t * direction lies within [0, length_a] and whose
 * distance d from the axis exceeds radius_a feels k_confine (d - radius_a)
 * toward the axis (kJ/mol/A; direction used as given, a unit vector).  Added
 * to og_compute_forces and every og_step force evaluation; not an energy
 * term (the reference's ExternalPotential has none).  origin or direction
 * NULL removes it. */
og_status og_set_tunnel(og_engine* e, const double* origin, const double* direction, double radius_a,
                        double length_a, double k_confine);

/* Forces at the current positions of every system: replaces
 * total_force_with_scratch (forces.rs:78).  f_out (optional) receives
 * 3*n_atoms doubles for system `sys` (or nothing when NULL).  The same
 * evaluation also leaves the forces on the device for the next og_step. */
og_status og_compute_forces(og_engine* e, int32_t sys, double* f_out);
/* Potential energy of system `sys` at its current positions, the sum that
 * origami's REMD swap and L-BFGS line search use (remd.rs:529
 * potential_energy, energy_eval.rs:20 total_energy_with_options): bonded +
 * LJ/RF-Coulomb within nb_cutoff + GB (Born radii within born_cutoff, pair
 * sum over ALL pairs, gb.rs:146-182) [+ SASA].  FP64 on the device.
 * sys = -1 evaluates every system at once; out then holds n_systems entries. */
og_status og_compute_energies(og_engine* e, int32_t sys, og_energies* out);
/* Effective Born radii of system `sys` (gb.rs:203 compute_born_radii_into_scratch);
 * out receives n_atoms doubles. */
og_status og_get_born_radii(og_engine* e, int32_t sys, double* radii);
/* The descreening integrals behind those radii (ForceScratch::gb_integral,
 * scratch.rs:95), n_atoms doubles in 1/A, from the last force evaluation. */
og_status og_get_born_integrals(og_engine* e, int32_t sys, double* integrals);

/* Advance every system by n_steps BAOAB(+SHAKE) steps (the loop body of
 * run_langevin, langevin.rs:223-342).  Per-system status words record
 * divergence and SHAKE failures; the call returns OG_E_NONFINITE if any
 * system diverged (it is then frozen, like REMD skips diverged replicas). */
og_status og_step(og_engine* e, int32_t n_steps);
/* Per-system counters: steps run, SHAKE failures, diverged flag. */
og_status og_system_stats(og_engine* e, int32_t sys, int64_t* steps, int64_t* shake_failures,
                          int32_t* diverged);
/* Instantaneous kinetic energy (langevin.rs:469) and temperature with
 * 3N degrees of freedom. */
og_status og_kinetic(og_engine* e, int32_t sys, double* ke_kj_mol, double* temperature_k);

/* ---- Whole-engine state, checkpoints and trajectory output.
 * The reference writes trajectories as multi-MODEL PDB (io/src/pdb.rs:31
 * write_pdb_trajectory) and has no binary checkpoint; both are here.
 *
 * og_state: the dynamic state of every system, systems in order, real atoms
 * only (n_atoms = the sum of the systems' atom counts, og_engine_counts):
 * positions and velocities (n_atoms x 3 doubles, A and A/fs), the forces of
 * the last evaluation in the engine's fixed point (n_atoms x 3 int64, 2^32
 * units per kJ/mol/A), and per system the step counter (which keys the
 * O-step noise), SHAKE failure count, status word and temperature.  Restoring
 * a state taken with og_get_state continues the run bit for bit.  Every
 * pointer may be NULL: og_get_state skips that part; og_set_state keeps the
 * engine's value, except that NULL forces (or new positions without forces)
 * make the next step evaluate the forces first.  Host buffers may be
 * pageable; page-locked buffers are copied by DMA without staging. */
typedef struct og_state {
  double* positions;
  double* velocities;
  int64_t* forces_fixed;
  int64_t* steps;
  int64_t* shake_failures;
  int32_t* status;
  double* temperature;
} og_state;
og_status og_engine_counts(const og_engine* e, int64_t* n_atoms, int32_t* n_systems);
og_status og_get_state(og_engine* e, const og_state* out);
og_status og_set_state(og_engine* e, const og_state* in);
/* The state above (plus the learned-radius switch and judge phase) in a
 * binary file: "OGCKPT01", u32 version 1, i32 systems, i64 atoms, i32 atoms
 * per system, then the arrays in og_state order, little endian.  Loading
 * requires an engine with the same systems' atom counts. */
og_status og_save_checkpoint(og_engine* e, const char* path);
og_status og_load_checkpoint(og_engine* e, const char* path);

/* PDB output, record for record as io/src/pdb.rs: one model of a chain
 * (write_pdb; xyz NULL = the chain's own positions), or a trajectory with
 * one MODEL block per frame (write_pdb_trajectory).  A frame comes from host
 * coordinates (og_trajectory_write) or from an engine system's device
 * positions (og_trajectory_capture: the copy is queued on the engine's
 * stream into page-locked memory and the call returns at once; the frame is
 * formatted and written at a later capture, write or close, so writing
 * overlaps the steps that follow).  The chain supplies names and residues;
 * the system must have the chain's atom count. */
typedef struct og_trajectory og_trajectory;
og_status og_pdb_write(const og_chain* chain, const double* xyz, const char* title, const char* path);
og_status og_trajectory_open(const og_chain* chain, const char* title, const char* path, og_trajectory** out);
og_status og_trajectory_write(og_trajectory* t, const double* xyz);
og_status og_trajectory_capture(og_trajectory* t, og_engine* e, int32_t sys);
og_status og_trajectory_close(og_trajectory* t);

/* Replica exchange (remd.rs:425-474): for each adjacent pair (a, a+1) with
 * a = parity, parity+2, ... of the temperature-sorted systems, Metropolis on
 * delta = (beta_a - beta_b)(E_a - E_b) with uniforms u[pair]; on acceptance
 * positions, velocities and forces are exchanged and velocities rescaled by
 * sqrt(T_a/T_b).  accepted[pair] (optional) receives 0/1.  With include_sasa
 * the surface term of E is the 960-point Shrake-Rupley energy with the
 * unscaled tension, as remd.rs:529-537 potential_energy uses. */
og_status og_remd_swap(og_engine* e, int32_t parity, const double* uniforms, int32_t* accepted);

/* Parallel tempering run on the device (remd.rs:136 run_remd's loop,
 * :425-474 attempt_swaps): n_rounds rounds of steps_per_swap og_step steps,
 * each followed by one swap round between neighbouring temperatures (pairs
 * (0,1), (2,3), ... on even rounds, (1,2), ... on odd ones, counting rounds
 * across calls).  The potential energies (bonded + LJ/RF + GB, FP64, as
 * og_compute_energies) stay on the device; the Metropolis decision uses
 * delta = (beta_i - beta_j)(E_i - E_j) with a uniform from a counter-based
 * generator keyed by (seed, round, pair); an accepted exchange swaps the two
 * systems' temperatures and rescales each one's velocities by
 * sqrt(T_new / T_old) -- the reference's exchange of coordinates between
 * temperatures, without moving coordinates.  The ladder is the systems'
 * temperatures at the first call, sorted.  attempts / accepts (optional,
 * n_systems - 1 entries) receive the cumulative counts per temperature pair,
 * sys_of_slot (optional, n_systems) the system now at each temperature,
 * ascending.  Systems must have equal atom counts; with include_sasa the
 * swap energy is the Shrake-Rupley one of og_remd_swap (OG_E_UNSUPPORTED
 * here).  A diverged system is skipped, as run_remd does. */
og_status og_remd_run(og_engine* e, int32_t n_rounds, int32_t steps_per_swap, uint64_t seed, int64_t* attempts,
                      int64_t* accepts, int32_t* sys_of_slot);

/* Per-atom solvent-accessible area (A^2, radius vdW + 1.4 A) of system `sys`
 * at its current positions; area_out receives n_atoms doubles.
 * method 0: analytical PowerSasa (powersasa/mod.rs:55 powersasa_energy's
 * per_atom_area); method 1: Shrake-Rupley with n_dots Fibonacci points
 * (sasa.rs:65 sasa_per_atom_with_dots; n_dots <= 0 means the reference's
 * 960).  FP64 on the device; works whether or not include_sasa is set. */
og_status og_compute_sasa(og_engine* e, int32_t sys, int32_t method, int32_t n_dots, double* area_out);

/* Launch configuration of the two O(N^2) pair passes (Born descreening,
 * far-field force) for this engine's systems.  No counterpart in the
 * reference: origami's replica loop (dynamics/src/remd.rs:286,
 * replicas.par_iter_mut()) and its per-call rayon pool take this role on
 * the CPU.  Every variant computes the same sums; shapes differ in the
 * fixed-point rounding of partial sums only (well inside the force
 * tolerance), and for a fixed configuration runs are bit-reproducible.
 *   shape       0: 8 i-tiles (256 atoms) per CTA at the default occupancy
 *               target (Born 4 CTAs/SM, force 2); 1: 4 i-tiles (128 atoms)
 *               per CTA at twice the CTAs per SM; 2: 8 i-tiles at 3 CTAs/SM;
 *               force pass only: 3: two i-tiles per warp, 16 per CTA at 2
 *               CTAs/SM; 4: two i-tiles per warp, 8 per CTA at 4 CTAs/SM;
 *               5, 6: as 4 at 5 or 6 CTAs/SM
 *   persistent  0: one CTA per work item; 1: resident CTAs taking items from
 *               an atomic work queue
 *   chunk       j-tiles per work item (default 16)
 * og_engine_autotune times every combination (3 Born / 7 force shapes x 2 x
 * chunks 8, 16, 32) of each pass on the engine's systems at their current positions and
 * keeps the fastest; the choice is cached in the JSON file cache_path (NULL
 * = no cache) under the workload's bucket (mode, total 32-atom tiles and
 * the largest system's tiles rounded up to powers of two), so a later
 * engine in the same bucket is configured without timing.  The next step
 * re-evaluates the forces. */
typedef struct og_autotune_result {
  int32_t born_shape, born_persistent, born_chunk;
  int32_t force_shape, force_persistent, force_chunk;
  double born_ms, force_ms;                 /* the chosen variants' times (ms per launch) */
  double born_ms_default, force_ms_default; /* shape 0, one CTA per item, chunk 16; -1 from cache */
  int32_t from_cache;
} og_autotune_result;
og_status og_engine_autotune(og_engine* e, const char* cache_path, og_autotune_result* out);
/* Sets one pass's launch by hand: pass 0 = Born, 1 = force. */
og_status og_engine_set_pair_launch(og_engine* e, int32_t pass, int32_t shape, int32_t persistent, int32_t chunk);

/* CUDA-event timing of the kernels the last og_step launched: fills up to
 * `cap` entries of (kernel id, milliseconds) summed over the call. */
typedef struct og_kernel_time { const char* name; double ms; int64_t launches; } og_kernel_time;
og_status og_profile_enable(og_engine* e, int32_t on);
og_status og_profile_read(og_engine* e, og_kernel_time* out, int32_t cap, int32_t* n_out);

/* GB solvation energy of one system with no device allocation.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * when they need the energy: a host whose GPU memory is reserved up front by
 * another framework's caching allocator, or a latency-critical loop that
 * forbids allocation (and the device synchronisation it implies) after
 * start-up.  Computes, in FP64, OBC-II effective Born radii (HCT
 * descreening over the pairs within born_cutoff, <= 0 or >= 1e30 = all
 * pairs; tanh map; radius floor) and then the generalized-Born energy: the
 * per-atom self terms plus the pair terms over ALL pairs, written as
 * energy_out[0..2] = {total, self, pair} in kJ/mol.  Every pointer is a
 * device pointer the caller owns: xyz (3 * n_atoms, interleaved), charge,
 * gb_rho, gb_scale (n_atoms each), energy_out (3); work is queued on
 * `stream` (cudaStream_t, NULL = legacy default stream) and the call does
 * not wait.  Scratch is a fixed device array inside the library, sized for
 * at most OG_NOALLOC_MAX_ATOMS atoms (~129 KiB held on every GPU that uses
 * it until exit); larger systems are rejected with OG_E_BADARG.
 * Set-up: the driver places that array and the kernels in device memory the
 * first time they are used on a device (CUDA's lazy module loading), which
 * can fail once another allocator holds all the memory.  A call with
 * n_atoms = 0 and every pointer NULL does that set-up for the current device
 * and nothing else; make it (or a first real call) before other frameworks
 * reserve their memory, and before any stream capture.  Each call outside
 * capture looks the array's address up again, so a cudaDeviceReset between
 * calls is harmless; calls made during capture reuse the last address found.
 * All calls share the array, so calls that overlap on the GPU race: order
 * them. */
#define OG_NOALLOC_MAX_ATOMS 16384
og_status og_gb_energy_noalloc(const double* xyz, const double* charge, const double* gb_rho,
                               const double* gb_scale, int32_t n_atoms, double born_cutoff,
                               double* energy_out, void* stream);

/* Measured FP32 FMA throughput of the current device (TFLOP/s, FMA = 2 flops)
 * from a register-resident FMA chain on every SM: the denominator of the
 * pair kernels' FP32-pipe roofline.  No counterpart in the reference. */
og_status og_measure_fp32_peak(double* tflops);

/* BF16 tensor-core GEMM (tcgen05, FP32 accumulate) on DEVICE buffers:
 *   c[m*c_sm + n*c_sn] = sum_k a[m*a_sm + k*a_sk] * b[n*b_sn + k*b_sk]
 * (+ bias[n] when bias is not NULL; c_act, when not NULL, receives SiLU(c)
 * with c's strides).  Operands are FP32 and rounded to BF16 for the MMA.
 * splits > 1 divides K among CTAs (c must then be row-major contiguous).
 * The learned-Born-radius network trains and runs on it.  No counterpart
 * in the reference. */
og_status og_tc_gemm(const float* a, int64_t a_sm, int64_t a_sk, const float* b, int64_t b_sn, int64_t b_sk,
                     float* c, int64_t c_sm, int64_t c_sn, int32_t m, int32_t n, int32_t k, const float* bias,
                     float* c_act, int32_t splits, void* cuda_stream);

/* ---- Learned Born radii (born_mode = 1).  No counterpart in the reference.
 * Per atom: 64 descriptors D (16 Gaussian shells, centres 1.5..12 A, width
 * 0.7 A, x 4 element classes C/S, N/P, O, H; partner-radius weighted, cosine
 * cutoff 12 A), input x = log(1 + D); an 80-128-128-128-1 SiLU network over
 * the inputs below (BF16 tensor-core products, FP32 accumulate) predicts
 * y = log(R / R_cfa), clamped to [-5, 5], R_cfa
 * the Coulomb-field radius in its pairwise (HCT) form over the same 12 A
 * neighbours: 1/R_cfa = max(1/rho~ - sum fc I_HCT(r, rho~_i, s_j rho~_j),
 * 1/30).  The network input is OG_LGB_N_INPUT = 80 wide: the 64
 * descriptors, then the atom's own class one-hot (4), rho~, HCT scale,
 * rho~/R_cfa, log R_cfa, 0, log(rho~/R_cfa) and 6 zeros; the output adds a
 * linear FP32 term v . x[64..80) to the network's.  Parameters:
 * OG_LGB_N_PARAMS floats, W1[128x80] b1[128] W2[128x128]
 * b2[128] W3[128x128] b3[128] w4[128] b4 v[16] (W row-major, out x in).  Forces use
 * the predicted radii frozen, like the plain pass's.  Energies
 * (og_compute_energies) stay plain GB. */
#define OG_LGB_N_PARAMS 43537
#define OG_LGB_N_INPUT 80

/* Uniform(+-1/sqrt(fan_in)) hidden weights, zero biases, zero output
 * weights w4 and v (the untrained network predicts y = 0, i.e. R = R_cfa),
 * from `seed`. */
og_status og_lgb_init_params(uint64_t seed, float* params);
/* Training: the linear path (v, b4) is first set by an FP64 least-squares
 * fit over all samples, then minibatch Adam (beta 0.9 / 0.999, step size lr
 * with cosine decay to 0 over `steps`) trains every parameter on the mean
 * squared error of y over
 * host samples x[n x 80], target[n]; params updated in place;
 * loss_per_step (optional) receives each step's batch loss. */
og_status og_lgb_train(const float* x, const float* target, int64_t n, int32_t steps, int32_t batch, double lr,
                       uint64_t seed, float* params, float* loss_per_step);
/* Mean squared error and its gradient (OG_LGB_N_PARAMS floats) over all n
 * samples in one batch (n <= 2^20), by the same kernels. */
og_status og_lgb_loss_and_gradient(const float* x, const float* target, int64_t n, const float* params,
                                   double* loss, float* grad);
/* Training samples of system `sys` (or of every system, in order, when
 * sys = -1) at the current positions: x_out (n_atoms x 80 network inputs) and
 * target_out (n_atoms) = log(R_plain / R_cfa) with R_plain the FP64
 * plain-GB radii.  Any born_mode. */
og_status og_lgb_samples(og_engine* e, int32_t sys, float* x_out, float* target_out);
/* Loads the network (born_mode = 1 engines); required before stepping. */
og_status og_lgb_set_params(og_engine* e, const float* params);
/* Every `interval_steps` steps (default 500; 0 = never) og_step evaluates
 * the forces with plain GB radii at the current positions; if the largest
 * per-system RMS relative force difference exceeds `tolerance` (default
 * 1e-3) the engine falls back to plain GB for the rest of the run. */
og_status og_lgb_set_judge(og_engine* e, int32_t interval_steps, double tolerance);
/* active = learned radii in use; judged = judge evaluations so far;
 * last_error = the last judge's error (-1 before the first). */
og_status og_lgb_status(og_engine* e, int32_t* active, int32_t* judged, double* last_error);
/* Runs the judge now (and falls back if it fails); rms_rel receives the error. */
og_status og_lgb_judge(og_engine* e, double* rms_rel);

#ifdef __cplusplus
}
#endif

#endif /* ORIGAMI_GPU_H */
