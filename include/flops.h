/*
 * flops.h -- algorithmic work per unit of origami's hot-path formulas, used
 * for the `roofline.achieved` figures.  Counted once from the reference
 * formulas (crates/energy/src/forces_nonbonded.rs:196-232,
 * forces_gb.rs:82-111, gb.rs:347-369), not from this library's kernels:
 * +, -, * count 1, a fused multiply-add counts 2, and each sqrt, reciprocal,
 * division, exp, log counts 1.  The unit is one UNORDERED atom pair, which is
 * what origami's pair loops visit; a kernel that evaluates both orders of a
 * pair does not get credit for the second evaluation.
 */
#ifndef ORIGAMI_FLOPS_H
#define ORIGAMI_FLOPS_H

/* LJ (1-4 aware) + reaction-field Coulomb + GB frozen-radii pair force:
 * distance 8, sqrt + 1/r^2 2, LJ 13, Coulomb 5, GB 16, coefficient combine,
 * apply to the separation and scatter to i and j 11. */
#define OG_FLOPS_FORCE_PAIR 55

/* Born descreening: distance + sqrt 9, two pairwise_descreening calls of 25
 * each, two accumulations 2 (rounded to 60). */
#define OG_FLOPS_BORN_PAIR 60

/* Bytes one BAOAB step moves per atom in the element-wise kernels: positions,
 * velocities and SHAKE references (FP64 x3 each, read and written), fixed-point
 * forces (3 x 8 read), mass (8) -- about 2 x 72 + 24 + 8. */
#define OG_BYTES_INTEGRATE_ATOM 176

#endif /* ORIGAMI_FLOPS_H */
