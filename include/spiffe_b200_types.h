/* spiffe_b200_types.h
 *
 * Plain-C descriptions of the state of one spiffe problem, shared by every
 * entry point of libspiffe_b200 (no C++ or torch types).  They mirror the
 * reference data model (spiffe.h:28-131 FIELDS, :201-221 BEAM, :341-352
 * SCREEN) with one change of representation: every mesh array is a single
 * contiguous (nz+1) x (nr+1) block indexed [iz*(nr+1) + ir] (ir fastest, the
 * order of the reference's zarray_2d rows) instead of a row-pointer array.
 * Array stagger, units and flag bits are the reference's (spiffe.h:50-100).
 */
#ifndef SPIFFE_B200_TYPES_H
#define SPIFFE_B200_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* mode bits, spiffe.h:50-56 */
#define SPIFFE_FL_TM_FIELDS 1u
#define SPIFFE_FL_TE_FIELDS 2u
#define SPIFFE_FL_SPACE_CHARGE 4u
#define SPIFFE_FL_RADIAL_INTERP 8u
#define SPIFFE_FL_LONGIT_INTERP 16u
#define SPIFFE_FL_RADIAL_SMEAR 32u
#define SPIFFE_FL_LONGIT_SMEAR 64u

/* metal-flag bits, spiffe.h:90-100 */
#define SPIFFE_FL_IS_SURFACE 1
#define SPIFFE_FL_IS_INSIDE 2
#define SPIFFE_FL_EZ_ZERO 4
#define SPIFFE_FL_ER_ZERO 8
#define SPIFFE_FL_IS_VACUUM 16
#define SPIFFE_FL_BPHI_ZERO 32
#define SPIFFE_FL_EPHI_ZERO 64
#define SPIFFE_FL_BZ_ZERO 128
#define SPIFFE_FL_BR_ZERO 256
#define SPIFFE_FL_IS_METAL (SPIFFE_FL_IS_SURFACE | SPIFFE_FL_IS_INSIDE)
#define SPIFFE_FL_LAST_ACTIVE_PT 512

/* boundary conditions, spiffe.h:38-39 */
#define SPIFFE_DIRICHLET 0
#define SPIFFE_NEUMANN 1

/* particle status bits, spiffe.h:219-220 */
#define SPIFFE_PART_ACTIVE 0x0001ull
#define SPIFFE_PART_LOST 0x0002ull

/* Mesh, time and uniform-field description (FIELDS scalars, spiffe.h:30-75,
 * :117-120).  dz=(zmax-zmin)/(nz-1), dr=rmax/(nr-1) as geometry.c:75-76. */
typedef struct spiffe_mesh {
  int32_t nz, nr;
  double zmin, zmax, rmax, dz, dr;
  int32_t lower_bc, upper_bc, right_bc, left_bc;
  uint32_t modes;
  double dt, start_time, time;
  int64_t time_step;
  double constant_E[3]; /* Ez, Er, Ephi */
  double constant_B[3]; /* Bz, Br, Bphi */
  int16_t turn_off[6];  /* Ez, Er, Ephi, Bz, Br, Bphi */
  int32_t has_solenoid; /* BzImposed/BrImposed take part in the gather */
  double imposed_ramp_time, imposed_flat_top_time;
} spiffe_mesh;

/* Mesh arrays, each (nz+1)*(nr+1) doubles or NULL when absent. */
typedef struct spiffe_field_set {
  int16_t *flags;
  double *Ez, *Er, *Bphi, *Bphi2, *Jz, *Jr;
  double *Ephi, *Jphi, *Br, *Br2, *Bz, *Bz2;
  double *EzImposed, *ErImposed, *PsiImposed;
  double *BzImposed, *BrImposed;
  double *Psi, *Q;
} spiffe_field_set;

/* Structure-of-arrays beam (BEAM, spiffe.h:201-221); arrays hold `capacity`
 * slots of which the first np are live. */
typedef struct spiffe_beam_set {
  int64_t np, npActive, capacity;
  int32_t nextParticleID;
  double QoMC, stiffness;
  double *z, *r, *pz, *pr, *r_pphi, *vz, *vr, *vphi, *Q;
  double *r0, *z0, *t0, *rmin, *rmax, *zmin, *zmax;
  int32_t *particleID;
  int16_t *generation;
  uint64_t *status;
} spiffe_beam_set;

/* Screen crossing records (SCREEN, spiffe.h:341-352; columns of screens.c:18). */
#define SPIFFE_MAX_SCREENS 8 /* screens one instance records */
#define SPIFFE_SCREEN_QUANS 8 /* r, pz, pr, pphi, t, q, r0, t0 */
typedef struct spiffe_screen_set {
  double z_position;
  int32_t direction; /* +1 forward, -1 backward */
  int64_t nb, capacity;
  double *col[SPIFFE_SCREEN_QUANS];
  double *rmin, *rmax, *zmin, *zmax;
  int16_t *generation;
  int32_t *particleID;
} spiffe_screen_set;

/* Rows of the lost-particle file (integrate's lost_particles;
 * setUpLostParticleFile, advance_particles.c:577-603, and the rows of the
 * loss epilogue, :437-487): the time, where the path left the open region
 * (findLossCoordinates, secondaryEmission.c:239), the momenta, birth
 * position, charge, generation and id, and the step of each row. */
typedef struct spiffe_lost_set {
  int64_t nb, capacity;
  double *t, *rLost, *zLost, *pz, *pr, *z0, *r0, *q;
  int16_t *generation;
  int32_t *particleID;
  int64_t *step; /* may be NULL */
  /* may be NULL: the impact momentum |p| (beta*gamma) and the side of the
   * surface the particle crossed (findLossCoordinates' directionCode,
   * secondaryEmission.c:239-352: 1 left, 2 right, 3 up, 4 down, 0 none), the
   * arguments the reference passes to queueSecondaryEmission
   * (advance_particles.c:443-451) */
  double *p;
  int16_t *direction;
} spiffe_lost_set;

/* define_secondary_emission (secondaryEmission.nl; processSecondaryEmission-
 * Definition, secondaryEmission.c:21-118): particles lost on a surface of
 * material `material_id` (the &po material_id of define_geometry) release a
 * Poisson-distributed number of secondaries with mean yield(K) (linear in the
 * table, K the impact kinetic energy in eV), each of momentum
 * emitted_momentum (beta*gamma) in a random direction away from the surface;
 * at most yield_limit each (0: no limit). */
typedef struct spiffe_secondary_options {
  int32_t material_id, verbosity;
  double emitted_momentum;
  int64_t yield_limit;
  int64_t n_data;
  const double *energy, *yield; /* energy in eV, increasing */
  int32_t log;                  /* keep the emission log (log_file) */
} spiffe_secondary_options;
#define SPIFFE_SECONDARY_LOG_COLS 10

/* TM field update of the split-precision form (spiffe_gpu_set_fdtd_kernel) */
#define SPIFFE_FDTD_AUTO 0        /* the fused kernel on meshes of 2^18 nodes and more, else two kernels */
#define SPIFFE_FDTD_TWO_KERNELS 1 /* an E and a B kernel over 2-D tiles */
#define SPIFFE_FDTD_FUSED 2       /* one persistent kernel sweeping bands of rows staged by bulk copies */

/* Poisson solver of the split-precision form (spiffe_gpu_set_poisson_solver) */
#define SPIFFE_POISSON_SOR 0       /* the reference's red-black SOR and stop rule (poisson.c:17-130) */
#define SPIFFE_POISSON_MULTIGRID 1 /* FP32 multigrid V-cycles in FP64 refinement, the same stop rule */

/* Lost-particle removal.  SPIFFE_COMPACT_REFERENCE reproduces
 * advance_particles.c:491-518 as it behaves: the loop tests is_lost[ip] but
 * never moves is_lost with the particle it copies down, so the first lost
 * index ends the beam (np becomes that index).  SPIFFE_COMPACT_SWAP removes
 * exactly the lost particles, each slot refilled from the end of the array.
 * SPIFFE_COMPACT_ANY removes exactly the lost particles in any order (the
 * cell-sorted single-precision form). */
#define SPIFFE_COMPACT_REFERENCE 0
#define SPIFFE_COMPACT_SWAP 1
#define SPIFFE_COMPACT_ANY 2

/* Screen momentum interpolation.  SPIFFE_SCREEN_REFERENCE reproduces
 * advance_particles.c:383-385 as it behaves: pz0/pr0/r_pphi0 are function
 * scope (:79) and hold the pre-kick values of the last particle of the push
 * loop.  SPIFFE_SCREEN_PARTICLE uses each particle's own pre-kick values. */
#define SPIFFE_SCREEN_REFERENCE 0
#define SPIFFE_SCREEN_PARTICLE 1

/* Options of advance_particles (advance_particles.c:67-76 arguments and the
 * test-beam forced-acceleration mode, :289-311). */
typedef struct spiffe_push_options {
  double z_forces_start; /* integrate.nl:18, -1 = off */
  double tb_electrons_per_macroparticle;
  double tb_z_force, tb_r_force;
  double tb_z_start_deceleration, tb_r_start_deceleration;
  int32_t compaction;      /* SPIFFE_COMPACT_* */
  int32_t screen_momentum; /* SPIFFE_SCREEN_* */
} spiffe_push_options;

/* Poisson correction command (poisson_correction.nl; defaults from
 * setup_poisson_correction, poisson_correction.c:38-46). */
typedef struct spiffe_poisson_options {
  double start_time;
  int64_t step_interval;
  double accuracy;
  double error_charge_threshold;
  int64_t maximum_iterations;
  int32_t verbosity;
  int32_t guess_code; /* 0 none, 1 line-charge, 2 point-charge, 3 zero */
} spiffe_poisson_options;

/* define_test_beam command (test_beam.nl, defaults test_beam.c:24-27): one
 * macroparticle of electrons_per_macroparticle electrons is added every step
 * from int((start_time-t0)/dt) to int((stop_time-t0)/dt) at (initial_z,
 * initial_r) with the given momenta (emit_test_particles, test_beam.c:57-104).
 * The forced acceleration (z_force, r_force and the deceleration starts) is
 * part of spiffe_push_options. */
typedef struct spiffe_test_beam_options {
  double start_time, stop_time;
  double initial_z, initial_r;
  double initial_pz, initial_pr, initial_rpphi;
  double electrons_per_macroparticle;
} spiffe_test_beam_options;

/* define_cathode command (cathode.nl:8-40, defaults cathode.c:32-40).  A
 * time profile, when given, is n_profile (t, factor) pairs in increasing t. */
typedef struct spiffe_cathode_options {
  double z_position, inner_radius, outer_radius;
  double current_density, temperature, work_function;
  int32_t field_emission;
  double field_emission_beta;
  double electrons_per_macroparticle;
  double start_time, stop_time, time_offset;
  int32_t autophase;
  double number_per_step, initial_pz, initial_omega, stiffness;
  int32_t discretize_radii, random_number_seed;
  int32_t distribution_correction_interval, spread_over_dt, zoned_emission;
  int32_t n_profile;
  const double *profile_t, *profile_A;
} spiffe_cathode_options;

/* define_emitter (emitter.nl; process_emitter_definition, emitter.c:19-167):
 * emission from the boundary segments of one material (the points and
 * directions of spiffe_geometry_boundary_points), at a current density given,
 * from the Richardson-Schottky law (temperature and work_function) or from
 * field emission, scaled by an optional time profile. */
#define SPIFFE_EMITS_RIGHT 1 /* the side a boundary segment emits to (spiffe.h:270-273) */
#define SPIFFE_EMITS_UP 2
#define SPIFFE_EMITS_LEFT 3
#define SPIFFE_EMITS_DOWN 4
typedef struct spiffe_emitter_options {
  int32_t material_id;
  double current_density, temperature, work_function; /* temperature already determined */
  int32_t field_emission;
  double field_emission_beta;
  double electrons_per_macroparticle;
  double start_time, stop_time;
  double initial_p, offset_factor;
  int32_t random_number_seed; /* random_2(-|seed|) */
  int32_t n_profile;
  const double *profile_t, *profile_A;
  int64_t n_points;           /* boundary nodes, direction per segment */
  const int32_t *iz, *ir;
  const int16_t *direction;
} spiffe_emitter_options;

/* define_field_sampling (field_sampling.nl; process_sampling_definition,
 * field_sampling.c:53-101): the component codes, in the order of the
 * component names of field_sampling.c:28-29.  (The reference's own macros
 * call 4 SAMPLE_BPHI and 5 SAMPLE_BR, so its TE check, :80-85, applies to
 * "Bphi" and not to "Br"; the values are those the names say.) */
#define SPIFFE_SAMPLE_EZ 0
#define SPIFFE_SAMPLE_ER 1
#define SPIFFE_SAMPLE_EPHI 2
#define SPIFFE_SAMPLE_BZ 3
#define SPIFFE_SAMPLE_BR 4
#define SPIFFE_SAMPLE_BPHI 5
#define SPIFFE_SAMPLE_JZ 6
#define SPIFFE_SAMPLE_JR 7
#define SPIFFE_SAMPLE_PHI 8
#define SPIFFE_SAMPLE_Q 9
#define SPIFFE_SAMPLE_E 10 /* Ez, Er, Ephi */
#define SPIFFE_SAMPLE_B 11 /* Bz, Br, Bphi */
typedef struct spiffe_sample_options {
  int32_t component; /* SPIFFE_SAMPLE_* */
  int32_t direction; /* 0: along z at r = position; 1: along r at z = position */
  double min_coord, max_coord, position, time_interval, start_time;
  int32_t time_sequence; /* one row per sample (the average over the range) instead of one page */
} spiffe_sample_options;

/* Samples taken since the last download, one entry per sample: its time,
 * its parameters (param[3k]: the rSample/zSample value, then for a time
 * sequence the start and stop of the range) and its rows (rows[k]), whose
 * coordinate (z or r; for a time sequence the row's time) goes to x and
 * whose values go to v[0..2] (one column, or three for SPIFFE_SAMPLE_E/B). */
typedef struct spiffe_sample_set {
  int64_t n_samples, n_rows;        /* filled in */
  int64_t max_samples, max_rows;    /* capacity of the arrays below */
  double *t, *param;                /* max_samples, 3*max_samples */
  int64_t *rows;                    /* max_samples */
  double *x, *v[3];                 /* max_rows */
} spiffe_sample_set;

/* Result of one Poisson correction (the quantities the reference prints,
 * poisson_correction.c:254-256, :284). */
typedef struct spiffe_poisson_report {
  int32_t ran;        /* 0 when skipped by interval or threshold */
  int64_t iterations; /* solve_poisson_cyl return value */
  double Qreal, Qerror, Qsurface;
  double residual, driving; /* final sum|residual|, sum|rhs| of the solve */
} spiffe_poisson_report;

/* One status report (do_status_printouts, status_pr.c:18-356): the values of
 * one row of the status file (setUpStatusOutputFile, status_pr.c:454-499)
 * except NewParticles, which is the caller's (Particles minus the previous
 * row's).  The beam moments cover all np particles, active or not, as the
 * reference's do; Charge sums the active ones. */
typedef struct spiffe_status_row {
  double t, JCathode, KineticEnergy, FieldEnergy, TotalEnergy, Charge, EzAbsMax, ErAbsMax;
  int64_t Particles, ActiveParticles, SecondaryParticles;
  double zMax, zMin, zAve, zRMS, zStDev;
  double rMax, rMin, rAve, rRMS, rStDev;
  double pzMax, pzMin, pzAve, pzRMS, pzStDev;
  double prMax, prMin, prAve, prRMS, prStDev;
  double EzOOEMin, EzOOEMax;
  double ElectricEnergy, MagneticEnergy; /* FieldEnergy's two parts */
} spiffe_status_row;

#ifdef __cplusplus
}
#endif

#endif
