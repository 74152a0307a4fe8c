/* spiffe_b200_session.h -- spiffe's command surface on libspiffe_b200.
 *
 * A session holds what spiffe's main holds (spiffe.c:97-122: the FIELDS
 * problem, cathodes, antennae, screens, the test beam, the Poisson and
 * field-saving definitions) and executes spiffe input text, one namelist
 * command after another as spiffe.c:213-308 does.  Mesh arrays stay on the
 * host until the first &integrate, which creates the device instance; later
 * commands act on that instance.  File names in commands are used as given
 * (relative to the working directory, as in spiffe); "%s" in an output name
 * is replaced by the rootname (compose_filename).
 *
 * Commands executed:
 *   define_geometry (geometry.c:21-369), set_constant_fields / constant_fields
 *   (constant_fields.c:18), define_solenoid (solenoid.c:18), define_cathode
 *   (cathode.c:21), define_antenna (antenna.c:18), define_screen (screens.c:29),
 *   define_test_beam (test_beam.c:17), poisson_correction
 *   (poisson_correction.c:31), load_fields (load_fields.c:20),
 *   define_field_saving (field_saving.c:16; time_interval saving),
 *   define_snapshots (snapshots.c:16), define_field_output (field_output.c:16),
 *   add_on_axis_fields (onAxisFields.c:18, with its fields_used table),
 *   translate (translate.c:21), integrate (integrate.c:24, with status_output,
 *   status_pr.c:454), trace (obsolete, as spiffe), stop.
 * Accepted with a warning and no output (diagnostic files only):
 *   define_field_sampling, and the
 *   output-file variables boundary_output, urmel_boundary_output,
 *   discrete_boundary_output, interior_points, emission_log, field_output,
 *   lost_particles.
 * Rejected with SPIFFE_ERR_UNSUPPORTED: define_resistor, load_particles,
 * define_secondary_emission, define_emitter, translate's reduction of the
 * integration region (z_lower, z_upper), and options whose physics the device
 * loop does not have (current smoothing and filtering, test charges, thermal
 * velocities, Halton sequences, field saving on an Ez trigger).
 *
 * Outputs: screens, field saves, beam snapshots, field output, the status
 * file and the on-axis fields_used table are SDDS1 binary files with the
 * reference's columns and parameters.  A screen page holds the crossings of
 * one run segment (the steps between two host synchronisations, at most
 * the session's flush interval) instead of one time step.
 */
#ifndef SPIFFE_B200_SESSION_H
#define SPIFFE_B200_SESSION_H

#include <stdint.h>

#include "spiffe_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* spiffe_session_execute's return value after a &stop command */
#define SPIFFE_SESSION_STOPPED 1

typedef struct spiffe_session spiffe_session;

/* A session computing in `precision` (SPIFFE_PRECISION_*); `rootname`
 * (may be NULL: "spiffe") names outputs as EM_problem->rootname does. */
int spiffe_session_create(int32_t precision, const char *rootname, spiffe_session **out);
int spiffe_session_destroy(spiffe_session *s);

/* Executes every command of `text` in order.  Returns 0, SPIFFE_SESSION_STOPPED
 * at &stop, or a negative code at the first failing command (the reference
 * exits there; the session keeps its state up to that command). */
int spiffe_session_execute(spiffe_session *s, const char *text);
/* Reads `path` and executes it (spiffe <inputfile>). */
int spiffe_session_run_file(spiffe_session *s, const char *path);

/* Session settings (no counterpart in the reference):
 *   "verbose"            0 quiet, 1 command echo and progress (default 1)
 *   "deposit_order"      FP64 form: 1 deposits in particle order (bit-identical
 *                        to the serial reference), 0 uses atomics (default 1)
 *   "particle_capacity"  initial device particle slots (default 65536; grown
 *                        on demand)
 *   "screen_capacity"    device records per screen between flushes (default
 *                        1048576)
 *   "flush_steps"        longest run segment between screen flushes (default 512)
 *   "compaction"         SPIFFE_COMPACT_* (default: REFERENCE for FP64, ANY for
 *                        the split form)
 *   "screen_momentum"    SPIFFE_SCREEN_* (default: REFERENCE for FP64, PARTICLE
 *                        for the split form)
 *   "poisson_solver"     split form: SPIFFE_POISSON_* (default MULTIGRID) */
int spiffe_session_set(spiffe_session *s, const char *name, double value);

/* The mesh after define_geometry (time and step after the last integrate). */
int spiffe_session_mesh(spiffe_session *s, spiffe_mesh *mesh);
/* Copies every array the session holds into the non-NULL pointers of `host`
 * (device arrays after an integrate); flags too when host->flags is set.
 * Arrays the problem does not have are left untouched. */
int spiffe_session_fields(spiffe_session *s, spiffe_field_set *host);
/* The device instance (NULL before the first integrate). */
int spiffe_session_instance(spiffe_session *s, spiffe_gpu_instance **inst);
/* Steps run by all integrate commands so far. */
int64_t spiffe_session_steps(spiffe_session *s);

/* define_solenoid's field (solenoid.c:18-117, Bsolenoid.c): adds current x the
 * field of `turns` 1 A rings of radius `radius` spread evenly from z_start to
 * z_end (mirrored about z=0 when symmetry is +-1) to Bz and Br at the nodes
 * z = zmin + iz*dz, r = ir*dr, ir <= the evaluation radius limit; with
 * bucking, the current cancels Bz on axis at z_buck; with Bz_peak != 0 the
 * whole of Bz/Br (including earlier solenoids) is scaled so that the largest
 * on-axis Bz is Bz_peak.  Bz and Br are (nz+1)*(nr+1), ir fastest.
 * *current_used (may be NULL) receives the current applied. */
typedef struct spiffe_solenoid_options {
  double radius, evaluation_radius_limit, z_start, z_end, current, Bz_peak;
  int64_t turns;
  int32_t symmetry, bucking;
  double z_buck;
} spiffe_solenoid_options;
int spiffe_solenoid_add(const spiffe_mesh *mesh, const spiffe_solenoid_options *opt, double *Bz, double *Br,
                        double *current_used);

#ifdef __cplusplus
}
#endif

#endif
