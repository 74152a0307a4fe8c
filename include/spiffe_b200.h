/* spiffe_b200.h -- C ABI of libspiffe_b200, the B200 implementation of
 * spiffe's per-timestep particle-in-cell loop.
 *
 * One spiffe problem (FIELDS + BEAM + screens, spiffe.h:28-131, :201-221,
 * :341-352) lives on the GPU as a spiffe_gpu_instance.  The calls below are
 * the reference's hot-path functions, one entry point each, so a host loop
 * shaped like perform_integration (integrate.c:134-194) can drive the GPU
 * step by step; spiffe_gpu_run_steps runs that whole loop on the device.
 * All arrays cross the boundary as contiguous (nz+1)x(nr+1) blocks, ir
 * fastest (spiffe_b200_types.h).
 *
 * Every function returns 0 on success or a negative error code;
 * spiffe_gpu_last_error() then describes the failure (thread-local).
 * Instances are independent; one instance must not be used by two host
 * threads at the same time.
 */
#ifndef SPIFFE_B200_H
#define SPIFFE_B200_H

#include <stdint.h>

#include "spiffe_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SPIFFE_PRECISION_F64 0     /* plain FP64, bit-faithful to the reference */
#define SPIFFE_PRECISION_SPLIT32 1 /* FP32 fields and push, split positions, fixed-point J */

#define SPIFFE_ERR_INVALID -1
#define SPIFFE_ERR_CUDA -2
#define SPIFFE_ERR_CAPACITY -3
#define SPIFFE_ERR_DEVICE -4
#define SPIFFE_ERR_UNSUPPORTED -5
#define SPIFFE_ERR_NOMEM -6

typedef struct spiffe_gpu_instance spiffe_gpu_instance;

/* Description of the last error on this thread. */
const char *spiffe_gpu_last_error(void);

/* Library version string. */
const char *spiffe_gpu_version(void);

/* Creates an instance for `mesh` with metal flags `flags` ((nz+1)*(nr+1)
 * values as geometry.c:319-362 sets them) and room for `particle_capacity`
 * macroparticles (grown on demand, like the reference's trealloc in
 * cathode.c:427-456).  Replaces: the allocations of process_geometry_definition
 * (geometry.c:78-107). */
int spiffe_gpu_create(const spiffe_mesh *mesh, const int16_t *flags, int32_t precision, int64_t particle_capacity,
                      spiffe_gpu_instance **out);
int spiffe_gpu_destroy(spiffe_gpu_instance *inst);

/* Time, dt, uniform fields and switches; the mesh geometry must not change. */
int spiffe_gpu_set_mesh(spiffe_gpu_instance *inst, const spiffe_mesh *mesh);
int spiffe_gpu_get_mesh(spiffe_gpu_instance *inst, spiffe_mesh *mesh);

/* Copies every non-NULL array of `host` to / from the device. */
int spiffe_gpu_upload_fields(spiffe_gpu_instance *inst, const spiffe_field_set *host);
int spiffe_gpu_download_fields(spiffe_gpu_instance *inst, spiffe_field_set *host);
int spiffe_gpu_upload_beam(spiffe_gpu_instance *inst, const spiffe_beam_set *host);
int spiffe_gpu_download_beam(spiffe_gpu_instance *inst, spiffe_beam_set *host);

/* 0: FP64 atomics (default); 1: deposit in particle order, bit-identical to
 * the serial reference (space_charge.c:130-137). */
int spiffe_gpu_set_deposit_order(spiffe_gpu_instance *inst, int32_t ordered);

/* zero_current_arrays, integrate.c:210 */
int spiffe_gpu_zero_current_arrays(spiffe_gpu_instance *inst);
/* advance_field_solutions, integrate.c:277 */
int spiffe_gpu_advance_field_solutions(spiffe_gpu_instance *inst);
/* add_particle_currents, space_charge.c:34 */
int spiffe_gpu_add_particle_currents(spiffe_gpu_instance *inst);
/* advance_particles, advance_particles.c:67 (screens added with
 * spiffe_gpu_add_screen; lost-particle logging is not produced) */
int spiffe_gpu_advance_particles(spiffe_gpu_instance *inst, const spiffe_push_options *opt);
/* solve_poisson_cyl, poisson.c:17: target 0 solves Psi with driving term Q,
 * target 1 solves PsiImposed with no driving term.  *iterations receives the
 * reference's return value (half-sweeps, or -1 at the limit). */
int spiffe_gpu_solve_poisson_cyl(spiffe_gpu_instance *inst, int32_t target, double accuracy, int64_t iteration_limit,
                                 int64_t *iterations);
/* No counterpart in the reference.  The same SOR solve on device arrays the
 * caller owns (Psi updated in place; rhs may be NULL; flags int16; all
 * (nz+1)*(nr+1), ir fastest), allocating nothing: for callers that may not
 * allocate device memory, such as a host application whose device memory
 * belongs to another framework's pool, or a control loop that forbids
 * allocation after start-up.  All scratch lives in one fixed 352 KB array
 * that every GPU loading the library holds until exit; limits: iteration_limit
 * <= 16384, nr <= 4096, ceil((nr-1)/32)*ceil(nz/8) <= 16384.  Larger sizes
 * are rejected with an error.  Each call looks up that array's device address
 * with the caller's device and context current, copies its coefficient tables
 * from host memory on `stream`, and waits on `stream` for the solve to finish
 * before it returns.  Every call shares the one array: calls that overlap on
 * the GPU (other threads, other streams) race and must be serialised by the
 * caller.  `stream` is a cudaStream_t (NULL: the default stream). */
int spiffe_gpu_solve_poisson_cyl_noalloc(const spiffe_mesh *mesh, double *psi, const double *rhs, const int16_t *flags,
                                         double accuracy, int64_t iteration_limit, int64_t *iterations, void *stream);
/* add_poisson_correction, poisson_correction.c:73 (interval and start-step
 * tests included; `report` may be NULL) */
int spiffe_gpu_add_poisson_correction(spiffe_gpu_instance *inst, int32_t space_charge, const spiffe_poisson_options *opt,
                                      spiffe_poisson_report *report);
/* No counterpart in the reference, which prints these values only when
 * verbose.  The instance's log of Poisson corrections that ran (one row each,
 * kept on the device so a run of steps needs no host synchronisation): rows
 * [k*4 + 0..3] = time step, iterations (half-sweeps or V-cycles, -1 at the
 * limit), final sum|residual|, sum|rhs| of the solve.  Copies at most
 * max_rows of the first 65536 rows; *n_total receives how many ran. */
int spiffe_gpu_poisson_log(spiffe_gpu_instance *inst, int64_t max_rows, double *rows, int64_t *n_total);
/* compute_imposed_Efield, poisson_correction.c:456 */
int spiffe_gpu_compute_imposed_efield(spiffe_gpu_instance *inst, const spiffe_poisson_options *opt, int32_t initialize);

/* define_screen (screens.c:29): records accumulate on the device until cleared. */
int spiffe_gpu_add_screen(spiffe_gpu_instance *inst, double z_position, int32_t direction, int64_t capacity);
int spiffe_gpu_screen_count(spiffe_gpu_instance *inst, int32_t screen, int64_t *nb);
int spiffe_gpu_download_screen(spiffe_gpu_instance *inst, int32_t screen, spiffe_screen_set *host);
int spiffe_gpu_clear_screens(spiffe_gpu_instance *inst);
/* The lost-particle file's rows (integrate's lost_particles, the loss
 * epilogue of advance_particles.c:437-487 with findLossCoordinates,
 * secondaryEmission.c:239): capacity > 0 makes every push record up to
 * `capacity` lost particles on the device between downloads; 0 stops it. */
int spiffe_gpu_set_lost_log(spiffe_gpu_instance *inst, int64_t capacity);
/* The rows recorded since the last download, in the reference's order (step,
 * then particle index), and empties the log; an error when more particles
 * were lost than the log or `host` holds. */
int spiffe_gpu_download_lost(spiffe_gpu_instance *inst, spiffe_lost_set *host);
/* The surface material of each node, (nz+1)*(nr+1) ir fastest: the
 * materialID array of FIELDS (spiffe.h:105), from define_geometry's &po
 * material_id (spiffe_geometry_rasterise's material output). */
int spiffe_gpu_set_materials(spiffe_gpu_instance *inst, const int16_t *material);
/* define_secondary_emission (secondaryEmission.c:21-118): each push queues
 * the lost particles that hit this material (queueSecondaryEmission, :120-237)
 * and the next step of spiffe_gpu_run_steps emits their secondaries before
 * the cathodes' births (emitSecondaryElectrons, :374-584; integrate.c:159-163),
 * drawing from the instance's generator in the reference's order.  With
 * opt->log set, each emitting source is logged as the reference's log_file
 * records it (:520-544), taking a particle ID as the reference does. */
int spiffe_gpu_add_secondary_emission(spiffe_gpu_instance *inst, const spiffe_secondary_options *opt);
/* define_field_sampling (field_sampling.c:53-101): adds a sampling
 * definition (checked as the reference checks it against the mesh's field
 * modes); *index receives its number.  spiffe_gpu_run_steps samples at the
 * top of every step (integrate.c:149) on the device, into a buffer the host
 * drains with spiffe_gpu_download_samples; spiffe_gpu_sample_fields samples
 * at the current time (the call after the loop, integrate.c:196). */
int spiffe_gpu_add_field_sampling(spiffe_gpu_instance *inst, const spiffe_sample_options *opt, int32_t *index);
int spiffe_gpu_sample_fields(spiffe_gpu_instance *inst);
/* The samples of definition `index` taken since the last download, and
 * empties them (sample_fields, field_sampling.c:103-1097: the rows and
 * values the reference writes).  With out->max_samples 0 only n_samples and
 * n_rows are set. */
int spiffe_gpu_download_samples(spiffe_gpu_instance *inst, int32_t index, spiffe_sample_set *out);
/* The emission log of secondary-emission definition `index` (the order of
 * spiffe_gpu_add_secondary_emission) since the last call, and empties it:
 * *n_rows rows of SPIFFE_SECONDARY_LOG_COLS doubles, row-major (time step of
 * the emission, z, r, t, K, yield, emitted, directionCode, generation,
 * particleID).  With rows NULL only *n_rows is set; an error when max_rows is
 * too small. */
int spiffe_gpu_secondary_log(spiffe_gpu_instance *inst, int32_t index, int64_t max_rows, double *rows,
                             int64_t *n_rows);
/* No counterpart in the reference, which leaves moments to external SDDS
 * tools.  The exit-plane moments of a screen's records, reduced on the device
 * in FP64 with weights |q|: out[0] records, [1] charge sum q, [2] mean kinetic
 * energy m c^2 <gamma-1> (eV), [3] its rms spread (eV), [4] rms bunch length
 * sigma_t <beta_z> c (m), [5] normalized rms emittance of the x projection,
 * <x^2> = <r^2>/2, <px^2> = (<pr^2> + <pphi^2>)/2, <x px> = <r pr>/2 (m). */
int spiffe_gpu_screen_moments(spiffe_gpu_instance *inst, int32_t screen, double *out);

/* define_cathode (cathode.c:21) and define_antenna (antenna.c:18) for the
 * device integration loop; waveform times must already include time_offset. */
int spiffe_gpu_add_cathode(spiffe_gpu_instance *inst, const spiffe_cathode_options *opt);
/* define_emitter (emitter.c:19-167): each step of spiffe_gpu_run_steps emits
 * from every segment of the surface after the cathodes
 * (emit_electrons_from_emitter, :169-390; integrate.c:164-165) and updates
 * the current density from the fields after the step (setEmitterCurrentDensity,
 * :392-440; integrate.c:132-133, :192-193), drawing positions from the
 * second generator (random_2), reseeded by each definition. */
int spiffe_gpu_add_emitter(spiffe_gpu_instance *inst, const spiffe_emitter_options *opt);
int spiffe_gpu_add_antenna(spiffe_gpu_instance *inst, int32_t direction, int64_t istart, int64_t iend,
                           int64_t iposition, double current, double frequency, double phase, const double *t,
                           const double *W, int64_t n_points);

/* define_test_beam (test_beam.c:17-56): emission of test particles by the
 * device integration loop.  NULL or electrons_per_macroparticle 0 removes it.
 * The reference gives each test particle only a position, momenta, velocities
 * and a charge (test_beam.c:91-103); the other values are those of a zeroed
 * slot (particle ID 0, extrema 0, inactive until its first push). */
int spiffe_gpu_set_test_beam(spiffe_gpu_instance *inst, const spiffe_test_beam_options *opt);

/* add_on_axis_fields (process_on_axis_field_definition, onAxisFields.c:18-172)
 * given the file's z and Ez columns (n points): z_offset is added to z, Ez
 * is scaled to peak |Ez| = Ez_peak, three derivatives are taken, and the push
 * then adds the field's off-axis expansion (addOffAxisExpansionFields,
 * onAxisFields.c:208-268) to every particle's fields, as advance_particles.c
 * :836-844 does.  phase is in radians (ON_AXIS_FIELD.phase; the command's
 * degrees times PI / 180).  Ez_peak = 0 ignores the field (the reference
 * warns).  A table the reference has already prepared gives the same device
 * field when passed with z_offset 0 and Ez_peak = its largest |Ez|.  Errors as the reference's: negative frequency,
 * expansion_order outside [0, 3], n <= 4, z not increasing, points not
 * equispaced to 1e-4.  At most 8 fields per instance. */
int spiffe_gpu_add_on_axis_field(spiffe_gpu_instance *inst, const double *z, const double *Ez, int64_t n,
                                 double z_offset, double Ez_peak, double frequency, double phase,
                                 int32_t expansion_order);
/* translate (setup_translation, translate.c:21-38): the moving window.  With
 * enable != 0, the device loop (and spiffe_gpu_translate_problem) moves the
 * problem by one dz whenever a particle lies past z_trigger, which must be in
 * [zmin+dz, zmax-dz].  The reference's reduction of the integration region
 * (z_lower, z_upper narrower than the mesh, translate.c:59-121) is not
 * provided. */
int spiffe_gpu_set_translation(spiffe_gpu_instance *inst, int32_t enable, double z_trigger);
/* translate_problem, translate.c:40-197: if any particle is past the trigger,
 * the TM (and TE) field rows move down one row (the top row zeroed), zmin,
 * zmax and the trigger grow by dz; *translated (may be NULL) is 1 then, and
 * *total (may be NULL) receives the total translation (FIELDS.zt).  Waits for
 * the device (one flag is read back). */
int spiffe_gpu_translate_problem(spiffe_gpu_instance *inst, int32_t *translated, double *total);
/* do_status_printouts' values (status_pr.c:18-356, kinetic_energy and
 * field_energy :358-452) for the current state; reads the fields and the
 * beam back, so it waits for the device.  JCathode is the first cathode's
 * current density (0 without one); EzOOEMin/Max are the last push's extremes
 * of the summed on-axis Ez (+inf/-inf when no particle met an on-axis field,
 * 0 before the first push). */
int spiffe_gpu_status_report(spiffe_gpu_instance *inst, spiffe_status_row *row);
/* The summed on-axis fields' (Ez, Er, Bphi) at (z, r) and time t, as the
 * push adds them; profile != 0 sets sine and cosine to 1 (the fields_used
 * output, onAxisFields.c:130-170). */
int spiffe_gpu_on_axis_fields_at(spiffe_gpu_instance *inst, double z, double r, double t, int32_t profile,
                                 double *EzErBphi);

/* perform_integration (integrate.c:24-194) on the device: configure, the
 * setup before the loop (:125-133), then any number of loop steps. */
int spiffe_gpu_configure_run(spiffe_gpu_instance *inst, int32_t space_charge, const spiffe_push_options *push,
                             const spiffe_poisson_options *poisson);
int spiffe_gpu_run_begin(spiffe_gpu_instance *inst, spiffe_poisson_report *report);
int spiffe_gpu_run_steps(spiffe_gpu_instance *inst, int64_t n_steps);

/* Waits for queued work and reports device-side errors. */
int spiffe_gpu_synchronize(spiffe_gpu_instance *inst);
int spiffe_gpu_counts(spiffe_gpu_instance *inst, int64_t *np, int64_t *np_active);
/* No counterpart in the reference.  Enqueues a copy of (np, npActive) into
 * out[0..1] behind the work queued so far, without waiting: a host loop can
 * read every step's particle count and synchronise once at the end.  `out`
 * should be page-locked host memory (pageable memory makes the copy wait);
 * the values are valid after spiffe_gpu_synchronize. */
int spiffe_gpu_counts_async(spiffe_gpu_instance *inst, int64_t *out);

/* Measurement (no counterpart in the reference, which has no timers): the device used by instances created afterwards on
 * this thread; the instance's CUDA stream (a cudaStream_t); per-phase device
 * time with CUDA events on that stream, in the order emission, deposition,
 * Poisson correction, FDTD, push (ms[5], count[5]; reading restarts the
 * accumulation); and the number of kernels this library has queued. */
int spiffe_gpu_select_device(int32_t device);
int spiffe_gpu_stream(spiffe_gpu_instance *inst, void **stream);
int spiffe_gpu_set_profiling(spiffe_gpu_instance *inst, int32_t on);
int spiffe_gpu_phase_times(spiffe_gpu_instance *inst, double *ms, int64_t *count);
int64_t spiffe_gpu_launch_count(void);
/* Split-precision form only (no counterpart in the reference): reorder the
 * particles by mesh cell every n steps of spiffe_gpu_run_steps (default 40;
 * 0 never), starting with the next step, and on the first step after each
 * beam upload; this keeps the gather and the deposition of neighbouring
 * threads on the same nodes.  No effect on the FP64 form. */
int spiffe_gpu_set_sort_interval(spiffe_gpu_instance *inst, int64_t n);
/* No counterpart in the reference (which has one solver).  The solver of the
 * split-precision form's Poisson correction and of spiffe_gpu_solve_poisson_cyl
 * with target 0: SPIFFE_POISSON_MULTIGRID (the default) solves the same
 * equations to the same stop rule, sum|residual| < accuracy sum|rhs| with the
 * residual over every updated node, by FP64 residual refinement around FP32
 * multigrid V-cycles, at most min(iteration_limit, 100) of them (the count is
 * reported in place of half-sweeps; -1 at the limit); SPIFFE_POISSON_SOR runs
 * the reference's red-black SOR.  Laplace solves (target 1, the imposed field)
 * always use SOR.  The FP64 form accepts SPIFFE_POISSON_SOR only. */
int spiffe_gpu_set_poisson_solver(spiffe_gpu_instance *inst, int32_t solver);
/* The split form's TM field update (integrate.c:308-433), one of
 * SPIFFE_FDTD_* (spiffe_b200_types.h).  All give the same bits.  The FP64
 * form accepts SPIFFE_FDTD_AUTO only. */
int spiffe_gpu_set_fdtd_kernel(spiffe_gpu_instance *inst, int32_t kernel);
/* Batched execution (no counterpart in the reference, which runs one problem
 * per process): advances n independent instances concurrently, instance i by
 * steps[i] steps of spiffe_gpu_run_steps, on `workers` host threads.  Each
 * instance keeps its own stream, so kernels of different instances overlap
 * on the device; an instance is advanced `chunk` steps at a time (<= 0: all
 * at once) by one thread at a time, the instances served round-robin.
 * done_ms[i] (may be null) receives the milliseconds from the call to the
 * completion of instance i.  Returns 0 or the first error; on an error the
 * other instances stop after their current chunk.  The instances must not be
 * used by other threads during the call. */
int spiffe_gpu_batch_run(spiffe_gpu_instance *const *inst, int32_t n, const int64_t *steps, int32_t workers,
                         int64_t chunk, double *done_ms);
/* Work done so far: out[0] particle-steps (active particles summed over
 * pushes), out[1] SOR half-sweeps, out[2] Poisson solves (either solver),
 * out[3] FDTD steps, out[4] multigrid V-cycles; out holds 5 values. */
int spiffe_gpu_work_counters(spiffe_gpu_instance *inst, int64_t *out);

#ifdef __cplusplus
}
#endif

#endif
