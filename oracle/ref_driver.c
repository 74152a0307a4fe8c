/* oracle/ref_driver.c -- TEST INFRASTRUCTURE (checker only, never shipped).
 *
 * Drives the reference spiffe code, compiled in place from its own sources by
 * oracle/Makefile, on one "session" that holds the same objects spiffe's main
 * holds (spiffe.c:97-122): the FIELDS problem, the BEAM, cathodes, screens,
 * antennae and the test-beam definition.  Commands are dispatched to the
 * reference's own command processors in the way spiffe.c:213-308 does, and
 * the per-step functions (advance_field_solutions, add_particle_currents,
 * advance_particles, add_poisson_correction, solve_poisson_cyl, cathode
 * emission) or the whole perform_integration() loop run on request.  Arrays
 * move in and out as contiguous (nz+1)x(nr+1) blocks, ir fastest, the layout
 * the CUDA path uses on the device.
 *
 * The reference keeps state in function-level statics (advance_particles.c:89,
 * poisson_correction.c:28-29, :463, solenoid.c:26), so one process serves one
 * session; the Python harness starts a fresh process per case.
 */
#include "spiffe.h"

uint64_t shim_rng_counter(void);
int64_t shim_sdds_column(SDDS_DATASET *t, const char *name, double **values);

static FIELDS EM;
static BEAM beam;
static CATHODE *cathode = NULL;
static long cathodes = 0;
static SCREEN *screen_defn = NULL;
static long n_screen_defns = 0;
static ANTENNA *antenna = NULL;
static long n_antennae = 0;
static TEST_BEAM_DEFN test_beam_defn;
static RESISTOR resistor_defns;
static FIELD_SAVING saving_defn;
static FIELD_OUTPUT field_output_defn;
static SNAPSHOT snapshot_defn;
static SECONDARY_EMISSION *secondary = NULL;
static long n_secondary = 0;
static EMITTER *emitter = NULL;
static long n_emitters = 0;
static SAMPLE_DEFN *sample_defn = NULL;
static long n_sample_defns = 0;
static int initialized = 0;

/* capacity of every particle and screen array: the reference sizes screen
 * buffers from max_np on its first advance_particles call only
 * (advance_particles.c:345-360), so the session fixes max_np up front */
static long capacity = 0;

static void beam_alloc(long n)
{
#define BA(f) beam.f = tmalloc(sizeof(*beam.f) * (uint64_t)n)
  BA(z); BA(r); BA(pz); BA(pr); BA(vz); BA(vr); BA(r0); BA(z0); BA(t0);
  BA(r_pphi); BA(vphi); BA(Q); BA(rmin); BA(rmax); BA(zmin); BA(zmax);
  BA(generation); BA(particleID); BA(status);
#undef BA
  beam.max_np = n;
}

int ref_session_init(long particle_capacity)
{
  if (initialized)
    return -1;
  initialized = 1;
  memset(&EM, 0, sizeof(EM));
  shim_n_closed_tables = 0;
  shim_n_updated_tables = 0;
  memset(&beam, 0, sizeof(beam));
  EM.run_name = "checker";
  EM.rootname = strdup("checker");
  beam.nextParticleID = 1;
  capacity = particle_capacity > 16 ? particle_capacity : 16;
  beam_alloc(capacity);
  test_beam_defn.electrons_per_macroparticle = 0;
  resistor_defns.n_resistors = 0;
  saving_defn.filename = NULL;
  field_output_defn.filename = NULL;
  snapshot_defn.filename = NULL;
  return 0;
}

/* One command in namelist text form, dispatched as spiffe.c:216-308 does for
 * the commands on the checked path.  Returns 0, or -1 for an unknown command. */
int ref_command(const char *text)
{
  NAMELIST_TEXT nl;
  char *s = strdup(text);
  int rc = 0;
  if (!scan_namelist(&nl, s)) {
    free(s);
    return -2;
  }
  if (strcmp(nl.group_name, "define_geometry") == 0)
    process_geometry_definition(&EM, &nl);
  else if (strcmp(nl.group_name, "define_cathode") == 0)
    process_cathode_definition(&EM, &cathode, &cathodes, &nl);
  else if (strcmp(nl.group_name, "define_screen") == 0)
    n_screen_defns = process_screen_definition(&screen_defn, n_screen_defns, &EM, &nl);
  else if (strcmp(nl.group_name, "define_solenoid") == 0)
    process_solenoid_definition(&EM, &nl);
  else if (strcmp(nl.group_name, "set_constant_fields") == 0 || strcmp(nl.group_name, "constant_fields") == 0)
    set_constant_fields(&EM, &nl);
  else if (strcmp(nl.group_name, "poisson_correction") == 0)
    setup_poisson_correction(&EM, &nl);
  else if (strcmp(nl.group_name, "define_antenna") == 0) {
    process_antenna_definition(&antenna, n_antennae, &EM, &nl);
    n_antennae++;
  } else if (strcmp(nl.group_name, "define_field_saving") == 0)
    process_field_saving_definition(&saving_defn, &EM, &nl);
  else if (strcmp(nl.group_name, "define_snapshots") == 0)
    process_snapshot_definition(&snapshot_defn, &EM, &nl);
  else if (strcmp(nl.group_name, "define_field_output") == 0)
    process_field_output_definition(&field_output_defn, &EM, &nl);
  else if (strcmp(nl.group_name, "translate") == 0)
    setup_translation(&EM, &nl);
  else if (strcmp(nl.group_name, "add_on_axis_fields") == 0)
    process_on_axis_field_definition(&EM, &nl);
  else if (strcmp(nl.group_name, "define_test_beam") == 0)
    process_testbeam_definition(&test_beam_defn, &EM, &nl);
  else if (strcmp(nl.group_name, "define_field_sampling") == 0)
    process_sampling_definition(&sample_defn, n_sample_defns++, &EM, &nl);
  else if (strcmp(nl.group_name, "define_emitter") == 0) {
    process_emitter_definition(&EM, &emitter, &n_emitters, &nl);
    /* the definition leaves stop_step unset (emitter.c:65-90) and the first
     * emission call compares it (:186): fresh heap memory holds 0 there, and
     * the checker makes it so every time */
    emitter[n_emitters - 1].stop_step = 0;
  } else if (strcmp(nl.group_name, "define_secondary_emission") == 0)
    processSecondaryEmissionDefinition(&secondary, &n_secondary, &nl, &EM);
  else if (strcmp(nl.group_name, "integrate") == 0)
    perform_integration(&EM, &beam, cathode, cathodes, &test_beam_defn, antenna, n_antennae, &resistor_defns,
                        sample_defn, n_sample_defns, &saving_defn, &snapshot_defn, screen_defn, n_screen_defns,
                        &field_output_defn, secondary, n_secondary, emitter, n_emitters, &nl);
  else
    rc = -1;
  free_namelist_text(&nl);
  free(s);
  if (beam.max_np != capacity) {
    fprintf(stderr, "ref_driver: particle capacity exceeded (%ld > %ld)\n", beam.max_np, capacity);
    exit(3);
  }
  return rc;
}

/* getBoundaryPoints (grid_drawing.c:541-760) of the last define_geometry:
 * the emitter surface of `material`, up to `max` nodes; the direction of the
 * last node, which the reference leaves unset, is reported as 0 */
long ref_boundary_points(long material, int32_t *iz, int32_t *ir, int16_t *dir, long max)
{
  long *z = NULL, *r = NULL, i, n;
  short *d = NULL;
  n = getBoundaryPoints(material, &z, &r, &d);
  for (i = 0; i < n && i < max; i++) {
    iz[i] = (int32_t)z[i];
    ir[i] = (int32_t)r[i];
    dir[i] = i < n - 1 ? d[i] : 0;
  }
  free(z);
  free(r);
  free(d);
  return n;
}

/* ------------------------------------------------------------------ mesh */

void ref_get_mesh(int32_t *nz, int32_t *nr, double *geom, int32_t *bc, uint32_t *modes)
{
  *nz = EM.nz;
  *nr = EM.nr;
  geom[0] = EM.zmin;
  geom[1] = EM.zmax;
  geom[2] = EM.rmax;
  geom[3] = EM.dz;
  geom[4] = EM.dr;
  geom[5] = EM.dti;
  geom[6] = EM.time;
  geom[7] = EM.start_time;
  bc[0] = (int32_t)EM.lower_bc;
  bc[1] = (int32_t)EM.upper_bc;
  bc[2] = (int32_t)EM.right_bc;
  bc[3] = (int32_t)EM.left_bc;
  *modes = (uint32_t)EM.modes;
}

/* Sets the integration time state that perform_integration normally sets
 * (integrate.c:86-92, :138) so single step functions can run. */
void ref_set_time(double dt, double start_time, int64_t time_step, uint32_t modes)
{
  EM.dti = dt;
  EM.start_time = start_time;
  EM.time_step = time_step;
  EM.time = time_step * dt + start_time;
  EM.modes = modes;
}

void ref_set_constant_fields(const double *c, const int16_t *turn_off)
{
  EM.constantEz = c[0];
  EM.constantEr = c[1];
  EM.constantEphi = c[2];
  EM.constantBz = c[3];
  EM.constantBr = c[4];
  EM.constantBphi = c[5];
  EM.turnOffEz = turn_off[0];
  EM.turnOffEr = turn_off[1];
  EM.turnOffEphi = turn_off[2];
  EM.turnOffBz = turn_off[3];
  EM.turnOffBr = turn_off[4];
  EM.turnOffBphi = turn_off[5];
}

static double **field_by_name(const char *name, int create)
{
  double ***slot = NULL;
  if (!strcmp(name, "Ez")) slot = &EM.Ez;
  else if (!strcmp(name, "Er")) slot = &EM.Er;
  else if (!strcmp(name, "Bphi")) slot = &EM.Bphi;
  else if (!strcmp(name, "Bphi2")) slot = &EM.Bphi2;
  else if (!strcmp(name, "Jz")) slot = &EM.Jz;
  else if (!strcmp(name, "Jr")) slot = &EM.Jr;
  else if (!strcmp(name, "Ephi")) slot = &EM.Ephi;
  else if (!strcmp(name, "Jphi")) slot = &EM.Jphi;
  else if (!strcmp(name, "Br")) slot = &EM.Br;
  else if (!strcmp(name, "Br2")) slot = &EM.Br2;
  else if (!strcmp(name, "Bz")) slot = &EM.Bz;
  else if (!strcmp(name, "Bz2")) slot = &EM.Bz2;
  else if (!strcmp(name, "EzImposed")) slot = &EM.EzImposed;
  else if (!strcmp(name, "ErImposed")) slot = &EM.ErImposed;
  else if (!strcmp(name, "PsiImposed")) slot = &EM.PsiImposed;
  else if (!strcmp(name, "BzImposed")) slot = &EM.BzImposed;
  else if (!strcmp(name, "BrImposed")) slot = &EM.BrImposed;
  else if (!strcmp(name, "Psi")) slot = &EM.Psi;
  else if (!strcmp(name, "Q")) slot = &EM.Q;
  if (!slot)
    return NULL;
  if (!*slot && create)
    *slot = (double **)zarray_2d(sizeof(double), EM.nz + 1, EM.nr + 1);
  return *slot;
}

/* rows of a zarray_2d may have been permuted; copy row by row */
int ref_get_field(const char *name, double *out)
{
  double **a = field_by_name(name, 0);
  long iz;
  if (!a)
    return -1;
  for (iz = 0; iz <= EM.nz; iz++)
    memcpy(out + iz * (EM.nr + 1), a[iz], sizeof(double) * (EM.nr + 1));
  return 0;
}

int ref_set_field(const char *name, const double *in)
{
  double **a = field_by_name(name, 1);
  long iz;
  if (!a)
    return -1;
  for (iz = 0; iz <= EM.nz; iz++)
    memcpy(a[iz], in + iz * (EM.nr + 1), sizeof(double) * (EM.nr + 1));
  return 0;
}

int ref_get_flags(int16_t *out)
{
  long iz;
  for (iz = 0; iz <= EM.nz; iz++)
    memcpy(out + iz * (EM.nr + 1), EM.metal_flags[iz], sizeof(short) * (EM.nr + 1));
  return 0;
}

int ref_set_flags(const int16_t *in)
{
  long iz;
  for (iz = 0; iz <= EM.nz; iz++)
    memcpy(EM.metal_flags[iz], in + iz * (EM.nr + 1), sizeof(short) * (EM.nr + 1));
  return 0;
}

/* ------------------------------------------------------------------ beam */

static double *beam_double(const char *name)
{
  if (!strcmp(name, "z")) return beam.z;
  if (!strcmp(name, "r")) return beam.r;
  if (!strcmp(name, "pz")) return beam.pz;
  if (!strcmp(name, "pr")) return beam.pr;
  if (!strcmp(name, "r_pphi")) return beam.r_pphi;
  if (!strcmp(name, "vz")) return beam.vz;
  if (!strcmp(name, "vr")) return beam.vr;
  if (!strcmp(name, "vphi")) return beam.vphi;
  if (!strcmp(name, "Q")) return beam.Q;
  if (!strcmp(name, "r0")) return beam.r0;
  if (!strcmp(name, "z0")) return beam.z0;
  if (!strcmp(name, "t0")) return beam.t0;
  if (!strcmp(name, "rmin")) return beam.rmin;
  if (!strcmp(name, "rmax")) return beam.rmax;
  if (!strcmp(name, "zmin")) return beam.zmin;
  if (!strcmp(name, "zmax")) return beam.zmax;
  return NULL;
}

void ref_get_beam_counts(int64_t *counts, double *scalars)
{
  counts[0] = beam.np;
  counts[1] = beam.npActive;
  counts[2] = beam.max_np;
  counts[3] = beam.nextParticleID;
  scalars[0] = beam.QoMC;
  scalars[1] = beam.stiffness;
}

void ref_set_beam_counts(const int64_t *counts, const double *scalars)
{
  beam.np = counts[0];
  beam.npActive = counts[1];
  beam.nextParticleID = (int32_t)counts[3];
  beam.QoMC = scalars[0];
  beam.stiffness = scalars[1];
}

/* doubles, or "particleID" (int32), "generation" (int16), "status" (uint64) */
int ref_get_beam(const char *name, void *out)
{
  double *d = beam_double(name);
  if (d) {
    memcpy(out, d, sizeof(double) * (size_t)beam.np);
    return 0;
  }
  if (!strcmp(name, "particleID"))
    memcpy(out, beam.particleID, sizeof(int32_t) * (size_t)beam.np);
  else if (!strcmp(name, "generation"))
    memcpy(out, beam.generation, sizeof(short) * (size_t)beam.np);
  else if (!strcmp(name, "status"))
    memcpy(out, beam.status, sizeof(unsigned long) * (size_t)beam.np);
  else
    return -1;
  return 0;
}

int ref_set_beam(const char *name, const void *in, int64_t n)
{
  double *d = beam_double(name);
  if (n > capacity)
    return -2;
  if (d) {
    memcpy(d, in, sizeof(double) * (size_t)n);
    return 0;
  }
  if (!strcmp(name, "particleID"))
    memcpy(beam.particleID, in, sizeof(int32_t) * (size_t)n);
  else if (!strcmp(name, "generation"))
    memcpy(beam.generation, in, sizeof(short) * (size_t)n);
  else if (!strcmp(name, "status"))
    memcpy(beam.status, in, sizeof(unsigned long) * (size_t)n);
  else
    return -1;
  return 0;
}

/* ------------------------------------------------------------- step parts */

void ref_calculate_areas_and_setup(void)
{
  extern void calculate_areas(FIELDS *);
  if (!EM.area_c) {
    EM.area_c = tmalloc(sizeof(double) * (EM.nr + 1));
    EM.area_o = tmalloc(sizeof(double) * (EM.nr + 1));
  }
  calculate_areas(&EM);
}

void ref_advance_field_solutions(void) { advance_field_solutions(&EM); }
void ref_zero_current_arrays(void) { zero_current_arrays(&EM); }
void ref_add_particle_currents(void) { add_particle_currents(&EM, &beam); }
void ref_add_poisson_correction(long space_charge) { add_poisson_correction(&EM, &beam, space_charge); }
void ref_compute_imposed_Efield(long initialize) { compute_imposed_Efield(&EM, initialize); }
void ref_add_antenna_excitation(double time) { add_antenna_excitation(&EM, antenna, n_antennae, time); }
void ref_set_current_density(void)
{
  long i;
  for (i = 0; i < cathodes; i++)
    set_current_density(cathode + i, &EM);
}
void ref_emit(void)
{
  long i;
  for (i = 0; i < cathodes; i++)
    emit_electrons_from_cathode(&beam, cathode + i, &EM, i);
  if (beam.max_np != capacity) {
    fprintf(stderr, "ref_driver: particle capacity exceeded\n");
    exit(3);
  }
}

/* advance_particles with the session's screens; z_forces_start as in the
 * integrate command (integrate.nl:18, default -1) */
void ref_advance_particles(double z_forces_start)
{
  advance_particles(&beam, &EM, &test_beam_defn, screen_defn, n_screen_defns, NULL, z_forces_start, NULL, 0);
}

long ref_solve_poisson_cyl(double *psi, const double *rhs, int has_rhs, double accuracy, long iteration_limit)
{
  double **P = (double **)zarray_2d(sizeof(double), EM.nz + 1, EM.nr + 1);
  double **R = has_rhs ? (double **)zarray_2d(sizeof(double), EM.nz + 1, EM.nr + 1) : NULL;
  long iz, n;
  for (iz = 0; iz <= EM.nz; iz++) {
    memcpy(P[iz], psi + iz * (EM.nr + 1), sizeof(double) * (EM.nr + 1));
    if (R)
      memcpy(R[iz], rhs + iz * (EM.nr + 1), sizeof(double) * (EM.nr + 1));
  }
  n = solve_poisson_cyl(P, R, EM.metal_flags, EM.left_bc, EM.right_bc, EM.nz, EM.nr, EM.dz, EM.dr,
                        accuracy, iteration_limit);
  for (iz = 0; iz <= EM.nz; iz++)
    memcpy(psi + iz * (EM.nr + 1), P[iz], sizeof(double) * (EM.nr + 1));
  free_zarray_2d((void **)P, 0, 0);
  if (R)
    free_zarray_2d((void **)R, 0, 0);
  return n;
}

/* One step of the perform_integration loop body (integrate.c:136-193) for the
 * commands on the checked path, with step counters advanced as the loop does. */
void ref_step(long space_charge, double z_forces_start)
{
  long i;
  if (EM.imposedEFieldRampTime > 0)
    compute_imposed_Efield(&EM, 0);
  EM.time = EM.time_step * EM.dti + EM.start_time;
  for (i = 0; i < cathodes; i++)
    emit_electrons_from_cathode(&beam, cathode + i, &EM, i);
  emit_test_particles(&beam, &test_beam_defn, &EM);
  zero_current_arrays(&EM);
  if (space_charge)
    add_particle_currents(&EM, &beam);
  add_antenna_excitation(&EM, antenna, n_antennae, EM.time + EM.dti / 2);
  add_poisson_correction(&EM, &beam, space_charge);
  advance_field_solutions(&EM);
  advance_particles(&beam, &EM, &test_beam_defn, screen_defn, n_screen_defns, NULL, z_forces_start, NULL, 0);
  for (i = 0; i < cathodes; i++)
    set_current_density(cathode + i, &EM);
  EM.time_step++;
  if (beam.max_np != capacity) {
    fprintf(stderr, "ref_driver: particle capacity exceeded\n");
    exit(3);
  }
}

/* -------------------------------------------- snapshots and field output */

/* every row written to the beam-snapshot table (which 0) or the field-output
 * table (which 1), all pages in order; returns the row count, -1 for an
 * unknown column */
/* which: 0 the beam snapshots, 1 the field output, 2 + k the k-th output
 * table the reference closed inside a command, 3 + SHIM_MAX_CLOSED_TABLES
 * the field saves, 100 + k the k-th table it wrote row by row (the status
 * file), 200 + k the log_file of the k-th define_secondary_emission, 300 + k
 * the file of the k-th define_field_sampling */
static SDDS_DATASET *ref_table(long which)
{
  if (which == 0)
    return &snapshot_defn.table;
  if (which == 1)
    return &field_output_defn.SDDSout;
  if (which == 3 + SHIM_MAX_CLOSED_TABLES)
    return &saving_defn.outTable;
  if (which >= 300)
    return which - 300 < n_sample_defns ? &sample_defn[which - 300].outTable : NULL;
  if (which >= 200)
    return which - 200 < n_secondary && secondary[which - 200].logFile ? &secondary[which - 200].SDDSlog : NULL;
  if (which >= 100)
    return which - 100 < shim_n_updated_tables ? &shim_updated_tables[which - 100] : NULL;
  if (which - 2 < shim_n_closed_tables)
    return &shim_closed_tables[which - 2];
  return NULL;
}

int64_t ref_table_column(long which, const char *column, double *out)
{
  double *v;
  SDDS_DATASET *t = ref_table(which);
  int64_t n;
  if (!t)
    return -1;
  n = shim_sdds_column(t, column, &v);
  if (n > 0 && v && out)
    memcpy(out, v, sizeof(double) * (size_t)n);
  return v ? n : -1;
}

int64_t ref_table_pages(long which)
{
  SDDS_DATASET *t = ref_table(which);
  return t ? t->pages : -1;
}

/* --------------------------------------------------------------- screens */

int64_t ref_screen_count(long is)
{
  double *v;
  if (is < 0 || is >= n_screen_defns)
    return -1;
  return shim_sdds_column(&screen_defn[is].table, "r", &v);
}

/* all rows the reference wrote to screen `is`, in write order */
int64_t ref_screen_column(long is, const char *column, double *out)
{
  double *v;
  int64_t n;
  if (is < 0 || is >= n_screen_defns)
    return -1;
  n = shim_sdds_column(&screen_defn[is].table, column, &v);
  if (n > 0 && v)
    memcpy(out, v, sizeof(double) * (size_t)n);
  return n;
}

/* rows written by the most recent advance_particles call (the live buffer) */
int64_t ref_screen_last_step(long is, int q, double *out)
{
  if (is < 0 || is >= n_screen_defns || q < 0 || q >= N_SCREEN_QUANS)
    return -1;
  if (screen_defn[is].nb && screen_defn[is].buffer[q])
    memcpy(out, screen_defn[is].buffer[q], sizeof(double) * (size_t)screen_defn[is].nb);
  return screen_defn[is].nb;
}

double ref_kinetic_energy(void) { return kinetic_energy(&beam); }

void ref_field_energy(double *out)
{
  double *e;
  ref_calculate_areas_and_setup();
  e = field_energy(&EM);
  out[0] = e[0];
  out[1] = e[1];
}

int64_t ref_time_step(void) { return EM.time_step; }
uint64_t ref_rng_counter(void) { return shim_rng_counter(); }
