/* spiffe_b200/dropin/spiffe_dropin.c -- link-time drop-in for spiffe's hot-path functions.
 *
 * Defines, with the reference's own prototypes (spiffe.h:476, :526-534,
 * :550-557, :561), the functions perform_integration calls every step, on
 * top of the device library's C ABI (spiffe_b200.h):
 *
 *   advance_field_solutions     integrate.c:277       (FDTD, TM and TE)
 *   add_particle_currents       space_charge.c:34     (current deposition)
 *   advance_particles           advance_particles.c:67 (gather, push, losses, screens)
 *   solve_poisson_cyl           poisson.c:17          (red-black SOR)
 *   setup_poisson_correction, add_poisson_correction, compute_imposed_Efield
 *                               poisson_correction.c:31, :73, :456 (they share
 *                               that file's settings, so all three are defined)
 *
 * plus spiffe_gpu_attach / spiffe_gpu_sync_to_host / spiffe_gpu_detach.
 *
 * It is compiled inside spiffe's source tree, against its spiffe.h and the
 * namelist header nlpp generates from poisson_correction.nl, and linked (or
 * preloaded) ahead of the reference's objects so that these definitions are
 * the ones the reference's callers bind to.  The rest of spiffe (command
 * processing, emission, diagnostics, output) is unchanged.
 *
 * Ownership: the host arrays of FIELDS and BEAM stay authoritative, as the
 * reference's other code reads and writes them between these calls (the
 * cathode appends particles, zero_current_arrays clears J, diagnostics read
 * everything).  Each function therefore copies in the arrays it reads, runs
 * on the device, and copies out the arrays it writes, row by row (translate
 * may permute the row pointers, translate.c:129-149).  The device instance
 * mirroring a problem is kept per FIELDS pointer (and created again when the
 * beam outgrows it); it uses the FP64 form, whose arithmetic is the
 * reference's, with the reference's compaction and screen-momentum
 * behaviour and the ordered deposition.  Secondary emission stays the
 * reference's: the device reports each lost particle's loss point and the
 * reference's queueSecondaryEmission and emitSecondaryElectrons (which
 * appends to the host beam) do the rest.  Errors call bomb() as the
 * reference does.  Not available: on-axis fields.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "spiffe.h"
#include "poisson_correction.h" /* nlpp: the poisson_correction namelist and its variables */

#include "spiffe_b200.h"

#define DROPIN_MAX 16

typedef struct {
  FIELDS *F;
  spiffe_gpu_instance *inst;
  int32_t nz, nr;
  double zmin;     /* the moving window (translate.c:40-197) changes it */
  unsigned modes;  /* TM/TE bits */
  int64_t capacity;
  size_t nodes;
  double *stage[20];          /* contiguous host copies, one per array */
  int16_t *flags;             /* contiguous metal flags */
  int n_screens;              /* screens registered on the device */
  double screen_z[SPIFFE_MAX_SCREENS];
  long screen_dir[SPIFFE_MAX_SCREENS];
  spiffe_screen_set scr;      /* download buffers */
  int64_t scr_capacity;
  int lost_on;                /* the device records lost particles */
} Mirror;

static Mirror mirrors[DROPIN_MAX];
static int n_mirrors;

/* the standalone solve_poisson_cyl's instance (keyed by its flags array) */
static Mirror solver;
static short **solver_flags;

static void fail(const char *what)
{
  static char msg[512];
  snprintf(msg, sizeof(msg), "%s: %s", what, spiffe_gpu_last_error());
  bomb(msg, NULL);
}

static void check(int rc, const char *what)
{
  if (rc)
    fail(what);
}

static void mesh_of(const FIELDS *F, spiffe_mesh *m)
{
  memset(m, 0, sizeof(*m));
  m->nz = F->nz;
  m->nr = F->nr;
  m->zmin = F->zmin;
  m->zmax = F->zmax;
  m->rmax = F->rmax;
  m->dz = F->dz;
  m->dr = F->dr;
  m->lower_bc = (int32_t)F->lower_bc;
  m->upper_bc = (int32_t)F->upper_bc;
  m->right_bc = (int32_t)F->right_bc;
  m->left_bc = (int32_t)F->left_bc;
  m->modes = (uint32_t)F->modes;
  m->dt = F->dti;
  m->start_time = F->start_time;
  m->time = F->time;
  m->time_step = F->time_step;
  m->constant_E[0] = F->constantEz;
  m->constant_E[1] = F->constantEr;
  m->constant_E[2] = F->constantEphi;
  m->constant_B[0] = F->constantBz;
  m->constant_B[1] = F->constantBr;
  m->constant_B[2] = F->constantBphi;
  m->turn_off[0] = F->turnOffEz;
  m->turn_off[1] = F->turnOffEr;
  m->turn_off[2] = F->turnOffEphi;
  m->turn_off[3] = F->turnOffBz;
  m->turn_off[4] = F->turnOffBr;
  m->turn_off[5] = F->turnOffBphi;
  m->has_solenoid = F->BzImposed != NULL;
  m->imposed_ramp_time = F->imposedEFieldRampTime;
  m->imposed_flat_top_time = F->imposedEFieldFlatTopTime;
}

/* rows of a row-pointer array <-> one contiguous block */
static void gather_rows(double **a, double *out, int32_t nz, int32_t nr)
{
  for (int32_t iz = 0; iz <= nz; iz++)
    memcpy(out + (size_t)iz * (nr + 1), a[iz], sizeof(double) * (nr + 1));
}

static void scatter_rows(double *in, double **a, int32_t nz, int32_t nr)
{
  for (int32_t iz = 0; iz <= nz; iz++)
    memcpy(a[iz], in + (size_t)iz * (nr + 1), sizeof(double) * (nr + 1));
}

enum {
  A_EZ, A_ER, A_BPHI, A_BPHI2, A_JZ, A_JR, A_EPHI, A_JPHI, A_BR, A_BR2, A_BZ, A_BZ2,
  A_EZI, A_ERI, A_PSII, A_BZI, A_BRI, A_PSI, A_Q, A_N
};

static double **field_rows(FIELDS *F, int k)
{
  switch (k) {
  case A_EZ: return F->Ez;
  case A_ER: return F->Er;
  case A_BPHI: return F->Bphi;
  case A_BPHI2: return F->Bphi2;
  case A_JZ: return F->Jz;
  case A_JR: return F->Jr;
  case A_EPHI: return F->Ephi;
  case A_JPHI: return F->Jphi;
  case A_BR: return F->Br;
  case A_BR2: return F->Br2;
  case A_BZ: return F->Bz;
  case A_BZ2: return F->Bz2;
  case A_EZI: return F->EzImposed;
  case A_ERI: return F->ErImposed;
  case A_PSII: return F->PsiImposed;
  case A_BZI: return F->BzImposed;
  case A_BRI: return F->BrImposed;
  case A_PSI: return F->Psi;
  case A_Q: return F->Q;
  }
  return NULL;
}

static double **set_slot(spiffe_field_set *s, int k, double *p)
{
  double **slot[A_N] = {&s->Ez, &s->Er, &s->Bphi, &s->Bphi2, &s->Jz, &s->Jr, &s->Ephi, &s->Jphi, &s->Br, &s->Br2,
                        &s->Bz, &s->Bz2, &s->EzImposed, &s->ErImposed, &s->PsiImposed, &s->BzImposed, &s->BrImposed,
                        &s->Psi, &s->Q};
  *slot[k] = p;
  return slot[k];
}

static double *stage_of(Mirror *M, int k)
{
  if (!M->stage[k] && !(M->stage[k] = malloc(sizeof(double) * M->nodes)))
    bomb("memory allocation failure (spiffe drop-in)", NULL);
  return M->stage[k];
}

/* copies the listed arrays that exist on the host to the device */
static void upload(Mirror *M, FIELDS *F, const int *ks, int n)
{
  spiffe_field_set s;
  memset(&s, 0, sizeof(s));
  for (int i = 0; i < n; i++) {
    double **a = field_rows(F, ks[i]);
    if (!a)
      continue;
    double *st = stage_of(M, ks[i]);
    gather_rows(a, st, M->nz, M->nr);
    set_slot(&s, ks[i], st);
  }
  check(spiffe_gpu_upload_fields(M->inst, &s), "spiffe drop-in: field upload failed");
}

static void download(Mirror *M, FIELDS *F, const int *ks, int n)
{
  spiffe_field_set s;
  memset(&s, 0, sizeof(s));
  for (int i = 0; i < n; i++)
    if (field_rows(F, ks[i]))
      set_slot(&s, ks[i], stage_of(M, ks[i]));
  check(spiffe_gpu_download_fields(M->inst, &s), "spiffe drop-in: field download failed");
  for (int i = 0; i < n; i++) {
    double **a = field_rows(F, ks[i]);
    if (a)
      scatter_rows(M->stage[ks[i]], a, M->nz, M->nr);
  }
}

static void mirror_free(Mirror *M)
{
  if (M->inst)
    spiffe_gpu_destroy(M->inst);
  for (int k = 0; k < 20; k++)
    free(M->stage[k]);
  free(M->flags);
  for (int q = 0; q < SPIFFE_SCREEN_QUANS; q++)
    free(M->scr.col[q]);
  free(M->scr.rmin);
  free(M->scr.rmax);
  free(M->scr.zmin);
  free(M->scr.zmax);
  free(M->scr.generation);
  free(M->scr.particleID);
  memset(M, 0, sizeof(*M));
}

static void mirror_create(Mirror *M, FIELDS *F, short **flags, int64_t capacity)
{
  spiffe_mesh m;
  mesh_of(F, &m);
  M->F = F;
  M->nz = F->nz;
  M->nr = F->nr;
  M->zmin = F->zmin;
  M->modes = (unsigned)F->modes & 3u;
  M->nodes = (size_t)(F->nz + 1) * (F->nr + 1);
  M->capacity = capacity;
  M->flags = malloc(sizeof(int16_t) * M->nodes);
  if (!M->flags)
    bomb("memory allocation failure (spiffe drop-in)", NULL);
  for (int32_t iz = 0; iz <= F->nz; iz++)
    for (int32_t ir = 0; ir <= F->nr; ir++)
      M->flags[(size_t)iz * (F->nr + 1) + ir] = flags[iz][ir];
  check(spiffe_gpu_create(&m, M->flags, SPIFFE_PRECISION_F64, capacity, &M->inst),
        "spiffe drop-in: instance creation failed");
  check(spiffe_gpu_set_deposit_order(M->inst, 1), "spiffe drop-in: deposit order");
}

/* the mirror of F, with room for `capacity` particles */
static Mirror *mirror_of(FIELDS *F, int64_t capacity)
{
  Mirror *M = NULL;
  for (int i = 0; i < n_mirrors; i++)
    if (mirrors[i].F == F)
      M = mirrors + i;
  if (M && (M->nz != F->nz || M->nr != F->nr || M->zmin != F->zmin || M->modes != ((unsigned)F->modes & 3u) ||
            M->capacity < capacity))
    mirror_free(M); /* a new mesh or window, or a beam that outgrew the instance */
  if (!M)
    for (int i = 0; i < n_mirrors && !M; i++)
      if (!mirrors[i].inst)
        M = mirrors + i;
  if (!M) {
    if (n_mirrors == DROPIN_MAX)
      bomb("too many problems for the spiffe drop-in", NULL);
    M = mirrors + n_mirrors++;
  }
  if (!M->inst)
    mirror_create(M, F, F->metal_flags, capacity < 1024 ? 1024 : capacity + capacity / 4);
  spiffe_mesh m;
  mesh_of(F, &m);
  check(spiffe_gpu_set_mesh(M->inst, &m), "spiffe drop-in: mesh update failed");
  return M;
}

static void beam_set_of(BEAM *b, spiffe_beam_set *s)
{
  memset(s, 0, sizeof(*s));
  s->np = b->np;
  s->npActive = b->npActive;
  s->capacity = b->max_np;
  s->nextParticleID = b->nextParticleID;
  s->QoMC = b->QoMC;
  s->stiffness = b->stiffness;
  s->z = b->z;
  s->r = b->r;
  s->pz = b->pz;
  s->pr = b->pr;
  s->r_pphi = b->r_pphi;
  s->vz = b->vz;
  s->vr = b->vr;
  s->vphi = b->vphi;
  s->Q = b->Q;
  s->r0 = b->r0;
  s->z0 = b->z0;
  s->t0 = b->t0;
  s->rmin = b->rmin;
  s->rmax = b->rmax;
  s->zmin = b->zmin;
  s->zmax = b->zmax;
  s->particleID = b->particleID;
  s->generation = b->generation;
  s->status = (uint64_t *)b->status;
}

static void beam_upload(Mirror *M, BEAM *b)
{
  spiffe_beam_set s;
  beam_set_of(b, &s);
  check(spiffe_gpu_upload_beam(M->inst, &s), "spiffe drop-in: beam upload failed");
}

static void beam_download(Mirror *M, BEAM *b)
{
  spiffe_beam_set s;
  beam_set_of(b, &s);
  check(spiffe_gpu_download_beam(M->inst, &s), "spiffe drop-in: beam download failed");
  b->np = (long)s.np;
  b->npActive = (long)s.npActive;
  b->nextParticleID = s.nextParticleID;
}

/* ------------------------------------------------------------ integrate.c */

static const int FDTD_IN[] = {A_EZ, A_ER, A_BPHI, A_BPHI2, A_JZ, A_JR, A_EPHI, A_JPHI, A_BR, A_BR2, A_BZ, A_BZ2};
static const int FDTD_OUT[] = {A_EZ, A_ER, A_BPHI, A_BPHI2, A_EPHI, A_BR, A_BR2, A_BZ, A_BZ2};

void advance_field_solutions(FIELDS *EM_problem)
{
  Mirror *M = mirror_of(EM_problem, 0);
  upload(M, EM_problem, FDTD_IN, sizeof(FDTD_IN) / sizeof(int));
  check(spiffe_gpu_advance_field_solutions(M->inst), "advance_field_solutions");
  download(M, EM_problem, FDTD_OUT, sizeof(FDTD_OUT) / sizeof(int));
}

/* --------------------------------------------------------- space_charge.c */

static const int CUR[] = {A_JZ, A_JR, A_JPHI};

void add_particle_currents(FIELDS *EM_problem, BEAM *beam)
{
  Mirror *M = mirror_of(EM_problem, beam->max_np);
  upload(M, EM_problem, CUR, 3);
  beam_upload(M, beam);
  check(spiffe_gpu_add_particle_currents(M->inst), "add_particle_currents");
  download(M, EM_problem, CUR, 3);
}

/* ---------------------------------------------------- advance_particles.c */

static const int GATHER[] = {A_EZ, A_ER, A_BPHI, A_BPHI2, A_EPHI, A_BR2, A_BZ2, A_EZI, A_ERI, A_BZI, A_BRI};

static void screen_buffers(Mirror *M, int64_t capacity)
{
  if (M->scr_capacity >= capacity)
    return;
  for (int q = 0; q < SPIFFE_SCREEN_QUANS; q++)
    M->scr.col[q] = realloc(M->scr.col[q], sizeof(double) * capacity);
  M->scr.rmin = realloc(M->scr.rmin, sizeof(double) * capacity);
  M->scr.rmax = realloc(M->scr.rmax, sizeof(double) * capacity);
  M->scr.zmin = realloc(M->scr.zmin, sizeof(double) * capacity);
  M->scr.zmax = realloc(M->scr.zmax, sizeof(double) * capacity);
  M->scr.generation = realloc(M->scr.generation, sizeof(int16_t) * capacity);
  M->scr.particleID = realloc(M->scr.particleID, sizeof(int32_t) * capacity);
  M->scr_capacity = capacity;
}

/* this push's lost particles into the lost-particle table, row by row in
 * pages of at most 1000 rows, as advance_particles.c:450-487 and :529-535
 * write them */
/* The push's lost particles, in the order of advance_particles.c:437-491:
 * each one queued for secondary emission (the reference's own
 * queueSecondaryEmission, with the loss point, impact momentum and side the
 * device found) and written to the lost-particle file.  Runs after the beam
 * came back, since the queue takes particle IDs from beam->nextParticleID. */
static void handle_lost(Mirror *M, SDDS_DATASET *SDDSlost, FIELDS *EM_problem, BEAM *beam,
                        SECONDARY_EMISSION *secondaryEmission, long nSecondaryDefns)
{
  int64_t cap = M->capacity;
  double *v = malloc(sizeof(double) * 9 * (size_t)cap);
  int16_t *gen = malloc(sizeof(int16_t) * 2 * (size_t)cap);
  int32_t *id = malloc(sizeof(int32_t) * (size_t)cap);
  if (!v || !gen || !id)
    bomb("memory allocation failure (spiffe drop-in)", NULL);
  spiffe_lost_set h = {0, cap, v, v + cap, v + 2 * cap, v + 3 * cap, v + 4 * cap, v + 5 * cap, v + 6 * cap,
                       v + 7 * cap, gen, id, NULL, v + 8 * cap, gen + cap};
  check(spiffe_gpu_download_lost(M->inst, &h), "spiffe drop-in: lost particles");
  long newLost = 0, maxLost = 0;
  for (int64_t k = 0; k < h.nb; k++) {
    if (nSecondaryDefns)
      queueSecondaryEmission(secondaryEmission, nSecondaryDefns, h.p[k], h.zLost[k], h.rLost[k], h.direction[k],
                             h.q[k], h.generation[k], EM_problem, beam);
    if (!SDDSlost)
      continue;
    if (newLost && newLost >= maxLost) {
      if (!SDDS_WritePage(SDDSlost)) {
        SDDS_SetError("Problem writing lost particle data.");
        SDDS_PrintErrors(stderr, SDDS_EXIT_PrintErrors | SDDS_VERBOSE_PrintErrors);
      }
      newLost = maxLost = 0;
    }
    if (maxLost == 0 && !SDDS_StartPage(SDDSlost, maxLost = 1000)) {
      SDDS_SetError("Problem writing lost particle data.");
      SDDS_PrintErrors(stderr, SDDS_EXIT_PrintErrors | SDDS_VERBOSE_PrintErrors);
    }
    if (!SDDS_SetRowValues(SDDSlost, SDDS_SET_BY_NAME | SDDS_PASS_BY_VALUE, newLost, "t", EM_problem->time, "rLost",
                           (float)h.rLost[k], "zLost", (float)h.zLost[k], "pz", (float)h.pz[k], "pr",
                           (float)h.pr[k], "r0", (float)h.r0[k], "z0", (float)h.z0[k], "q", (float)h.q[k],
                           "generation", h.generation[k], "particleID", h.particleID[k], NULL)) {
      SDDS_SetError("Problem writing lost particle data.");
      SDDS_PrintErrors(stderr, SDDS_EXIT_PrintErrors | SDDS_VERBOSE_PrintErrors);
    }
    newLost++;
  }
  if (SDDSlost && newLost && !SDDS_WritePage(SDDSlost)) {
    SDDS_SetError("Problem writing lost particle data.");
    SDDS_PrintErrors(stderr, SDDS_EXIT_PrintErrors | SDDS_VERBOSE_PrintErrors);
  }
  free(v);
  free(gen);
  free(id);
}

/* the screen's SDDS page, as advance_particles.c:538-569 writes it */
static void write_screen_page(SCREEN *sc, FIELDS *EM_problem)
{
  long ib;
  if (!SDDS_StartTable(&sc->table, sc->nb))
    SDDS_PrintErrors(stderr, SDDS_EXIT_PrintErrors | SDDS_VERBOSE_PrintErrors);
  for (ib = 0; ib < N_SCREEN_QUANS; ib++)
    if (!SDDS_SetColumn(&sc->table, SDDS_SET_BY_INDEX, sc->buffer[ib], sc->nb, ib))
      SDDS_PrintErrors(stderr, SDDS_EXIT_PrintErrors | SDDS_VERBOSE_PrintErrors);
  if (!SDDS_SetColumn(&sc->table, SDDS_SET_BY_NAME, sc->generation, sc->nb, "generation") ||
      !SDDS_SetColumn(&sc->table, SDDS_SET_BY_NAME, sc->particleID, sc->nb, "particleID") ||
      !SDDS_SetColumn(&sc->table, SDDS_SET_BY_NAME, sc->rmin, sc->nb, "rMin") ||
      !SDDS_SetColumn(&sc->table, SDDS_SET_BY_NAME, sc->rmax, sc->nb, "rMax") ||
      !SDDS_SetColumn(&sc->table, SDDS_SET_BY_NAME, sc->zmin, sc->nb, "zMin") ||
      !SDDS_SetColumn(&sc->table, SDDS_SET_BY_NAME, sc->zmax, sc->nb, "zMax") ||
      !SDDS_SetParameters(&sc->table, SDDS_SET_BY_NAME | SDDS_PASS_BY_VALUE, "Time", EM_problem->time, "Timestep",
                          EM_problem->time_step, NULL))
    SDDS_PrintErrors(stderr, SDDS_EXIT_PrintErrors | SDDS_VERBOSE_PrintErrors);
  if (!SDDS_WriteTable(&sc->table)) {
    fprintf(stderr, "Problem writing to screen %s\n", sc->filename);
    SDDS_PrintErrors(stderr, SDDS_EXIT_PrintErrors | SDDS_VERBOSE_PrintErrors);
  }
}

void advance_particles(BEAM *beam, FIELDS *EM_problem, TEST_BEAM_DEFN *test_beam_defn, SCREEN *screen_defn,
                       long n_screens, SDDS_DATASET *SDDSlost, double zForcesStart,
                       SECONDARY_EMISSION *secondaryEmission, long nSecondaryDefns)
{
  if (!secondaryEmission)
    nSecondaryDefns = 0;
  if (EM_problem->onAxisFields > 0)
    bomb("on-axis fields are not available in the spiffe drop-in", NULL);
  if (n_screens > SPIFFE_MAX_SCREENS)
    bomb("too many screens for the spiffe drop-in", NULL);
  Mirror *M = mirror_of(EM_problem, beam->max_np);
  /* the screens, registered once (their definitions do not change) */
  int same = M->n_screens == n_screens;
  for (long is = 0; same && is < n_screens; is++)
    same = M->screen_z[is] == screen_defn[is].z_position && M->screen_dir[is] == screen_defn[is].direction;
  if (!same) {
    check(spiffe_gpu_clear_screens(M->inst), "spiffe drop-in: screens");
    if (M->n_screens) { /* the device keeps registrations: start again */
      mirror_free(M);
      M = mirror_of(EM_problem, beam->max_np);
    }
    for (long is = 0; is < n_screens; is++) {
      check(spiffe_gpu_add_screen(M->inst, screen_defn[is].z_position, (int32_t)screen_defn[is].direction,
                                  M->capacity),
            "spiffe drop-in: screen definition");
      M->screen_z[is] = screen_defn[is].z_position;
      M->screen_dir[is] = screen_defn[is].direction;
    }
    M->n_screens = (int)n_screens;
  }
  upload(M, EM_problem, GATHER, sizeof(GATHER) / sizeof(int));
  beam_upload(M, beam);
  spiffe_push_options o;
  memset(&o, 0, sizeof(o));
  o.z_forces_start = zForcesStart;
  if (test_beam_defn) {
    o.tb_electrons_per_macroparticle = test_beam_defn->electrons_per_macroparticle;
    o.tb_z_force = test_beam_defn->z_force;
    o.tb_r_force = test_beam_defn->r_force;
    o.tb_z_start_deceleration = test_beam_defn->z_start_deceleration;
    o.tb_r_start_deceleration = test_beam_defn->r_start_deceleration;
  }
  o.compaction = SPIFFE_COMPACT_REFERENCE;
  o.screen_momentum = SPIFFE_SCREEN_REFERENCE;
  if ((SDDSlost || nSecondaryDefns) && !M->lost_on) {
    check(spiffe_gpu_set_lost_log(M->inst, M->capacity), "spiffe drop-in: lost-particle log");
    M->lost_on = 1;
  }
  check(spiffe_gpu_advance_particles(M->inst, &o), "advance_particles");
  beam_download(M, beam);
  if (M->lost_on)
    handle_lost(M, SDDSlost, EM_problem, beam, secondaryEmission, nSecondaryDefns);
  /* this push's screen records into the reference's buffers, then its page */
  for (long is = 0; is < n_screens; is++) {
    SCREEN *sc = screen_defn + is;
    int64_t nb = 0;
    check(spiffe_gpu_screen_count(M->inst, (int32_t)is, &nb), "spiffe drop-in: screen count");
    sc->nb = 0;
    sc->max_nb = beam->max_np;
    if (!nb)
      continue;
    screen_buffers(M, nb);
    M->scr.capacity = M->scr_capacity;
    check(spiffe_gpu_download_screen(M->inst, (int32_t)is, &M->scr), "spiffe drop-in: screen records");
    if (!sc->buffer && !(sc->buffer = calloc(N_SCREEN_QUANS, sizeof(*sc->buffer))))
      bomb("memory allocation failure (spiffe drop-in)", NULL);
    for (int q = 0; q < N_SCREEN_QUANS; q++)
      sc->buffer[q] = realloc(sc->buffer[q], sizeof(double) * nb);
    sc->generation = realloc(sc->generation, sizeof(short) * nb);
    sc->particleID = realloc(sc->particleID, sizeof(int32_t) * nb);
    sc->rmin = realloc(sc->rmin, sizeof(double) * nb);
    sc->rmax = realloc(sc->rmax, sizeof(double) * nb);
    sc->zmin = realloc(sc->zmin, sizeof(double) * nb);
    sc->zmax = realloc(sc->zmax, sizeof(double) * nb);
    for (int q = 0; q < N_SCREEN_QUANS; q++)
      memcpy(sc->buffer[q], M->scr.col[q], sizeof(double) * nb);
    for (int64_t i = 0; i < nb; i++) {
      sc->generation[i] = M->scr.generation[i];
      sc->particleID[i] = M->scr.particleID[i];
    }
    memcpy(sc->rmin, M->scr.rmin, sizeof(double) * nb);
    memcpy(sc->rmax, M->scr.rmax, sizeof(double) * nb);
    memcpy(sc->zmin, M->scr.zmin, sizeof(double) * nb);
    memcpy(sc->zmax, M->scr.zmax, sizeof(double) * nb);
    sc->nb = (long)nb;
    write_screen_page(sc, EM_problem);
  }
  if (n_screens)
    check(spiffe_gpu_clear_screens(M->inst), "spiffe drop-in: screens");
}

/* --------------------------------------------------------------- poisson.c */

long solve_poisson_cyl(double **Psi, double **driving_term, short **flags, long left_bc, long right_bc, long nz,
                       long nr, double dz, double dr, double accuracy, long iteration_limit)
{
  if (accuracy <= 0)
    bomb("accuracy is <= 0 in solve_poisson_cyl", NULL);
  if (iteration_limit <= 1)
    bomb("iteration_limit is <= 1 in solve_poisson_cyl", NULL);
  if (!solver.inst || solver_flags != flags || solver.nz != nz || solver.nr != nr) {
    mirror_free(&solver);
    FIELDS F;
    memset(&F, 0, sizeof(F));
    F.nz = (int32_t)nz;
    F.nr = (int32_t)nr;
    F.dz = dz;
    F.dr = dr;
    F.rmax = dr * (nr - 1);
    F.zmax = dz * (nz - 1);
    F.left_bc = left_bc;
    F.right_bc = right_bc;
    F.modes = FL_TM_FIELDS;
    mirror_create(&solver, &F, flags, 0);
    solver_flags = flags;
  }
  spiffe_mesh m;
  check(spiffe_gpu_get_mesh(solver.inst, &m), "solve_poisson_cyl");
  m.dz = dz;
  m.dr = dr;
  m.left_bc = (int32_t)left_bc;
  m.right_bc = (int32_t)right_bc;
  check(spiffe_gpu_set_mesh(solver.inst, &m), "solve_poisson_cyl");
  spiffe_field_set s;
  memset(&s, 0, sizeof(s));
  s.Psi = stage_of(&solver, A_PSI);
  gather_rows(Psi, s.Psi, (int32_t)nz, (int32_t)nr);
  s.Q = stage_of(&solver, A_Q);
  if (driving_term)
    gather_rows(driving_term, s.Q, (int32_t)nz, (int32_t)nr);
  else
    memset(s.Q, 0, sizeof(double) * solver.nodes);
  check(spiffe_gpu_upload_fields(solver.inst, &s), "solve_poisson_cyl");
  int64_t it = 0;
  check(spiffe_gpu_solve_poisson_cyl(solver.inst, 0, accuracy, iteration_limit, &it), "solve_poisson_cyl");
  memset(&s, 0, sizeof(s));
  s.Psi = solver.stage[A_PSI];
  check(spiffe_gpu_download_fields(solver.inst, &s), "solve_poisson_cyl");
  scatter_rows(s.Psi, Psi, (int32_t)nz, (int32_t)nr);
  if (it < 0)
    printf("warning: maximum number of iterations exceeded in solve_poisson_cyl\n");
  return (long)it;
}

/* ---------------------------------------------------- poisson_correction.c */

static long guess_code;
static const char *guess_name[4] = {"none", "line-charge", "point-charge", "zero"};

void setup_poisson_correction(FIELDS *EM_problem, NAMELIST_TEXT *nl_text)
{
  /* the defaults and checks of poisson_correction.c:31-71 */
  start_time = 0;
  step_interval = 0;
  accuracy = 1e-6;
  maximum_iterations = 1000;
  verbosity = 0;
  test_charge = z_test_charge = r_test_charge = 0;
  error_charge_threshold = 0;
  guess_type = "none";
  process_namelist(&poisson_correction, nl_text);
  print_namelist(stdout, &poisson_correction);
  if (start_time < 0)
    bomb("start_time < 0 for poisson_correction", NULL);
  if (step_interval < 0)
    bomb("step_interval < 0 for poisson_correction", NULL);
  if (accuracy <= 0)
    bomb("accuracy <= 0 for poisson_correction", NULL);
  if (maximum_iterations <= 0)
    bomb("maximum iterations <= 0 for poisson_correction", NULL);
  if (verbosity < 0)
    bomb("verbosity < 0 for poisson_correction", NULL);
  if (test_charge)
    bomb("test_charge is not available in the spiffe drop-in", NULL);
  if ((guess_code = match_string(guess_type, (char **)guess_name, 4, 0)) < 0)
    bomb("unknown guess type for poisson_correction", NULL);
  if (!(EM_problem->modes & FL_TM_FIELDS))
    bomb("TM fields must be enabled in order to do poisson correction", NULL);
}

static spiffe_poisson_options options(void)
{
  spiffe_poisson_options o;
  memset(&o, 0, sizeof(o));
  o.start_time = start_time;
  o.step_interval = step_interval;
  o.accuracy = accuracy;
  o.error_charge_threshold = error_charge_threshold;
  o.maximum_iterations = maximum_iterations;
  o.verbosity = (int32_t)verbosity;
  o.guess_code = (int32_t)guess_code;
  return o;
}

static const int PC_IN[] = {A_EZ, A_ER, A_PSI, A_Q};
static const int PC_OUT[] = {A_EZ, A_ER, A_PSI, A_Q};

void add_poisson_correction(FIELDS *EM_problem, BEAM *beam, long space_charge)
{
  if (maximum_iterations <= 0)
    return;
  if (EM_problem->dti <= 0)
    bomb("integration step size is not defined (add_poisson_correction)", NULL);
  if (step_interval <= 0 || EM_problem->time_step % step_interval != 0)
    return; /* the device applies the start-step test as well (poisson_correction.c:113-117) */
  if (!EM_problem->Psi)
    bomb("Psi array is unexpectedly null in add_poisson_correction", NULL);
  if (!EM_problem->Q)
    bomb("Q array is unexpectedly null in add_poisson_correction", NULL);
  Mirror *M = mirror_of(EM_problem, beam->max_np);
  upload(M, EM_problem, PC_IN, 4);
  beam_upload(M, beam);
  spiffe_poisson_options o = options();
  spiffe_poisson_report rep;
  check(spiffe_gpu_add_poisson_correction(M->inst, (int32_t)space_charge, &o, &rep), "add_poisson_correction");
  if (rep.ran)
    download(M, EM_problem, PC_OUT, 4);
  if (verbosity && rep.ran) {
    printf("    \"real\" charge: %23.16e C    error charge: %23.16e C    surface charge: %23.16e\n", rep.Qreal,
           rep.Qerror, rep.Qsurface);
    printf("    Poisson solution took %ld iterations\n", (long)rep.iterations);
    printf("    Poisson correction completed\n");
    fflush(stdout);
  }
}

static const int IMP[] = {A_EZI, A_ERI, A_PSII};

void compute_imposed_Efield(FIELDS *EM_problem, long initialize)
{
  if (maximum_iterations <= 0)
    return;
  if (EM_problem->dti <= 0)
    bomb("integration step size is not defined (compute_imposed_Efield)", NULL);
  if (!EM_problem->PsiImposed)
    bomb("PsiImposed array is unexpectedly null in compute_imposed_Efield", NULL);
  if (!EM_problem->EzImposed)
    bomb("EzImposed array is unexpectedly null in compute_imposed_Efield", NULL);
  if (!EM_problem->ErImposed)
    bomb("ErImposed array is unexpectedly null in compute_imposed_Efield", NULL);
  Mirror *M = mirror_of(EM_problem, 0);
  upload(M, EM_problem, IMP, 3);
  spiffe_poisson_options o = options();
  check(spiffe_gpu_compute_imposed_efield(M->inst, &o, (int32_t)initialize), "compute_imposed_Efield");
  download(M, EM_problem, IMP, 3);
}

/* ------------------------------------------------- explicit device control */

/* Creates (or refreshes) the device mirror of a problem and its beam and
 * copies their host state in.  Returns 0. */
int spiffe_gpu_attach(FIELDS *EM_problem, BEAM *beam)
{
  static const int ALL[] = {A_EZ, A_ER, A_BPHI, A_BPHI2, A_JZ, A_JR, A_EPHI, A_JPHI, A_BR, A_BR2, A_BZ, A_BZ2,
                            A_EZI, A_ERI, A_PSII, A_BZI, A_BRI, A_PSI, A_Q};
  Mirror *M = mirror_of(EM_problem, beam ? beam->max_np : 0);
  upload(M, EM_problem, ALL, A_N);
  if (beam)
    beam_upload(M, beam);
  return 0;
}

/* Copies the device state of an attached problem back to its host arrays:
 * `what` bit 1 the fields, bit 2 the beam. */
int spiffe_gpu_sync_to_host(FIELDS *EM_problem, BEAM *beam, unsigned what)
{
  static const int ALL[] = {A_EZ, A_ER, A_BPHI, A_BPHI2, A_JZ, A_JR, A_EPHI, A_JPHI, A_BR, A_BR2, A_BZ, A_BZ2,
                            A_EZI, A_ERI, A_PSII, A_BZI, A_BRI, A_PSI, A_Q};
  for (int i = 0; i < n_mirrors; i++)
    if (mirrors[i].F == EM_problem && mirrors[i].inst) {
      if (what & 1u)
        download(mirrors + i, EM_problem, ALL, A_N);
      if ((what & 2u) && beam)
        beam_download(mirrors + i, beam);
      return 0;
    }
  return SPIFFE_ERR_INVALID;
}

/* The device instance of an attached problem (for spiffe_gpu_run_steps and
 * the other instance entry points), or NULL. */
spiffe_gpu_instance *spiffe_gpu_attached_instance(FIELDS *EM_problem)
{
  for (int i = 0; i < n_mirrors; i++)
    if (mirrors[i].F == EM_problem)
      return mirrors[i].inst;
  return NULL;
}

int spiffe_gpu_detach(FIELDS *EM_problem)
{
  for (int i = 0; i < n_mirrors; i++)
    if (mirrors[i].F == EM_problem) {
      mirror_free(mirrors + i);
      mirrors[i] = mirrors[--n_mirrors];
      memset(mirrors + n_mirrors, 0, sizeof(Mirror));
      return 0;
    }
  return SPIFFE_ERR_INVALID;
}
