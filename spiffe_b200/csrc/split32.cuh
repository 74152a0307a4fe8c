// spiffe_b200/csrc/split32.cuh -- data model of the split-precision form.
//
// The same spiffe problem as the FP64 form (common.cuh), stored for speed:
//
//  * fields E, B in FP32 on rows padded to a multiple of 32 elements, plus a
//    one-byte update mask per node that folds the reference's per-node flag
//    tests and its FL_LAST_ACTIVE_PT row cut-off (integrate.c:345-346) into
//    bits, so the stencil reads 1 byte of metadata per node instead of 2;
//  * currents Jz, Jr, Jphi as 64-bit fixed point: a particle's contribution
//    is rounded to an integer number of quanta and added with integer
//    atomics, so the sum is exact and independent of the order of addition
//    (bit-reproducible run to run);
//  * Psi, PsiImposed and the Poisson charge Q in FP64, since the Poisson
//    correction forms its residual in FP64 and only the SOR correction
//    sweeps run in FP32;
//  * particles as an integer cell (iz in the high 16 bits, ir in the low
//    16) plus FP32 offsets in [0,1) within the cell, FP32 momenta and
//    charge, a status byte, FP32 path extrema, and the cold per-particle
//    data (birth position and time, id, generation) apart.  Velocities are
//    not stored: the reference derives them from the momenta at the end of
//    every push (setParticleVelocities, advance_particles.c:605-620), so a
//    push recomputes them from the stored momenta instead of reading them.
#pragma once

#include "common.cuh"

// update-mask bits (one byte per node)
#define S32_U_EZ 1u    // Ez interior update (iz <= cut1[ir], no FL_EZ_ZERO)
#define S32_U_ER 2u    // Er interior update (iz <= cut0[ir], no FL_ER_ZERO)
#define S32_U_BPHI 4u  // Bphi interior update (iz <= cut1[ir], no FL_BPHI_ZERO)
#define S32_U_EPHI 8u  // Ephi interior update (iz <= cut0[ir], no FL_EPHI_ZERO)
#define S32_U_BR 16u   // Br interior update (iz <= cut1[ir], no FL_BR_ZERO)
#define S32_U_BZ 32u   // Bz interior update (iz <= cut0[ir], no FL_BZ_ZERO)
#define S32_U_METAL 64u // FL_IS_METAL
#define S32_U_CLEAN 128u // no flag set on rows iz-1..iz+1 x columns ir..ir+1: the gather's metal
                         // fix-ups (advance_particles.c:672-690, :730-735) cannot apply in cell (iz, ir)

// particle status byte
#define S32_ACTIVE 1u
#define S32_LOST 2u

struct DevFields32 {
  const int16_t *flags; // reference flags, pitch P
  const uint8_t *umask; // update mask, pitch P
  float *Ez, *Er, *Bphi, *Bphi2;
  float *Ephi, *Br, *Br2, *Bz, *Bz2;
  float *EzImposed, *ErImposed, *BzImposed, *BrImposed;
  long long *Jz, *Jr, *Jphi; // fixed point, quantum S32Scales::qJ
  double *Psi, *PsiImposed, *Q;
  long long *Qp; // particle charge per node (fixed point, quantum qQ) of the last correction
  // The rows that may hold nonzero current: [0] lowest, [1] highest (empty
  // when [0] > [1]).  Every deposit widens it; the FDTD step that zeroes J
  // reads and clears only those rows, then empties it.
  int *jbox;
};

// Fixed-point scales.  q_ref bounds |Q| of every macroparticle; a current
// contribution is at most 4 |Q| c / (pi dz dr^2) (the on-axis factor 4 of
// space_charge.c:110-112), which maps to 2^40 quanta, so one node holds
// the sum of 2^23 maximal contributions without overflow.
struct S32Scales {
  float s_charge;  // 2^38 / q_ref: per-particle charge in current units (x v/c x weights)
  double qJ;       // A/m^2 per quantum of J
  float kJ;        // -dt qJ / eps0: Ez/Er/Ephi increment per quantum
  float sq_charge; // 2^38 / q_ref for the charge removal
  double qQ;       // C per quantum of Qp
};

// Split-precision beam.  cell = (iz << 16) | (ir & 0xffff) with iz signed.
struct DevBeam32 {
  int32_t *cell;
  float *fz, *fr;
  float *pz, *pr, *rpphi;
  float *Q;
  uint8_t *status;
  float *zmin, *zmax, *rmin, *rmax;
  double *r0, *z0, *t0;
  int32_t *particleID;
  int16_t *generation;
  int64_t capacity;
};

__host__ __device__ inline int s32_iz(int32_t c) { return c >> 16; }
__host__ __device__ inline int s32_ir(int32_t c) { return (int)(int16_t)(c & 0xffff); }
__host__ __device__ inline int32_t s32_cell(int iz, int ir) { return (int32_t)(((uint32_t)iz << 16) | ((uint32_t)ir & 0xffffu)); }

// host-side per-row metric tables and the mask builder live in fdtd_f32.cu
struct Fdtd32Tables {
  float *cpd = nullptr, *cmd = nullptr; // dt * Ez metric coefficients per ir (integrate.c:327-340)
  float *bzf = nullptr;                 // Bz factor per ir (integrate.c:515)
  float fEr = 0, topf = 0, fEphi = 0;   // dt/(mu0 eps0 dz), (rmax-dr/2)/(rmax+dr/2), dt/(eps0 mu0)
  // the fused TM kernel (fdtd_f32.cu k_tm_fused32): bands of rows, the Er
  // row each band publishes to the next, the bands' epoch flags
  int fused = -1;                       // -1 not yet decided, 0 two kernels, 1 fused
  int mode = 0;                         // SPIFFE_FDTD_*
  int bands = 0, rows_per = 0, threads = 0;
  size_t smem = 0;
  float *pub = nullptr;
  unsigned *flag = nullptr, *arrivals = nullptr;
  unsigned epoch = 0;
};
extern "C" int s32_fdtd_tables(const DevMesh *m, const int16_t *host_flags, Fdtd32Tables *t, uint8_t *d_umask,
                               cudaStream_t s);
extern "C" void s32_fdtd_tables_free(Fdtd32Tables *t);
extern "C" int s32_fdtd_step(const DevMesh *m, const DevFields32 *f, Fdtd32Tables *t, float kJ, int zero_j,
                             unsigned *err, cudaStream_t s);
// jbox = [lo, hi] (rows; lo > hi: empty)
extern "C" int s32_jbox_set(int *jbox, int lo, int hi, cudaStream_t s);
// FP64 host array (pitch nr+1) <-> FP32 device array (pitch P) through a device staging buffer
extern "C" int s32_to_f32(const DevMesh *m, const double *d_staging, float *dst, cudaStream_t s);
extern "C" int s32_from_f32(const DevMesh *m, const float *src, double *d_staging, cudaStream_t s);
extern "C" int s32_to_f64p(const DevMesh *m, const double *d_staging, double *dst, cudaStream_t s);
extern "C" int s32_from_f64p(const DevMesh *m, const double *src, double *d_staging, cudaStream_t s);
extern "C" int s32_to_fixed(const DevMesh *m, const double *d_staging, long long *dst, double quantum, cudaStream_t s);
extern "C" int s32_from_fixed(const DevMesh *m, const long long *src, double *d_staging, double quantum, cudaStream_t s);
extern "C" int s32_rescale_fixed(long long *a, size_t n, int shift, cudaStream_t s);
extern "C" int s32_antenna(long long *J, int *jbox, int pitch, int direction, long istart, long iend, long iposition,
                           double value, double qJ, cudaStream_t s);
// the moving window's trigger test and the particles' (and deposited
// current rows') move down one row (translate.cu)
extern "C" int s32_beyond(const int32_t *cell, const float *fz, const DevCounts *cnt, long long np_bound, double zmin,
                          double dz, double trigger, int *flag, cudaStream_t s);
extern "C" int s32_cells_down(int32_t *cell, int *jbox, const DevCounts *cnt, long long np_bound, cudaStream_t s);

// particles (particles_f32.cu)
struct Particles32Work {
  int32_t *lost_list = nullptr; // indices lost this step (any order)
  int32_t *keys = nullptr, *keys_alt = nullptr, *idx = nullptr, *idx_alt = nullptr;
  void *cub_tmp = nullptr;
  size_t cub_bytes = 0;
  DevBeam32 alt{}; // second beam buffer for the cell sort
  long long capacity = 0;
};
struct Push32Params {
  double time;
  float dt, dt_dz, dt_dr, QoMC_dt, stiff_inv; // dt, dt/dz, dt/dr, QoMC dt, 1/stiffness
  double z_forces_start;
  int zfs_on; // z_forces_start lies inside (zmin, zmax)
  int forced;
  float tb_z_force_dt, tb_r_force_dt;
  double tb_z_decel, tb_r_decel;
  int screen_momentum;
  int deposit; // fused deposition of the pushed particles for the next step
  LostLog lost;
};
extern "C" int s32_particles_work(Particles32Work *w, long long capacity);
extern "C" void s32_particles_work_free(Particles32Work *w);
extern "C" int s32_beam_alloc(DevBeam32 *b, long long capacity);
extern "C" void s32_beam_free(DevBeam32 *b);
extern "C" int s32_beam_copy(DevBeam32 *dst, const DevBeam32 *src, long long n, cudaStream_t s);
extern "C" int s32_deposit(const DevMesh *m, const DevFields32 *f, const DevBeam32 *b, const DevCounts *cnt,
                           long long np_bound, const S32Scales *sc, cudaStream_t s);
extern "C" int s32_push(const DevMesh *m, const DevFields32 *f, const DevBeam32 *b, const Push32Params *p,
                        const DevScreens *scr, DevCounts *cnt, long long np_bound, int compaction,
                        const S32Scales *sc, Particles32Work *w, cudaStream_t s);
extern "C" int s32_gather_points(const DevMesh *m, const DevFields32 *f, const double *zr, int n, int ncomp, double *E,
                                 cudaStream_t s);
extern "C" int s32_sort(const DevMesh *m, DevBeam32 *b, DevCounts *cnt, long long np_bound, Particles32Work *w,
                        cudaStream_t s);
// FP64 SoA (device staging, one array at a time) <-> split beam
extern "C" int s32_beam_pack_pos(const DevMesh *m, const double *z, const double *r, DevBeam32 *b, long long n,
                                 DevCounts *cnt, cudaStream_t s);
extern "C" int s32_beam_unpack_pos(const DevMesh *m, const DevBeam32 *b, double *z, double *r, long long n,
                                   cudaStream_t s);
extern "C" int s32_beam_unpack_vel(const DevMesh *m, const DevBeam32 *b, double *vz, double *vr, double *vphi,
                                   long long n, cudaStream_t s);
extern "C" int s32_d2f(const double *src, float *dst, long long n, cudaStream_t s);
extern "C" int s32_f2d(const float *src, double *dst, long long n, cudaStream_t s);
extern "C" int s32_status_pack(const uint64_t *src, uint8_t *dst, long long n, cudaStream_t s);
extern "C" int s32_status_unpack(const uint8_t *src, uint64_t *dst, long long n, cudaStream_t s);
// births (emit.cu's BirthParams), with their current when `deposit`
struct BirthParams;
extern "C" int s32_births(const DevMesh *m, const DevFields32 *f, const DevBeam32 *b, const BirthParams *p,
                          DevCounts *cnt, const S32Scales *sc, int deposit, cudaStream_t s);

// Multigrid solve (multigrid_f32.cu): level 0 is the mesh itself (the
// five-point operator of poisson.c:57-117 in FP32 on the correction u0 with
// right-hand side f0); each coarser level holds nodes 2I, 2J of the level
// above, with the Galerkin operator R A P of that level (nine points) built
// on the host.
#define MG_MAX_LEVELS 14
#define MG_NCOEF 10 // 8 off-diagonal coefficients divided by the diagonal, 1/diagonal, diagonal
struct MgLevel {
  int Z = 0, R = 0, P = 0; // nodes in z and r; row pitch with one halo node a side
  float *u = nullptr, *f = nullptr; // (Z+2) x P, node (I, J) at (I+1) P + J + 1; halo nodes stay 0
  const float *coef = nullptr;      // MG_NCOEF arrays of (Z+2) x P; 1/diagonal 0 marks a held node
  const float *rw = nullptr;        // restriction weights from the level above: [J][3], columns cr J - 1, cr J, cr J + 1
  int cz = 2, cr = 2;               // coarsening from the level above in z and r: node (I, J) is its (cz I, cr J)
};
struct Mg32Work {
  int nlev = 0, tail = 0; // levels; first level that CTA 0 works alone
  MgLevel lev[MG_MAX_LEVELS];
  float *u0 = nullptr, *f0 = nullptr; // level 0 at the mesh pitch
  void *mem = nullptr;                // every level array, one allocation
  double *part = nullptr;             // per-CTA partial sums [grid][2]
  unsigned long long *bar = nullptr;  // [0] barrier arrivals, [16] abort
  long long *iters = nullptr;
  int grid = 0, threads = 0;
  size_t bytes = 0;
  float *cinv = nullptr; // the coarsest level's inverse (exact coarse solve), cn x cn
  int *cidx = nullptr;   // its unknowns' array indices
  int cn = 0;
};
extern "C" int s32_mg_setup(const DevMesh *m, const int16_t *host_flags, Mg32Work *w, cudaStream_t s);
extern "C" void s32_mg_free(Mg32Work *w);
struct PcState;
extern "C" int s32_mg_solve(const DevMesh *m, Mg32Work *w, const float *crow, const float *drow, double *Psi,
                            const double *rhs, const uint8_t *umask, double accuracy, long long max_cycles,
                            PcState *st, long long *iters_out, DevCounts *cnt, cudaStream_t s);

// Poisson correction (poisson_f32.cu)
struct PcState;
struct Poisson32Work {
  double *Az = nullptr, *Ari = nullptr, *Aro = nullptr, *volume = nullptr;
  double *part = nullptr;
  size_t part_n = 0;
  double *scalars = nullptr; // [0] Qsurface [1] centroid [2] Qreal [3] Qerror [4] driving
  long long *qreal_fixed = nullptr;
  PcState *st = nullptr;
  long long *iters = nullptr;
  // SOR: Chebyshev factors, row coefficients, exchange rows, barrier words
  float *omega = nullptr;
  long long omega_n = 0;
  float *crow = nullptr, *drow = nullptr;
  float *xbuf = nullptr;
  unsigned long long *bar = nullptr; // [0] barrier counter, [16..39] fixed-point sum slots
  double *dpart = nullptr;           // per-CTA driving partials
  int grid = 0, threads = 0, depth = 2; // depth: halo rows a side = half-sweeps per barrier
  size_t smem = 0;
  int rows_per = 0, half = 0; // rows of the widest CTA band; half-row length (nodes of one colour)
  // solver of the Poisson correction: SPIFFE_POISSON_MULTIGRID (mg) or SPIFFE_POISSON_SOR
  int solver = 1;
  Mg32Work mg;
};

struct PoissonHostOptions;
extern "C" int s32_poisson_setup(const DevMesh *m, Poisson32Work *w, long long np_capacity, cudaStream_t s);
extern "C" void s32_poisson_free(Poisson32Work *w);
extern "C" int s32_sor(const DevMesh *m, Poisson32Work *w, double *Psi, const double *rhs, const uint8_t *umask,
                       double accuracy, long long limit, PcState *st, DevCounts *cnt, cudaStream_t s);
// the instance's solver (multigrid where it was set up, else SOR); the
// count of half-sweeps or V-cycles, -1 at the limit, lands in w->iters
extern "C" int s32_solve(const DevMesh *m, Poisson32Work *w, double *Psi, const double *rhs, const uint8_t *umask,
                         double accuracy, long long limit, PcState *st, DevCounts *cnt, cudaStream_t s);
extern "C" int s32_poisson_correction(const DevMesh *m, const DevFields32 *f, const DevBeam32 *b, DevCounts *cnt,
                                      long long np_bound, const PoissonHostOptions *o, const S32Scales *sc,
                                      Poisson32Work *w, cudaStream_t s);
extern "C" int s32_poisson_report(Poisson32Work *w, spiffe_poisson_report *rep, cudaStream_t s);
extern "C" int s32_imposed_field(const DevMesh *m, const DevFields32 *f, double factor, cudaStream_t s);
