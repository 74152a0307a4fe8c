// spiffe_b200/csrc/modules.cuh -- host-side interface between the kernel
// modules (fdtd_f64, particles_f64, poisson_f64, emit) and the runtime: the
// work-buffer structs each module owns and the launch wrappers it exports.
#pragma once

#include "common.cuh"

struct Fdtd64Tables {
  double *cpz = nullptr, *cmz = nullptr, *bzf = nullptr;
  int *cut0 = nullptr, *cut1 = nullptr;
  double fEr = 0, topf = 0, fEphi = 0;
};
extern "C" int spiffe_fdtd64_tables(const DevMesh *m, const int16_t *host_flags, Fdtd64Tables *t, cudaStream_t s);
extern "C" void spiffe_fdtd64_tables_free(Fdtd64Tables *t);
extern "C" int spiffe_fdtd64_step(const DevMesh *m, const DevFields<double> *f, const Fdtd64Tables *t, cudaStream_t s);

struct Particles64Work {
  uint8_t *lost = nullptr;
  int *surv = nullptr, *surv_before = nullptr, *map = nullptr;
  int *keys = nullptr, *keys_alt = nullptr;
  double *vals = nullptr, *vals_alt = nullptr;
  void *cub_tmp = nullptr;
  size_t cub_bytes = 0;
  long long capacity = 0;
};
extern "C" int spiffe_particles64_work(Particles64Work *w, long long capacity, bool ordered);
extern "C" void spiffe_particles64_work_free(Particles64Work *w);
extern "C" int spiffe_deposit64(const DevMesh *m, const DevFields<double> *f, const DevBeam64 *b, const DevCounts *cnt,
                                long long np_bound, bool ordered, Particles64Work *w, cudaStream_t s);
struct PushHostParams {
  double time, z_forces_start, QoMC, stiffness;
  double tb_epm, tb_z_force, tb_r_force, tb_z_decel, tb_r_decel;
  int screen_momentum, compaction;
  LostLog lost;
};
extern "C" int spiffe_gather_points64(const DevMesh *m, const DevFields<double> *f, const double *zr, int n, int ncomp,
                                      double *E, cudaStream_t s);
extern "C" int spiffe_push64(const DevMesh *m, const DevFields<double> *f, const DevBeam64 *b, const PushHostParams *hp,
                             const DevScreens *scr, DevCounts *cnt, long long np_bound, Particles64Work *w,
                             cudaStream_t s);

// device-side state of one Poisson correction
struct PcState {
  double Qreal, Qerror, Qsurface, centroid, driving, residual;
  long long iterations;
  int do_solve, pad;
};
struct Poisson64Work {
  double *Az = nullptr, *Ari = nullptr, *Aro = nullptr, *volume = nullptr;
  double *part = nullptr;
  double *scalars = nullptr;
  double *omega = nullptr;
  long long omega_n = 0;
  unsigned *bar = nullptr;
  PcState *st = nullptr;
  long long *iters = nullptr;
  int sor_grid = 0;
  size_t part_n = 0;
  double *crow = nullptr, *drow = nullptr;
};
struct PoissonHostOptions {
  double accuracy, error_charge_threshold;
  long long maximum_iterations;
  int guess_code, space_charge;
};
extern "C" int spiffe_poisson64_setup(const DevMesh *m, Poisson64Work *w, long long np_capacity, cudaStream_t s);
extern "C" void spiffe_poisson64_free(Poisson64Work *w);
extern "C" int spiffe_sor64(const DevMesh *m, Poisson64Work *w, double *Psi, const double *rhs, const int16_t *flags,
                            double accuracy, long long limit, DevCounts *cnt, long long *iterations, cudaStream_t s);
// ordered: the particles' charge leaves Q through the ordered reduction on
// pw's key/value buffers (sized by spiffe_particles64_work with ordered set)
// instead of FP64 atomics.
extern "C" int spiffe_poisson_correction64(const DevMesh *m, const DevFields<double> *f, const DevBeam64 *b,
                                           DevCounts *cnt, long long np_bound, const PoissonHostOptions *o,
                                           Poisson64Work *w, Particles64Work *pw, bool ordered, cudaStream_t s);
// Applies n (node, value) entries held in w->keys / w->vals to dst: a stable
// sort by node, then each node's values added in entry order starting from
// dst's current value.  INT_MAX keys are skipped.
extern "C" int spiffe_ordered_add64(Particles64Work *w, long long n, double *dst, cudaStream_t s);
extern "C" int spiffe_poisson64_report(Poisson64Work *w, spiffe_poisson_report *rep, cudaStream_t s);
extern "C" int spiffe_imposed_field64(const DevMesh *m, const DevFields<double> *f, double factor, cudaStream_t s);

struct BirthBin {
  long long start, count;
  double area, rmin;
};
// mode 0: uniform in r^2 from the generator; 1: per-bin counts (distribution
// correction); 2: discrete radii; 3: test-beam particle (emit_test_particles,
// test_beam.c:57-104) at (z_position, inner_radius) with momenta pz0, pr0,
// rpphi0, inactive until the push activates it.
#define SPIFFE_BIRTH_TEST 3
#define SPIFFE_BIRTH_LIST 4 // explicit particles (secondary electrons): list holds BIRTH_LIST_COLS rows of total
#define BIRTH_LIST_COLS 10  // z, r, pz, pr, vz, vr, Q, t0, generation, particleID
struct BirthParams {
  long long total;
  uint64_t key, counter_base;
  int mode;
  int spread;
  double z_position, inner_radius, outer_radius, inner_r2, dr2;
  double initial_vz, initial_omega, Q, time, dt, QoMC, stiffness;
  double pz0, pr0, rpphi0;
  const BirthBin *bins;
  int n_bins;
  const double *list; // SPIFFE_BIRTH_LIST
};
extern "C" int spiffe_births64(const DevMesh *m, const DevFields<double> *f, const DevBeam64 *b, const BirthParams *p,
                               DevCounts *cnt, cudaStream_t s);
extern "C" int spiffe_antenna64(double *J, int pitch, int direction, long istart, long iend, long iposition,
                                double value, cudaStream_t s);

// translate_problem (translate.c:51-57, :123-196): *flag = 1 when a particle
// ip < np lies past `trigger`; rows 0..nz of an array move down one row
// (`scratch` holds nz rows), the last row zeroed
extern "C" int spiffe_beyond64(const double *z, const DevCounts *cnt, long long np_bound, double trigger, int *flag,
                               cudaStream_t s);
extern "C" int spiffe_rows_down(void *a, size_t row, int nz, void *scratch, cudaStream_t s);

