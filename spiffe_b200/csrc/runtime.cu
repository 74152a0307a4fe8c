// spiffe_b200/csrc/runtime.cu -- host runtime behind the C ABI (spiffe_b200.h).
//
// Owns the device mirror of one spiffe problem and drives the kernels in the
// order perform_integration uses (integrate.c:134-194).  The host keeps only
// what the reference keeps on the host between steps and what is cheap to
// decide there: time, the emission counts of each cathode with the shared
// counter-based generator (cathode.c:349-422), the antenna current
// (antenna.c:374-418) and the Poisson interval test (poisson_correction.c:
// 116-119).  Particle counts live on the device; the host tracks an upper
// bound for launch sizes and reads the true count only when it must.
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <algorithm>
#include <type_traits>
#include <vector>

#include "common.cuh"

#include "../../include/spiffe_b200.h"
#include "../../include/spiffe_b200_rng.h"

#include "modules.cuh"
#include "onaxis.hpp"
#include "split32.cuh"

// ---------------------------------------------------------------- errors
static thread_local std::string g_error;

static int fail(int code, const char *fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_error = buf;
  return code;
}

// lets the host-only modules (geometry, commands) report through the same channel
extern "C" int spiffe_set_error(int code, const char *msg)
{
  g_error = msg ? msg : "";
  return code;
}

// process-wide count of kernels queued by this library
static std::atomic<long long> g_launches{0};
extern "C" void spiffe_note_launches(int n) { g_launches += n; }
extern "C" int64_t spiffe_gpu_launch_count(void) { return g_launches.load(); }

// Phases of one step, timed with CUDA events on the instance's stream.
enum Phase { PH_EMIT, PH_DEPOSIT, PH_POISSON, PH_FDTD, PH_PUSH, PH_COUNT };

struct PhaseTimer {
  bool on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool[PH_COUNT];
  size_t used[PH_COUNT] = {};
  cudaEvent_t take_start(int ph)
  {
    if (used[ph] == pool[ph].size()) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      pool[ph].push_back({a, b});
    }
    return pool[ph][used[ph]].first;
  }
  void release()
  {
    for (auto &v : pool)
      for (auto &e : v) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
      }
  }
};

#define CUDA_TRY(x)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess)                                                                   \
      return fail(SPIFFE_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_));            \
  } while (0)

// Kernel-module helpers return a CUDA error code (> 0) or 0; runtime helpers
// return 0 or a SPIFFE_ERR_* code with the message already set.
#define RC_TRY(x)                                                                            \
  do {                                                                                       \
    const int rc_ = (x);                                                                     \
    if (rc_ > 0)                                                                             \
      return fail(SPIFFE_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString((cudaError_t)rc_)); \
    if (rc_ < 0)                                                                             \
      return rc_;                                                                            \
  } while (0)

// ------------------------------------------------------------- host state

// One secondary-emission material as the reference holds it
// (SECONDARY_EMISSION, spiffe.h:293-317) with its queue of sources.
struct HostSecondary {
  int material = 1, verbosity = 0;
  double em = 0; // emitted momentum, beta*gamma
  long long limit = 0;
  std::vector<double> E, Y; // kinetic energy (eV), mean yield
  double pMin = 0, pMax = 0;
  std::vector<double> qz, qr, qp, qQ;
  std::vector<int16_t> qdir, qgen;
  std::vector<int32_t> qid;
  bool log = false;
  std::vector<double> log_rows; // SPIFFE_SECONDARY_LOG_COLS per emitting source
};

// One surface emitter as the reference holds it (EMITTER, spiffe.h:265-299):
// the boundary nodes it emits from, the side of each segment, and each
// segment's current density.
struct HostEmitter {
  spiffe_emitter_options o{};
  std::vector<long> iz, ir;
  std::vector<short> dir;
  std::vector<double> prof_t, prof_A;
  std::vector<double> J; // current density per segment
  double initial_v = 0, Q = 0, QoMC = 0;
  // stop_step is first computed by the first call that passes the profile;
  // until then it is 0, as fresh memory holds in the reference (emitter.c:186
  // reads it before any assignment), so a first call after step 0 emits nothing
  long long start_step = -1, stop_step = 0, step_emission_started = -1;
};

// One field sample waiting for download: its rows' coordinates and where
// its values sit in the device sample buffer (6 per gathered point, or 1
// per node read).
struct SampleEvent {
  double t = 0, param[3] = {0, 0, 0};
  std::vector<double> x; // row coordinates (snapshot pages)
  bool gathered = false; // interpolated at points, else read at nodes
  size_t offset = 0, n = 0;
  long long div = 1; // a time sequence's divisor, iz1 - iz0 + 1
};

// One define_field_sampling (SAMPLE_DEFN, spiffe.h:338-349).
struct HostSampling {
  spiffe_sample_options o{};
  long long step_interval = -1, start_step = -1, sample_index = -1;
  bool initialized = false; // fileInitialized: the parameters are fixed from the first sample
  double param[3] = {0, 0, 0};
  std::vector<SampleEvent> events;
};

// One cathode as the reference holds it (CATHODE, spiffe.h:236-262).
struct HostCathode {
  spiffe_cathode_options o;
  std::vector<double> prof_t, prof_A;
  double initial_vz = 0, QoMC = 0, Q = 0, inner_r2 = 0, outer_r2 = 0, ref_current_density = 0, current_density = 0;
  double totalArea = 0, start_time = 0, stop_time = 0, number_per_step = 0, electrons_per_macroparticle = 0;
  long long start_step = -1, stop_step = 0, step_emission_started = -1, n_bins = 0, correction_interval = 0;
  long long zoned_emission = 0;
  std::vector<long> distribution, deficit;
  std::vector<double> area, rmin;
};

// The test beam (TEST_BEAM_DEFN, spiffe.h); start_step -1 until the first step.
struct HostTestBeam {
  spiffe_test_beam_options o{};
  long long start_step = -1, stop_step = -1;
};

struct HostAntenna {
  int direction;
  long istart, iend, iposition;
  double current, frequency, phase;
  std::vector<double> t, W;
  long last_index = 0;
};

// Device state of the split-precision form (split32.cuh).
enum { S32_J_UNKNOWN = 0, S32_J_ZERO = 1, S32_J_DEPOSITED = 2 };
struct S32State {
  DevFields32 f{};
  DevBeam32 b{};
  uint8_t *umask = nullptr;
  Fdtd32Tables fdtd;
  int fdtd_mode = SPIFFE_FDTD_AUTO;
  double fdtd_dt = -1;
  Particles32Work pw;
  Poisson32Work pcw;
  bool pc_ready = false;
  int qexp = -60; // q_ref = 2^qexp bounds |Q| of every macroparticle (fixed-point scale)
  S32Scales sc{};
  // what J holds: unknown, zero, or exactly the deposit of the current
  // particles (left by the push of the previous step inside the loop)
  int j_state = S32_J_UNKNOWN;
  // cell sort every 40 steps (on the gun, 20 / 40 / 80 / 160: 173.5 /
  // 170.8 / 170.5 / 171.1 us a step; 10: 178.8)
  long long sort_interval = 40, since_sort = 0;
  double *staging = nullptr; // device FP64 staging for host transfers
  size_t staging_n = 0;
  float *tm_slab = nullptr; // Ez, Er, Bphi, Bphi2 in one allocation
  bool l2_window = false;   // the stream holds an L2 persisting window over tm_slab
};

struct spiffe_gpu_instance {
  int precision = SPIFFE_PRECISION_F64;
  S32State *s32 = nullptr; // the split-precision form's device state (null for FP64)
  spiffe_mesh mesh{};
  DevMesh dm{};
  cudaStream_t stream = nullptr;
  size_t nodes = 0;
  std::vector<int16_t> h_flags;
  int16_t *d_flags = nullptr;
  DevFields<double> f{};
  DevBeam64 b{};
  long long capacity = 0, np_upper = 0;
  DevCounts *cnt = nullptr, *h_cnt = nullptr;
  DevScreens screens{};
  Fdtd64Tables fdtd;
  double fdtd_dt = -1;
  long long fdtd_steps = 0;
  Particles64Work pw;
  Poisson64Work pcw;
  bool pc_ready = false;
  int deposit_ordered = 0;
  // integration state
  int space_charge = 0;
  spiffe_push_options push{};
  spiffe_poisson_options pc{};
  long long pc_start_step = -1;
  double last_imposed_factor = -1;
  // one row per Poisson correction: time step, iterations, residual, driving
  double *d_pclog = nullptr;
  double *d_status = nullptr; // status-row reduction scratch
  LostRecord *d_lost = nullptr; // lost-particle rows since the last fetch
  unsigned long long *d_lost_n = nullptr;
  long long lost_cap = 0;
  bool lost_user = false;             // the caller reads the rows (spiffe_gpu_set_lost_log)
  std::vector<LostRecord> lost_host;  // rows fetched, not yet handed to the caller
  // secondary emission (define_secondary_emission) and the surface materials
  std::vector<HostSecondary> secondaries;
  std::vector<int16_t> h_material;
  double *d_points = nullptr;         // gather points and their fields
  size_t points_cap = 0;
  double *d_list = nullptr;           // births listed by the host
  size_t list_cap = 0;
  double *d_moments = nullptr; // exit-moment reduction scratch
  unsigned long long *d_pclog_n = nullptr;
  std::vector<HostCathode> cathodes;
  uint64_t rng_key = 0, rng_counter = 0;
  std::vector<HostEmitter> emitters;
  uint64_t rng2_key = 0, rng2_counter = 0; // random_2, the emitters' stream
  std::vector<HostSampling> samplings;
  double *d_samples = nullptr; // sampled values not yet downloaded
  size_t samples_cap = 0, samples_used = 0;
  long long *d_sample_idx = nullptr;
  double *d_sample_pts = nullptr;
  size_t sample_pts_cap = 0;
  long long *d_nodes = nullptr;            // node indices of field reads on the host's behalf
  double *d_node_vals = nullptr;
  size_t nodes_cap = 0;
  std::vector<HostAntenna> antennas;
  HostTestBeam test_beam;
  double QoMC = 0, stiffness = 1;
  BirthBin *d_bins = nullptr, *h_bins = nullptr;
  size_t bins_n = 0;
  double *h_probe = nullptr; // pinned scratch for single values
  // add_on_axis_fields: the prepared tables on the host, their device copy
  // (z, Ez, D1, D2, D3 of each field, back to back) and the device views
  std::vector<OnAxisProfile> onaxis;
  double *d_onaxis_data = nullptr;
  OnAxisField *d_onaxis = nullptr;
  // translate (the moving window): the trigger, the total translation, a
  // device flag and a scratch array of nz rows
  bool tr_on = false;
  double tr_trigger = 0, tr_zt = 0;
  int *d_tr_flag = nullptr;
  void *d_tr_scratch = nullptr;
  PhaseTimer timer;
};

// Brackets one phase with events when profiling is on.
struct PhaseScope {
  spiffe_gpu_instance *in;
  int ph;
  PhaseScope(spiffe_gpu_instance *i, int p) : in(i), ph(p)
  {
    if (in->timer.on)
      cudaEventRecord(in->timer.take_start(ph), in->stream);
  }
  ~PhaseScope()
  {
    if (in->timer.on) {
      cudaEventRecord(in->timer.pool[ph][in->timer.used[ph]].second, in->stream);
      in->timer.used[ph]++;
    }
  }
};

// ------------------------------------------------------------- utilities

static void set_devmesh(spiffe_gpu_instance *in)
{
  const spiffe_mesh &m = in->mesh;
  DevMesh &d = in->dm;
  d.nz = m.nz;
  d.nr = m.nr;
  d.pitch = in->s32 ? (m.nr + 1 + 31) / 32 * 32 : m.nr + 1;
  d.zmin = m.zmin;
  d.zmax = m.zmax;
  d.rmax = m.rmax;
  d.dz = m.dz;
  d.dr = m.dr;
  d.dt = m.dt;
  d.lower_bc = m.lower_bc;
  d.upper_bc = m.upper_bc;
  d.right_bc = m.right_bc;
  d.left_bc = m.left_bc;
  d.modes = m.modes;
  for (int k = 0; k < 3; k++) {
    d.constE[k] = m.constant_E[k];
    d.constB[k] = m.constant_B[k];
  }
  for (int k = 0; k < 6; k++)
    d.turn_off[k] = m.turn_off[k];
  d.has_solenoid = m.has_solenoid && (in->s32 ? in->s32->f.BzImposed != nullptr : in->f.BzImposed != nullptr);
  d.n_onaxis = (int)in->onaxis.size();
  d.onaxis = in->d_onaxis;
  d.oa_ext = in->cnt ? (double *)((char *)in->cnt + offsetof(DevCounts, oa_min)) : nullptr;
}

// The sine and cosine terms of every on-axis field at the push's time
// (onAxisFields.c:229-238), into the mesh parameters the push receives.
static void onaxis_terms(spiffe_gpu_instance *in)
{
  for (size_t i = 0; i < in->onaxis.size(); i++)
    in->onaxis[i].terms(in->mesh.time, false, in->dm.oa_sin[i], in->dm.oa_bf[i]);
}

static int alloc_field(double **p, size_t n, cudaStream_t s)
{
  CUDA_TRY(cudaMalloc(p, n * sizeof(double)));
  CUDA_TRY(cudaMemsetAsync(*p, 0, n * sizeof(double), s));
  return 0;
}

static int alloc_beam(DevBeam64 *b, long long n)
{
#define BA(x) CUDA_TRY(cudaMalloc(&b->x, sizeof(*b->x) * (size_t)n))
  BA(z); BA(r); BA(pz); BA(pr); BA(r_pphi); BA(vz); BA(vr); BA(vphi); BA(Q);
  BA(r0); BA(z0); BA(t0); BA(rmin); BA(rmax); BA(zmin); BA(zmax);
  BA(particleID); BA(generation); BA(status);
#undef BA
  b->capacity = n;
  return 0;
}

static void free_beam(DevBeam64 *b)
{
  void *p[] = {b->z, b->r, b->pz, b->pr, b->r_pphi, b->vz, b->vr, b->vphi, b->Q, b->r0, b->z0, b->t0,
               b->rmin, b->rmax, b->zmin, b->zmax, b->particleID, b->generation, b->status};
  for (void *q : p)
    cudaFree(q);
  *b = DevBeam64{};
}

static int s32_grow(spiffe_gpu_instance *in, long long need);

// Grows the particle arrays so `need` particles fit (trealloc of cathode.c:427-456).
static int grow_beam(spiffe_gpu_instance *in, long long need)
{
  if (need <= in->capacity)
    return 0;
  if (in->s32)
    return s32_grow(in, need);
  long long cap = in->capacity * 3 / 2;
  if (cap < need + need / 10 + 1)
    cap = need + need / 10 + 1;
  DevBeam64 nb{};
  RC_TRY(alloc_beam(&nb, cap));
  const size_t n = (size_t)in->capacity;
  cudaStream_t s = in->stream;
#define CP(x) CUDA_TRY(cudaMemcpyAsync(nb.x, in->b.x, sizeof(*nb.x) * n, cudaMemcpyDeviceToDevice, s))
  CP(z); CP(r); CP(pz); CP(pr); CP(r_pphi); CP(vz); CP(vr); CP(vphi); CP(Q);
  CP(r0); CP(z0); CP(t0); CP(rmin); CP(rmax); CP(zmin); CP(zmax);
  CP(particleID); CP(generation); CP(status);
#undef CP
  CUDA_TRY(cudaStreamSynchronize(s));
  free_beam(&in->b);
  in->b = nb;
  in->capacity = cap;
  RC_TRY(spiffe_particles64_work(&in->pw, cap, in->deposit_ordered));
  if (in->pc_ready)
    RC_TRY(spiffe_poisson64_setup(&in->dm, &in->pcw, cap, s));
  return 0;
}

static int read_counts(spiffe_gpu_instance *in)
{
  CUDA_TRY(cudaMemcpyAsync(in->h_cnt, in->cnt, sizeof(DevCounts), cudaMemcpyDeviceToHost, in->stream));
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  in->np_upper = in->h_cnt->np;
  if (in->h_cnt->error & SPIFFE_DEV_ERR_CAPACITY)
    return fail(SPIFFE_ERR_CAPACITY, "particle capacity exceeded on the device");
  if (in->h_cnt->error & SPIFFE_DEV_ERR_BARRIER)
    return fail(SPIFFE_ERR_DEVICE, "Poisson solver grid barrier timed out");
  if (in->h_cnt->error & SPIFFE_DEV_ERR_WAIT)
    return fail(SPIFFE_ERR_DEVICE, "a bounded wait of the fused FDTD kernel ran out");
  if (in->h_cnt->error & SPIFFE_DEV_ERR_INDEX)
    return fail(SPIFFE_ERR_INVALID, "a particle moved more than 32767 cells outside the mesh (split-precision cell range)");
  if (in->h_cnt->screen_overflow)
    return fail(SPIFFE_ERR_CAPACITY, "screen record capacity exceeded (%lld records dropped)",
                in->h_cnt->screen_overflow);
  return 0;
}

static int ensure_fdtd(spiffe_gpu_instance *in)
{
  if (in->fdtd_dt == in->mesh.dt)
    return 0;
  RC_TRY(spiffe_fdtd64_tables(&in->dm, in->h_flags.data(), &in->fdtd, in->stream));
  in->fdtd_dt = in->mesh.dt;
  return 0;
}

static int ensure_poisson(spiffe_gpu_instance *in)
{
  if (in->pc_ready)
    return 0;
  RC_TRY(spiffe_poisson64_setup(&in->dm, &in->pcw, in->capacity, in->stream));
  in->pc_ready = true;
  return 0;
}

// ------------------------------------------------- split-precision form
//
// The same entry points on the split32.cuh representation.  Host arrays
// cross the boundary as FP64 and are converted on the device through one
// FP64 staging buffer; inside the integration loop the deposition of step
// n+1 is fused into the push of step n (j_state tracks what J holds).

static int s32_staging(spiffe_gpu_instance *in, size_t n)
{
  S32State &S = *in->s32;
  if (S.staging_n >= n)
    return 0;
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  cudaFree(S.staging);
  S.staging = nullptr;
  S.staging_n = 0;
  CUDA_TRY(cudaMalloc(&S.staging, n * sizeof(double)));
  S.staging_n = n;
  return 0;
}

static void s32_scales(spiffe_gpu_instance *in)
{
  S32State &S = *in->s32;
  const spiffe_mesh &m = in->mesh;
  const double q_ref = std::ldexp(1.0, S.qexp);
  const double one_over = 1 / (SPIFFE_PI * m.dz * (m.dr * m.dr));
  S.sc.s_charge = (float)std::ldexp(1.0, 38 - S.qexp);
  S.sc.sq_charge = S.sc.s_charge;
  S.sc.qJ = 4 * q_ref * SPIFFE_C_MKS * one_over * std::ldexp(1.0, -40);
  S.sc.kJ = (float)(-m.dt * S.sc.qJ / SPIFFE_EPSILON_O);
  S.sc.qQ = std::ldexp(1.0, S.qexp - 38);
}

static size_t s32_nodes(const spiffe_gpu_instance *in) { return (size_t)(in->mesh.nz + 1) * (size_t)in->dm.pitch; }

// Makes the fixed-point scale cover a macroparticle charge |Q| = qabs: the
// quantum grows by a power of two and the currents already accumulated are
// rescaled to it.
static int s32_cover_charge(spiffe_gpu_instance *in, double qabs)
{
  S32State &S = *in->s32;
  if (!(qabs > std::ldexp(1.0, S.qexp)) || !std::isfinite(qabs))
    return 0;
  int e = 0;
  std::frexp(qabs, &e); // qabs < 2^e
  const int shift = e - S.qexp;
  const size_t n = s32_nodes(in);
  long long *J[] = {S.f.Jz, S.f.Jr, S.f.Jphi};
  for (long long *a : J)
    RC_TRY(s32_rescale_fixed(a, n, shift, in->stream));
  S.qexp = e;
  s32_scales(in);
  return 0;
}

static int s32_alloc_f(float **p, size_t n, cudaStream_t s)
{
  CUDA_TRY(cudaMalloc(p, n * sizeof(float)));
  CUDA_TRY(cudaMemsetAsync(*p, 0, n * sizeof(float), s));
  return 0;
}

template <typename T> static int s32_alloc_z(T **p, size_t n, cudaStream_t s)
{
  CUDA_TRY(cudaMalloc(p, n * sizeof(T)));
  CUDA_TRY(cudaMemsetAsync(*p, 0, n * sizeof(T), s));
  return 0;
}

// Marks [base, base+bytes) persisting in L2 for this instance's stream: the
// FDTD reads and writes the TM fields every step and the push gathers from
// them, while the particle stream between two steps (tens of MB) would
// otherwise evict them.  The set-aside is the smaller of the device's maximum
// and the window; it belongs to this process's context.  Without support the
// call does nothing.
static int s32_l2_window(spiffe_gpu_instance *in, const void *base, size_t bytes)
{
  int dev = 0, max_persist = 0, max_window = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev));
  CUDA_TRY(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev));
  if (max_persist <= 0 || max_window <= 0)
    return 0;
  const size_t win = bytes < (size_t)max_window ? bytes : (size_t)max_window;
  size_t cur = 0;
  CUDA_TRY(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
  const size_t want = win < (size_t)max_persist ? win : (size_t)max_persist;
  if (want > cur)
    CUDA_TRY(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
  CUDA_TRY(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
  cudaStreamAttrValue a{};
  a.accessPolicyWindow.base_ptr = const_cast<void *>(base);
  a.accessPolicyWindow.num_bytes = win;
  a.accessPolicyWindow.hitRatio = cur >= win ? 1.0f : (float)cur / (float)win;
  a.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  a.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  CUDA_TRY(cudaStreamSetAttribute(in->stream, cudaStreamAttributeAccessPolicyWindow, &a));
  in->s32->l2_window = true;
  return 0;
}

static int s32_create(spiffe_gpu_instance *in, const int16_t *flags)
{
  in->s32 = new S32State();
  S32State &S = *in->s32;
  set_devmesh(in);
  const int nz = in->mesh.nz, nr = in->mesh.nr, P = in->dm.pitch;
  const size_t n = s32_nodes(in);
  cudaStream_t s = in->stream;
  RC_TRY(s32_alloc_z(&in->d_flags, n, s));
  CUDA_TRY(cudaMemcpy2DAsync(in->d_flags, (size_t)P * sizeof(int16_t), flags, (size_t)(nr + 1) * sizeof(int16_t),
                             (size_t)(nr + 1) * sizeof(int16_t), (size_t)nz + 1, cudaMemcpyHostToDevice, s));
  RC_TRY(s32_alloc_z(&S.umask, n, s));
  S.f.flags = in->d_flags;
  S.f.umask = S.umask;
  if (in->mesh.modes & SPIFFE_FL_TM_FIELDS) {
    // Ez, Er, Bphi, Bphi2 in one block, so one L2 access window can cover them
    RC_TRY(s32_alloc_f(&S.tm_slab, 4 * n, s));
    S.f.Ez = S.tm_slab;
    S.f.Er = S.tm_slab + n;
    S.f.Bphi = S.tm_slab + 2 * n;
    S.f.Bphi2 = S.tm_slab + 3 * n;
    RC_TRY(s32_alloc_z(&S.f.Jz, n, s));
    RC_TRY(s32_alloc_z(&S.f.Jr, n, s));
    // large problems only: windows of many small instances would compete
    // for one set-aside (a batch's instances are small)
    if (4 * n * sizeof(float) >= ((size_t)32 << 20))
      RC_TRY(s32_l2_window(in, S.tm_slab, 4 * n * sizeof(float)));
  }
  if (in->mesh.modes & SPIFFE_FL_TE_FIELDS) {
    float **te[] = {&S.f.Ephi, &S.f.Br, &S.f.Br2, &S.f.Bz, &S.f.Bz2};
    for (float **p : te)
      RC_TRY(s32_alloc_f(p, n, s));
    RC_TRY(s32_alloc_z(&S.f.Jphi, n, s));
  }
  RC_TRY(s32_alloc_f(&S.f.EzImposed, n, s));
  RC_TRY(s32_alloc_f(&S.f.ErImposed, n, s));
  RC_TRY(s32_alloc_z(&S.f.Psi, n, s));
  RC_TRY(s32_alloc_z(&S.f.PsiImposed, n, s));
  RC_TRY(s32_alloc_z(&S.f.Q, n, s));
  RC_TRY(s32_alloc_z(&S.f.Qp, n, s));
  CUDA_TRY(cudaMalloc(&S.f.jbox, 2 * sizeof(int)));
  RC_TRY(s32_jbox_set(S.f.jbox, 0x7fffffff, -1, s));
  RC_TRY(s32_beam_alloc(&S.b, in->capacity));
  RC_TRY(s32_particles_work(&S.pw, in->capacity));
  RC_TRY(s32_fdtd_tables(&in->dm, in->h_flags.data(), &S.fdtd, S.umask, s));
  S.fdtd_dt = in->mesh.dt;
  s32_scales(in);
  S.j_state = S32_J_ZERO;
  return 0;
}

static void s32_destroy(spiffe_gpu_instance *in)
{
  S32State &S = *in->s32;
  if (S.l2_window) {
    cudaStreamAttrValue a{};
    a.accessPolicyWindow.num_bytes = 0; // no window: release the persisting lines
    cudaStreamSetAttribute(in->stream, cudaStreamAttributeAccessPolicyWindow, &a);
    cudaCtxResetPersistingL2Cache();
  }
  void *p[] = {S.tm_slab, S.f.Ephi, S.f.Br, S.f.Br2, S.f.Bz, S.f.Bz2,
               S.f.EzImposed, S.f.ErImposed, S.f.BzImposed, S.f.BrImposed, S.f.Jz, S.f.Jr, S.f.Jphi,
               S.f.Psi, S.f.PsiImposed, S.f.Q, S.f.Qp, S.f.jbox, S.umask, S.staging};
  for (void *q : p)
    cudaFree(q);
  s32_beam_free(&S.b);
  s32_particles_work_free(&S.pw);
  s32_poisson_free(&S.pcw);
  s32_fdtd_tables_free(&S.fdtd);
  delete in->s32;
  in->s32 = nullptr;
}

static int s32_grow(spiffe_gpu_instance *in, long long need)
{
  S32State &S = *in->s32;
  long long cap = in->capacity * 3 / 2;
  if (cap < need + need / 10 + 1)
    cap = need + need / 10 + 1;
  DevBeam32 nb{};
  RC_TRY(s32_beam_alloc(&nb, cap));
  RC_TRY(s32_beam_copy(&nb, &S.b, in->capacity, in->stream));
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  s32_beam_free(&S.b);
  S.b = nb;
  in->capacity = cap;
  RC_TRY(s32_particles_work(&S.pw, cap));
  return 0;
}

static int s32_ensure_fdtd(spiffe_gpu_instance *in)
{
  S32State &S = *in->s32;
  if (S.fdtd_dt == in->mesh.dt)
    return 0;
  RC_TRY(s32_fdtd_tables(&in->dm, in->h_flags.data(), &S.fdtd, S.umask, in->stream));
  S.fdtd_dt = in->mesh.dt;
  s32_scales(in);
  return 0;
}

static int s32_ensure_poisson(spiffe_gpu_instance *in)
{
  S32State &S = *in->s32;
  if (S.pc_ready)
    return 0;
  const int rc = s32_poisson_setup(&in->dm, &S.pcw, in->capacity, in->stream);
  if (rc == (int)cudaErrorInvalidConfiguration)
    return fail(SPIFFE_ERR_UNSUPPORTED,
                "mesh %d x %d is too large for the shared-memory Poisson solver of the split-precision form",
                in->mesh.nz, in->mesh.nr);
  RC_TRY(rc);
  // the multigrid levels (a mesh too small to coarsen keeps SOR)
  const int mrc = s32_mg_setup(&in->dm, in->h_flags.data(), &S.pcw.mg, in->stream);
  if (mrc && mrc != (int)cudaErrorInvalidConfiguration)
    return fail(SPIFFE_ERR_CUDA, "multigrid set-up failed: %s", cudaGetErrorString((cudaError_t)mrc));
  S.pc_ready = true;
  return 0;
}

#define S32_FLOAT_FIELDS(X) X(Ez) X(Er) X(Bphi) X(Bphi2) X(Ephi) X(Br) X(Br2) X(Bz) X(Bz2) \
  X(EzImposed) X(ErImposed) X(BzImposed) X(BrImposed)
#define S32_F64_FIELDS(X) X(Psi) X(PsiImposed) X(Q)
#define S32_FIXED_FIELDS(X) X(Jz) X(Jr) X(Jphi)

static int s32_upload_fields(spiffe_gpu_instance *in, const spiffe_field_set *h)
{
  S32State &S = *in->s32;
  const size_t bytes = in->nodes * sizeof(double);
  cudaStream_t s = in->stream;
  RC_TRY(s32_staging(in, in->nodes));
  if (h->BzImposed && !S.f.BzImposed) {
    RC_TRY(s32_alloc_f(&S.f.BzImposed, s32_nodes(in), s));
    RC_TRY(s32_alloc_f(&S.f.BrImposed, s32_nodes(in), s));
  }
#define UP(x, call)                                                                             \
  if (h->x) {                                                                                   \
    if (!S.f.x)                                                                                 \
      return fail(SPIFFE_ERR_INVALID, "array " #x " is not part of this instance's field modes"); \
    CUDA_TRY(cudaMemcpyAsync(S.staging, h->x, bytes, cudaMemcpyHostToDevice, s));               \
    RC_TRY(call);                                                                               \
  }
#define UPF(x) UP(x, s32_to_f32(&in->dm, S.staging, S.f.x, s))
#define UPD(x) UP(x, s32_to_f64p(&in->dm, S.staging, S.f.x, s))
#define UPJ(x) UP(x, s32_to_fixed(&in->dm, S.staging, S.f.x, S.sc.qJ, s))
  S32_FLOAT_FIELDS(UPF)
  S32_F64_FIELDS(UPD)
  S32_FIXED_FIELDS(UPJ)
  if (h->Jz || h->Jr || h->Jphi) // uploaded current may be anywhere
    RC_TRY(s32_jbox_set(S.f.jbox, 0, 0x7ffffffe, s));
#undef UPF
#undef UPD
#undef UPJ
#undef UP
  if (h->Jz || h->Jr || h->Jphi)
    S.j_state = S32_J_UNKNOWN;
  set_devmesh(in);
  CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

static int s32_download_fields(spiffe_gpu_instance *in, spiffe_field_set *h)
{
  S32State &S = *in->s32;
  const size_t bytes = in->nodes * sizeof(double);
  cudaStream_t s = in->stream;
  RC_TRY(s32_staging(in, in->nodes));
#define DOWN(x, call)                                                           \
  if (h->x && S.f.x) {                                                          \
    RC_TRY(call);                                                               \
    CUDA_TRY(cudaMemcpyAsync(h->x, S.staging, bytes, cudaMemcpyDeviceToHost, s)); \
  }
#define DOF(x) DOWN(x, s32_from_f32(&in->dm, S.f.x, S.staging, s))
#define DOD(x) DOWN(x, s32_from_f64p(&in->dm, S.f.x, S.staging, s))
#define DOJ(x) DOWN(x, s32_from_fixed(&in->dm, S.f.x, S.staging, S.sc.qJ, s))
  S32_FLOAT_FIELDS(DOF)
  S32_F64_FIELDS(DOD)
  S32_FIXED_FIELDS(DOJ)
#undef DOF
#undef DOD
#undef DOJ
#undef DOWN
  if (h->flags)
    CUDA_TRY(cudaMemcpy2DAsync(h->flags, (size_t)(in->mesh.nr + 1) * sizeof(int16_t), in->d_flags,
                               (size_t)in->dm.pitch * sizeof(int16_t), (size_t)(in->mesh.nr + 1) * sizeof(int16_t),
                               (size_t)in->mesh.nz + 1, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

static int s32_upload_beam(spiffe_gpu_instance *in, const spiffe_beam_set *h)
{
  S32State &S = *in->s32;
  cudaStream_t s = in->stream;
  const long long n = h->np;
  const size_t nn = (size_t)n;
  if (n) {
    const void *need[] = {h->z, h->r, h->pz, h->pr, h->r_pphi, h->Q, h->r0, h->z0, h->t0, h->rmin, h->rmax,
                          h->zmin, h->zmax, h->particleID, h->generation, h->status};
    for (const void *p : need)
      if (!p)
        return fail(SPIFFE_ERR_INVALID, "beam array missing");
    RC_TRY(s32_staging(in, 2 * nn));
    CUDA_TRY(cudaMemcpyAsync(S.staging, h->z, nn * sizeof(double), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(S.staging + nn, h->r, nn * sizeof(double), cudaMemcpyHostToDevice, s));
    RC_TRY(s32_beam_pack_pos(&in->dm, S.staging, S.staging + nn, &S.b, n, in->cnt, s));
#define UPB(hx, dx)                                                                                 \
  CUDA_TRY(cudaMemcpyAsync(S.staging, h->hx, nn * sizeof(double), cudaMemcpyHostToDevice, s));     \
  RC_TRY(s32_d2f(S.staging, S.b.dx, n, s));
    UPB(pz, pz) UPB(pr, pr) UPB(r_pphi, rpphi) UPB(Q, Q) UPB(zmin, zmin) UPB(zmax, zmax) UPB(rmin, rmin)
    UPB(rmax, rmax)
#undef UPB
#define UPD(x) CUDA_TRY(cudaMemcpyAsync(S.b.x, h->x, nn * sizeof(*h->x), cudaMemcpyHostToDevice, s));
    UPD(r0) UPD(z0) UPD(t0) UPD(particleID) UPD(generation)
#undef UPD
    CUDA_TRY(cudaMemcpyAsync(S.staging, h->status, nn * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    RC_TRY(s32_status_pack((const uint64_t *)S.staging, S.b.status, n, s));
    double qmax = 0;
    for (size_t i = 0; i < nn; i++)
      qmax = std::fmax(qmax, std::fabs(h->Q[i]));
    RC_TRY(s32_cover_charge(in, qmax));
  }
  RC_TRY(read_counts(in));
  in->h_cnt->np = h->np;
  in->h_cnt->npActive = h->npActive;
  in->h_cnt->nextParticleID = h->nextParticleID;
  CUDA_TRY(cudaMemcpyAsync(in->cnt, in->h_cnt, sizeof(DevCounts), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  RC_TRY(read_counts(in));
  in->np_upper = h->np;
  in->QoMC = h->QoMC;
  in->stiffness = h->stiffness;
  S.j_state = S32_J_UNKNOWN;
  S.since_sort = S.sort_interval; // an uploaded beam is sorted on the next step
  return 0;
}

static int s32_download_beam(spiffe_gpu_instance *in, spiffe_beam_set *h)
{
  S32State &S = *in->s32;
  RC_TRY(read_counts(in));
  const long long np = in->h_cnt->np;
  if (np > h->capacity)
    return fail(SPIFFE_ERR_CAPACITY, "host beam holds %lld particles, device has %lld", (long long)h->capacity, np);
  cudaStream_t s = in->stream;
  const size_t n = (size_t)np;
  if (n) {
    RC_TRY(s32_staging(in, 3 * n));
    double *a = S.staging, *b = S.staging + n, *c = S.staging + 2 * n;
    RC_TRY(s32_beam_unpack_pos(&in->dm, &S.b, a, b, np, s));
    if (h->z) CUDA_TRY(cudaMemcpyAsync(h->z, a, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->r) CUDA_TRY(cudaMemcpyAsync(h->r, b, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    RC_TRY(s32_beam_unpack_vel(&in->dm, &S.b, a, b, c, np, s));
    if (h->vz) CUDA_TRY(cudaMemcpyAsync(h->vz, a, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->vr) CUDA_TRY(cudaMemcpyAsync(h->vr, b, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->vphi) CUDA_TRY(cudaMemcpyAsync(h->vphi, c, n * sizeof(double), cudaMemcpyDeviceToHost, s));
#define DNB(hx, dx)                                                                               \
  if (h->hx) {                                                                                    \
    RC_TRY(s32_f2d(S.b.dx, a, np, s));                                                            \
    CUDA_TRY(cudaMemcpyAsync(h->hx, a, n * sizeof(double), cudaMemcpyDeviceToHost, s));           \
  }
    DNB(pz, pz) DNB(pr, pr) DNB(r_pphi, rpphi) DNB(Q, Q) DNB(zmin, zmin) DNB(zmax, zmax) DNB(rmin, rmin)
    DNB(rmax, rmax)
#undef DNB
#define DND(x) if (h->x) CUDA_TRY(cudaMemcpyAsync(h->x, S.b.x, n * sizeof(*h->x), cudaMemcpyDeviceToHost, s));
    DND(r0) DND(z0) DND(t0) DND(particleID) DND(generation)
#undef DND
    if (h->status) {
      RC_TRY(s32_status_unpack(S.b.status, (uint64_t *)a, np, s));
      CUDA_TRY(cudaMemcpyAsync(h->status, a, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    }
  }
  CUDA_TRY(cudaStreamSynchronize(s));
  h->np = np;
  h->npActive = in->h_cnt->npActive;
  h->nextParticleID = (int32_t)in->h_cnt->nextParticleID;
  h->QoMC = in->QoMC;
  h->stiffness = in->stiffness;
  return 0;
}

static int s32_zero_j(spiffe_gpu_instance *in)
{
  S32State &S = *in->s32;
  const size_t bytes = s32_nodes(in) * sizeof(long long);
  long long *J[] = {S.f.Jz, S.f.Jr, S.f.Jphi};
  for (long long *a : J)
    if (a)
      CUDA_TRY(cudaMemsetAsync(a, 0, bytes, in->stream));
  RC_TRY(s32_jbox_set(S.f.jbox, 0x7fffffff, -1, in->stream));
  S.j_state = S32_J_ZERO;
  return 0;
}

static int s32_fdtd(spiffe_gpu_instance *in, int zero_j)
{
  S32State &S = *in->s32;
  RC_TRY(s32_ensure_fdtd(in));
  PhaseScope ps(in, PH_FDTD);
  in->fdtd_steps++;
  S.fdtd.mode = S.fdtd_mode;
  const int rc = s32_fdtd_step(&in->dm, &S.f, &S.fdtd, S.sc.kJ, zero_j, &in->cnt->error, in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "FDTD launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  if (zero_j)
    S.j_state = S32_J_ZERO;
  return 0;
}

static int s32_deposit_all(spiffe_gpu_instance *in)
{
  S32State &S = *in->s32;
  PhaseScope ps(in, PH_DEPOSIT);
  const int rc = s32_deposit(&in->dm, &S.f, &S.b, in->cnt, in->np_upper, &S.sc, in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "deposition launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  return 0;
}

static int after_push(spiffe_gpu_instance *in);
static int emit_emitters(spiffe_gpu_instance *in);

static LostLog lost_log(const spiffe_gpu_instance *in)
{
  return LostLog{in->d_lost, in->d_lost_n, in->lost_cap, (long long)in->mesh.time_step};
}

static int s32_push_step(spiffe_gpu_instance *in, const spiffe_push_options *o, int deposit)
{
  S32State &S = *in->s32;
  const spiffe_mesh &m = in->mesh;
  if (o->tb_electrons_per_macroparticle)
    in->stiffness = 1; // advance_particles.c:280-281
  onaxis_terms(in);
  Push32Params p{};
  p.time = m.time;
  p.dt = (float)m.dt;
  p.dt_dz = (float)(m.dt / m.dz);
  p.dt_dr = (float)(m.dt / m.dr);
  p.QoMC_dt = (float)(in->QoMC * m.dt);
  p.stiff_inv = (float)(1 / in->stiffness);
  p.z_forces_start = o->z_forces_start;
  p.zfs_on = o->z_forces_start > m.zmin && o->z_forces_start < m.zmax;
  p.forced = o->tb_electrons_per_macroparticle && (o->tb_z_force || o->tb_r_force);
  p.tb_z_force_dt = (float)(m.dt * o->tb_z_force);
  p.tb_r_force_dt = (float)(m.dt * o->tb_r_force);
  p.tb_z_decel = o->tb_z_start_deceleration;
  p.tb_r_decel = o->tb_r_start_deceleration;
  p.screen_momentum = o->screen_momentum;
  p.deposit = deposit;
  p.lost = lost_log(in);
  PhaseScope ps(in, PH_PUSH);
  in->screens.step = in->mesh.time_step;
  const int rc = s32_push(&in->dm, &S.f, &S.b, &p, &in->screens, in->cnt, in->np_upper, o->compaction, &S.sc, &S.pw,
                          in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "push launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  S.j_state = deposit ? S32_J_DEPOSITED : S32_J_UNKNOWN;
  return after_push(in);
}

// ------------------------------------------------------------------ C ABI

extern "C" const char *spiffe_gpu_last_error(void) { return g_error.c_str(); }
extern "C" const char *spiffe_gpu_version(void) { return "spiffe_b200 0.1 (sm_100a)"; }

extern "C" int spiffe_gpu_create(const spiffe_mesh *mesh, const int16_t *flags, int32_t precision,
                                 int64_t particle_capacity, spiffe_gpu_instance **out)
{
  if (!mesh || !flags || !out)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (precision != SPIFFE_PRECISION_F64 && precision != SPIFFE_PRECISION_SPLIT32)
    return fail(SPIFFE_ERR_UNSUPPORTED, "unknown precision %d", (int)precision);
  if (mesh->nz < 3 || mesh->nr < 4)
    return fail(SPIFFE_ERR_INVALID, "mesh too small (nz=%d nr=%d; need nz>=3, nr>=4)", mesh->nz, mesh->nr);
  if (!(mesh->dz > 0) || !(mesh->dr > 0))
    return fail(SPIFFE_ERR_INVALID, "dz and dr must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(SPIFFE_ERR_CUDA, "no CUDA device available");
  spiffe_gpu_instance *in = new spiffe_gpu_instance();
  in->precision = precision;
  in->mesh = *mesh;
  in->nodes = (size_t)(mesh->nz + 1) * (size_t)(mesh->nr + 1);
  in->h_flags.assign(flags, flags + in->nodes);
  int rc = 0;
  auto bail = [&](int code) {
    spiffe_gpu_destroy(in);
    return code;
  };
  if (cudaStreamCreateWithFlags(&in->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(SPIFFE_ERR_CUDA, "stream creation failed"));
  cudaStream_t s = in->stream;
  const size_t n = in->nodes;
  in->capacity = particle_capacity > 1024 ? particle_capacity : 1024;
  if (cudaMalloc(&in->cnt, sizeof(DevCounts)) != cudaSuccess ||
      cudaMallocHost(&in->h_cnt, sizeof(DevCounts)) != cudaSuccess ||
      cudaMallocHost(&in->h_probe, 8 * sizeof(double)) != cudaSuccess)
    return bail(fail(SPIFFE_ERR_NOMEM, "counter allocation failed"));
  memset(in->h_cnt, 0, sizeof(DevCounts));
  in->h_cnt->nextParticleID = 1;
  in->h_cnt->first_lost = 0x7fffffffffffffffLL;
  if (cudaMemcpyAsync(in->cnt, in->h_cnt, sizeof(DevCounts), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return bail(fail(SPIFFE_ERR_CUDA, "counter upload failed"));
  if (precision == SPIFFE_PRECISION_SPLIT32) {
    if (mesh->nz > 32767 || mesh->nr > 32767)
      return bail(fail(SPIFFE_ERR_INVALID, "the split-precision form holds at most 32767 cells per axis"));
    if ((rc = s32_create(in, flags)))
      return bail(rc);
    if (cudaStreamSynchronize(s) != cudaSuccess)
      return bail(fail(SPIFFE_ERR_CUDA, "instance setup failed: %s", cudaGetErrorString(cudaGetLastError())));
    *out = in;
    return 0;
  }
  if (cudaMalloc(&in->d_flags, n * sizeof(int16_t)) != cudaSuccess ||
      cudaMemcpyAsync(in->d_flags, flags, n * sizeof(int16_t), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return bail(fail(SPIFFE_ERR_NOMEM, "flag allocation failed"));
  DevFields<double> &f = in->f;
  f.flags = in->d_flags;
  double **tm[] = {&f.Ez, &f.Er, &f.Bphi, &f.Bphi2, &f.Jz, &f.Jr, &f.EzImposed, &f.ErImposed, &f.PsiImposed, &f.Psi, &f.Q};
  for (double **p : tm)
    if ((rc = alloc_field(p, n, s)))
      return bail(rc);
  if (mesh->modes & SPIFFE_FL_TE_FIELDS) {
    double **te[] = {&f.Ephi, &f.Jphi, &f.Br, &f.Br2, &f.Bz, &f.Bz2};
    for (double **p : te)
      if ((rc = alloc_field(p, n, s)))
        return bail(rc);
  }
  if ((rc = alloc_beam(&in->b, in->capacity)))
    return bail(rc);
  if ((rc = spiffe_particles64_work(&in->pw, in->capacity, false)))
    return bail(fail(SPIFFE_ERR_NOMEM, "particle work allocation failed"));
  set_devmesh(in);
  if (cudaStreamSynchronize(s) != cudaSuccess)
    return bail(fail(SPIFFE_ERR_CUDA, "instance setup failed: %s", cudaGetErrorString(cudaGetLastError())));
  *out = in;
  return 0;
}

extern "C" int spiffe_gpu_destroy(spiffe_gpu_instance *in)
{
  if (!in)
    return 0;
  if (in->stream)
    cudaStreamSynchronize(in->stream);
  if (in->s32)
    s32_destroy(in);
  DevFields<double> &f = in->f;
  void *p[] = {f.Ez, f.Er, f.Bphi, f.Bphi2, f.Jz, f.Jr, f.Ephi, f.Jphi, f.Br, f.Br2, f.Bz, f.Bz2,
               f.EzImposed, f.ErImposed, f.PsiImposed, f.BzImposed, f.BrImposed, f.Psi, f.Q, in->d_flags,
               in->cnt, in->d_bins, in->d_onaxis_data, in->d_onaxis, in->d_tr_flag, in->d_tr_scratch, in->d_pclog, in->d_status, in->d_moments, in->d_lost, in->d_points,
               in->d_list, in->d_nodes, in->d_node_vals, in->d_samples, in->d_sample_idx, in->d_sample_pts};
  for (void *q : p)
    cudaFree(q);
  for (int k = 0; k < in->screens.n; k++) {
    DevScreen &sc = in->screens.s[k];
    for (int c = 0; c < SPIFFE_SCREEN_QUANS; c++)
      cudaFree(sc.col[c]);
    cudaFree(sc.rmin);
    cudaFree(sc.rmax);
    cudaFree(sc.zmin);
    cudaFree(sc.zmax);
    cudaFree(sc.generation);
    cudaFree(sc.particleID);
    cudaFree(sc.order);
  }
  free_beam(&in->b);
  spiffe_fdtd64_tables_free(&in->fdtd);
  spiffe_particles64_work_free(&in->pw);
  spiffe_poisson64_free(&in->pcw);
  in->timer.release();
  if (in->h_cnt)
    cudaFreeHost(in->h_cnt);
  if (in->h_bins)
    cudaFreeHost(in->h_bins);
  if (in->h_probe)
    cudaFreeHost(in->h_probe);
  if (in->stream)
    cudaStreamDestroy(in->stream);
  delete in;
  return 0;
}

extern "C" int spiffe_gpu_set_mesh(spiffe_gpu_instance *in, const spiffe_mesh *m)
{
  if (!in || !m)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (m->nz != in->mesh.nz || m->nr != in->mesh.nr || m->dz != in->mesh.dz || m->dr != in->mesh.dr ||
      m->zmin != in->mesh.zmin || (m->modes & 3u) != (in->mesh.modes & 3u))
    return fail(SPIFFE_ERR_INVALID, "set_mesh cannot change the mesh geometry or field modes");
  const bool bc_changed = m->left_bc != in->mesh.left_bc || m->right_bc != in->mesh.right_bc ||
                          m->upper_bc != in->mesh.upper_bc || m->lower_bc != in->mesh.lower_bc;
  in->mesh = *m;
  set_devmesh(in);
  if (bc_changed && in->s32 && in->s32->pc_ready) {
    // the multigrid's operators include the end rows' conditions
    const int mrc = s32_mg_setup(&in->dm, in->h_flags.data(), &in->s32->pcw.mg, in->stream);
    if (mrc && mrc != (int)cudaErrorInvalidConfiguration)
      return fail(SPIFFE_ERR_CUDA, "multigrid set-up failed: %s", cudaGetErrorString((cudaError_t)mrc));
  }
  return 0;
}

extern "C" int spiffe_gpu_get_mesh(spiffe_gpu_instance *in, spiffe_mesh *m)
{
  if (!in || !m)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  *m = in->mesh;
  return 0;
}

#define FIELD_LIST(X) X(Ez) X(Er) X(Bphi) X(Bphi2) X(Jz) X(Jr) X(Ephi) X(Jphi) X(Br) X(Br2) X(Bz) X(Bz2) \
  X(EzImposed) X(ErImposed) X(PsiImposed) X(BzImposed) X(BrImposed) X(Psi) X(Q)

extern "C" int spiffe_gpu_upload_fields(spiffe_gpu_instance *in, const spiffe_field_set *h)
{
  if (!in || !h)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (in->s32)
    return s32_upload_fields(in, h);
  const size_t bytes = in->nodes * sizeof(double);
  cudaStream_t s = in->stream;
  if (h->BzImposed && !in->f.BzImposed) {
    RC_TRY(alloc_field(&in->f.BzImposed, in->nodes, s));
    RC_TRY(alloc_field(&in->f.BrImposed, in->nodes, s));
  }
#define UP(x)                                                                                   \
  if (h->x) {                                                                                   \
    if (!in->f.x)                                                                               \
      return fail(SPIFFE_ERR_INVALID, "array " #x " is not part of this instance's field modes"); \
    CUDA_TRY(cudaMemcpyAsync(in->f.x, h->x, bytes, cudaMemcpyHostToDevice, s));                 \
  }
  FIELD_LIST(UP)
#undef UP
  set_devmesh(in);
  CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

extern "C" int spiffe_gpu_download_fields(spiffe_gpu_instance *in, spiffe_field_set *h)
{
  if (!in || !h)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (in->s32)
    return s32_download_fields(in, h);
  const size_t bytes = in->nodes * sizeof(double);
  cudaStream_t s = in->stream;
#define DOWN(x)                                                                 \
  if (h->x && in->f.x)                                                          \
    CUDA_TRY(cudaMemcpyAsync(h->x, in->f.x, bytes, cudaMemcpyDeviceToHost, s));
  FIELD_LIST(DOWN)
#undef DOWN
  if (h->flags)
    CUDA_TRY(cudaMemcpyAsync(h->flags, in->d_flags, in->nodes * sizeof(int16_t), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

#define BEAM_LIST(X) X(z) X(r) X(pz) X(pr) X(r_pphi) X(vz) X(vr) X(vphi) X(Q) X(r0) X(z0) X(t0) \
  X(rmin) X(rmax) X(zmin) X(zmax) X(particleID) X(generation) X(status)

extern "C" int spiffe_gpu_upload_beam(spiffe_gpu_instance *in, const spiffe_beam_set *h)
{
  if (!in || !h)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (h->np < 0)
    return fail(SPIFFE_ERR_INVALID, "negative particle count");
  RC_TRY(grow_beam(in, h->np));
  if (in->s32)
    return s32_upload_beam(in, h);
  cudaStream_t s = in->stream;
  const size_t n = (size_t)h->np;
#define UPB(x)                                                                                 \
  if (n) {                                                                                     \
    if (!h->x)                                                                                 \
      return fail(SPIFFE_ERR_INVALID, "beam array " #x " missing");                            \
    CUDA_TRY(cudaMemcpyAsync(in->b.x, h->x, sizeof(*h->x) * n, cudaMemcpyHostToDevice, s));    \
  }
  BEAM_LIST(UPB)
#undef UPB
  RC_TRY(read_counts(in));
  in->h_cnt->np = h->np;
  in->h_cnt->npActive = h->npActive;
  in->h_cnt->nextParticleID = h->nextParticleID;
  CUDA_TRY(cudaMemcpyAsync(in->cnt, in->h_cnt, sizeof(DevCounts), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  in->np_upper = h->np;
  in->QoMC = h->QoMC;
  in->stiffness = h->stiffness;
  return 0;
}

extern "C" int spiffe_gpu_download_beam(spiffe_gpu_instance *in, spiffe_beam_set *h)
{
  if (!in || !h)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (in->s32)
    return s32_download_beam(in, h);
  RC_TRY(read_counts(in));
  const long long np = in->h_cnt->np;
  if (np > h->capacity)
    return fail(SPIFFE_ERR_CAPACITY, "host beam holds %lld particles, device has %lld", (long long)h->capacity, np);
  cudaStream_t s = in->stream;
  const size_t n = (size_t)np;
#define DOWNB(x)                                                                                \
  if (n && h->x)                                                                                \
    CUDA_TRY(cudaMemcpyAsync(h->x, in->b.x, sizeof(*h->x) * n, cudaMemcpyDeviceToHost, s));
  BEAM_LIST(DOWNB)
#undef DOWNB
  CUDA_TRY(cudaStreamSynchronize(s));
  h->np = np;
  h->npActive = in->h_cnt->npActive;
  h->nextParticleID = (int32_t)in->h_cnt->nextParticleID;
  h->QoMC = in->QoMC;
  h->stiffness = in->stiffness;
  return 0;
}

extern "C" int spiffe_gpu_set_deposit_order(spiffe_gpu_instance *in, int32_t ordered)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (in->s32)
    return 0; // fixed-point deposition is order-independent already
  in->deposit_ordered = ordered ? 1 : 0;
  RC_TRY(spiffe_particles64_work(&in->pw, in->capacity, in->deposit_ordered));
  return 0;
}

extern "C" int spiffe_gpu_zero_current_arrays(spiffe_gpu_instance *in)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (in->s32)
    return s32_zero_j(in);
  const size_t bytes = in->nodes * sizeof(double);
  if (in->mesh.modes & SPIFFE_FL_TM_FIELDS) {
    CUDA_TRY(cudaMemsetAsync(in->f.Jz, 0, bytes, in->stream));
    CUDA_TRY(cudaMemsetAsync(in->f.Jr, 0, bytes, in->stream));
  }
  if (in->mesh.modes & SPIFFE_FL_TE_FIELDS)
    CUDA_TRY(cudaMemsetAsync(in->f.Jphi, 0, bytes, in->stream));
  return 0;
}

extern "C" int spiffe_gpu_advance_field_solutions(spiffe_gpu_instance *in)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (in->s32)
    return s32_fdtd(in, 0);
  RC_TRY(ensure_fdtd(in));
  PhaseScope ps(in, PH_FDTD);
  in->fdtd_steps++;
  const int rc = spiffe_fdtd64_step(&in->dm, &in->f, &in->fdtd, in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "FDTD launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  return 0;
}

extern "C" int spiffe_gpu_add_particle_currents(spiffe_gpu_instance *in)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (in->s32) {
    RC_TRY(s32_deposit_all(in));
    in->s32->j_state = S32_J_UNKNOWN;
    return 0;
  }
  PhaseScope ps(in, PH_DEPOSIT);
  const int rc = spiffe_deposit64(&in->dm, &in->f, &in->b, in->cnt, in->np_upper, in->deposit_ordered, &in->pw,
                                  in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "deposition launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  return 0;
}

extern "C" int spiffe_gpu_advance_particles(spiffe_gpu_instance *in, const spiffe_push_options *o)
{
  if (!in || !o)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (in->s32)
    return s32_push_step(in, o, 0);
  if (o->tb_electrons_per_macroparticle)
    in->stiffness = 1; // advance_particles.c:280-281
  onaxis_terms(in);
  PushHostParams p{in->mesh.time, o->z_forces_start, in->QoMC, in->stiffness, o->tb_electrons_per_macroparticle,
                   o->tb_z_force, o->tb_r_force, o->tb_z_start_deceleration, o->tb_r_start_deceleration,
                   o->screen_momentum, o->compaction, lost_log(in)};
  {
    PhaseScope ps(in, PH_PUSH);
    in->screens.step = in->mesh.time_step;
    const int rc = spiffe_push64(&in->dm, &in->f, &in->b, &p, &in->screens, in->cnt, in->np_upper, &in->pw,
                                 in->stream);
    if (rc)
      return fail(SPIFFE_ERR_CUDA, "push launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  }
  return after_push(in);
}

extern "C" int spiffe_gpu_solve_poisson_cyl(spiffe_gpu_instance *in, int32_t target, double accuracy,
                                            int64_t limit, int64_t *iterations)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (accuracy <= 0)
    return fail(SPIFFE_ERR_INVALID, "accuracy is <= 0 in solve_poisson_cyl"); // poisson.c:27-28
  if (limit <= 1)
    return fail(SPIFFE_ERR_INVALID, "iteration_limit is <= 1 in solve_poisson_cyl"); // poisson.c:29-30
  if (in->s32) {
    S32State &S = *in->s32;
    RC_TRY(s32_ensure_poisson(in));
    const int rc = target ? s32_sor(&in->dm, &S.pcw, S.f.PsiImposed, nullptr, S.umask, accuracy, limit, nullptr,
                                    in->cnt, in->stream)
                          : s32_solve(&in->dm, &S.pcw, S.f.Psi, S.f.Q, S.umask, accuracy, limit, nullptr, in->cnt,
                                      in->stream);
    if (rc)
      return fail(SPIFFE_ERR_CUDA, "SOR launch failed: %s", cudaGetErrorString((cudaError_t)rc));
    long long it = 0;
    CUDA_TRY(cudaMemcpyAsync(&it, S.pcw.iters, sizeof(it), cudaMemcpyDeviceToHost, in->stream));
    RC_TRY(read_counts(in));
    if (iterations)
      *iterations = it;
    return 0;
  }
  RC_TRY(ensure_poisson(in));
  long long it = 0;
  double *psi = target ? in->f.PsiImposed : in->f.Psi;
  const double *rhs = target ? nullptr : in->f.Q;
  const int rc = spiffe_sor64(&in->dm, &in->pcw, psi, rhs, in->d_flags, accuracy, limit, in->cnt, &it, in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "SOR launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  RC_TRY(read_counts(in));
  if (iterations)
    *iterations = it;
  return 0;
}

constexpr long long PCLOG_ROWS = 1 << 16;

// appends this correction's row to the instance's log (rows past the
// capacity are counted, not stored)
__global__ void k_pc_log(const PcState *st, const double *driving, long long step, double *log,
                         unsigned long long *n)
{
  if (!st->do_solve)
    return;
  const unsigned long long k = (*n)++;
  if (k < (unsigned long long)PCLOG_ROWS) {
    log[4 * k] = (double)step;
    log[4 * k + 1] = (double)st->iterations;
    log[4 * k + 2] = st->residual;
    log[4 * k + 3] = *driving;
  }
}

static int pc_log(spiffe_gpu_instance *in, const PcState *st, const double *driving)
{
  if (!in->d_pclog) {
    CUDA_TRY(cudaMalloc(&in->d_pclog, sizeof(double) * 4 * PCLOG_ROWS + sizeof(unsigned long long)));
    in->d_pclog_n = (unsigned long long *)(in->d_pclog + 4 * PCLOG_ROWS);
    CUDA_TRY(cudaMemsetAsync(in->d_pclog_n, 0, sizeof(unsigned long long), in->stream));
  }
  k_pc_log<<<1, 1, 0, in->stream>>>(st, driving, in->mesh.time_step, in->d_pclog, in->d_pclog_n);
  spiffe_note_launches(1);
  return 0;
}

extern "C" int spiffe_gpu_poisson_log(spiffe_gpu_instance *in, int64_t max_rows, double *rows, int64_t *n_total)
{
  if (!in || (max_rows > 0 && !rows) || !n_total)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  unsigned long long n = 0;
  if (in->d_pclog) {
    CUDA_TRY(cudaMemcpyAsync(&n, in->d_pclog_n, sizeof(n), cudaMemcpyDeviceToHost, in->stream));
    CUDA_TRY(cudaStreamSynchronize(in->stream));
    const long long k = std::min<long long>(std::min<long long>((long long)n, PCLOG_ROWS), max_rows);
    if (k > 0)
      CUDA_TRY(cudaMemcpy(rows, in->d_pclog, sizeof(double) * 4 * (size_t)k, cudaMemcpyDeviceToHost));
  }
  *n_total = (int64_t)n;
  return 0;
}

static int poisson_correction(spiffe_gpu_instance *in, int space_charge, const spiffe_poisson_options *o)
{
  // poisson_correction.c:84-119
  if (o->maximum_iterations <= 0)
    return 0;
  if (in->pc_start_step == -1) {
    if (in->mesh.dt <= 0)
      return fail(SPIFFE_ERR_INVALID, "integration step size is not defined (add_poisson_correction)");
    in->pc_start_step = (long long)((o->start_time - in->mesh.start_time) / in->mesh.dt);
  }
  if (o->step_interval <= 0 || in->mesh.time_step % o->step_interval != 0 || in->pc_start_step > in->mesh.time_step)
    return 0;
  PoissonHostOptions h{o->accuracy, o->error_charge_threshold, o->maximum_iterations, o->guess_code, space_charge};
  if (in->s32) {
    S32State &S = *in->s32;
    RC_TRY(s32_ensure_poisson(in));
    PhaseScope ps(in, PH_POISSON);
    const int rc = s32_poisson_correction(&in->dm, &S.f, &S.b, in->cnt, in->np_upper, &h, &S.sc, &S.pcw, in->stream);
    if (rc)
      return fail(SPIFFE_ERR_CUDA, "Poisson correction launch failed: %s", cudaGetErrorString((cudaError_t)rc));
    RC_TRY(pc_log(in, S.pcw.st, &S.pcw.st->driving));
    return 1;
  }
  RC_TRY(ensure_poisson(in));
  PhaseScope ps(in, PH_POISSON);
  const int rc = spiffe_poisson_correction64(&in->dm, &in->f, &in->b, in->cnt, in->np_upper, &h, &in->pcw, &in->pw,
                                                 in->deposit_ordered, in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "Poisson correction launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  RC_TRY(pc_log(in, in->pcw.st, in->pcw.scalars + 4));
  return 1;
}

extern "C" int spiffe_gpu_add_poisson_correction(spiffe_gpu_instance *in, int32_t space_charge,
                                                 const spiffe_poisson_options *o, spiffe_poisson_report *rep)
{
  if (!in || !o)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  const int ran = poisson_correction(in, space_charge, o);
  if (ran < 0)
    return ran;
  if (rep) {
    memset(rep, 0, sizeof(*rep));
    if (ran) {
      RC_TRY(in->s32 ? s32_poisson_report(&in->s32->pcw, rep, in->stream)
                     : spiffe_poisson64_report(&in->pcw, rep, in->stream));
      RC_TRY(read_counts(in));
    }
  }
  return 0;
}

// compute_imposed_Efield, poisson_correction.c:456-562
static int imposed_efield(spiffe_gpu_instance *in, const spiffe_poisson_options *o, int initialize)
{
  if (o->maximum_iterations <= 0)
    return 0;
  if (in->pc_start_step == -1) {
    if (in->mesh.dt <= 0)
      return fail(SPIFFE_ERR_INVALID, "integration step size is not defined (compute_imposed_Efield)");
    in->pc_start_step = (long long)((o->start_time - in->mesh.start_time) / in->mesh.dt);
  }
  if (initialize && in->s32) {
    S32State &S = *in->s32;
    RC_TRY(s32_ensure_poisson(in));
    const int rc = s32_sor(&in->dm, &S.pcw, S.f.PsiImposed, nullptr, S.umask, o->accuracy, o->maximum_iterations,
                           nullptr, in->cnt, in->stream);
    if (rc)
      return fail(SPIFFE_ERR_CUDA, "SOR launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  } else if (initialize) {
    RC_TRY(ensure_poisson(in));
    const int rc = spiffe_sor64(&in->dm, &in->pcw, in->f.PsiImposed, nullptr, in->d_flags, o->accuracy,
                                o->maximum_iterations, in->cnt, nullptr, in->stream);
    if (rc)
      return fail(SPIFFE_ERR_CUDA, "SOR launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  }
  const double T = in->mesh.imposed_ramp_time, F = in->mesh.imposed_flat_top_time, t = in->mesh.time;
  double ff = 1;
  if (T) {
    if (t < T)
      ff = t / T;
    else if (t < (T + F))
      ff = 1;
    else if (t < (2 * T + F))
      ff = ((2 * T + F) - t) / T;
    else
      ff = 0;
    if (ff < 0)
      ff = 0;
  }
  if (ff == in->last_imposed_factor)
    return 0;
  in->last_imposed_factor = ff;
  const int rc = in->s32 ? s32_imposed_field(&in->dm, &in->s32->f, ff, in->stream)
                         : spiffe_imposed_field64(&in->dm, &in->f, ff, in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "imposed field launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  return 0;
}

extern "C" int spiffe_gpu_compute_imposed_efield(spiffe_gpu_instance *in, const spiffe_poisson_options *o,
                                                 int32_t initialize)
{
  if (!in || !o)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  RC_TRY(imposed_efield(in, o, initialize));
  return 0;
}

// ----------------------------------------------------------------- screens

extern "C" int spiffe_gpu_add_screen(spiffe_gpu_instance *in, double z_position, int32_t direction, int64_t capacity)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (in->screens.n >= SPIFFE_MAX_SCREENS)
    return fail(SPIFFE_ERR_INVALID, "at most %d screens", SPIFFE_MAX_SCREENS);
  if (direction != 1 && direction != -1)
    return fail(SPIFFE_ERR_INVALID, "screen direction must be +1 or -1");
  if (capacity <= 0)
    return fail(SPIFFE_ERR_INVALID, "screen capacity must be positive");
  DevScreen &sc = in->screens.s[in->screens.n];
  sc = DevScreen{};
  sc.z_position = z_position;
  sc.direction = direction;
  sc.cell = (int)std::floor((z_position - in->mesh.zmin) / in->mesh.dz);
  sc.capacity = capacity;
  const size_t n = (size_t)capacity;
  for (int c = 0; c < SPIFFE_SCREEN_QUANS; c++)
    CUDA_TRY(cudaMalloc(&sc.col[c], n * sizeof(double)));
  CUDA_TRY(cudaMalloc(&sc.rmin, n * sizeof(double)));
  CUDA_TRY(cudaMalloc(&sc.rmax, n * sizeof(double)));
  CUDA_TRY(cudaMalloc(&sc.zmin, n * sizeof(double)));
  CUDA_TRY(cudaMalloc(&sc.zmax, n * sizeof(double)));
  CUDA_TRY(cudaMalloc(&sc.generation, n * sizeof(int16_t)));
  CUDA_TRY(cudaMalloc(&sc.particleID, n * sizeof(int32_t)));
  CUDA_TRY(cudaMalloc(&sc.order, n * sizeof(long long)));
  in->screens.n++;
  return 0;
}

extern "C" int spiffe_gpu_screen_count(spiffe_gpu_instance *in, int32_t is, int64_t *nb)
{
  if (!in || !nb || is < 0 || is >= in->screens.n)
    return fail(SPIFFE_ERR_INVALID, "bad screen index");
  RC_TRY(read_counts(in));
  const long long n = in->h_cnt->screen_nb[is];
  *nb = n < in->screens.s[is].capacity ? n : in->screens.s[is].capacity;
  return 0;
}

extern "C" int spiffe_screen_moments_device(const DevScreen *scr, const long long *nb, double *scratch,
                                            double *host_out, cudaStream_t s);

extern "C" int spiffe_gpu_screen_moments(spiffe_gpu_instance *in, int32_t is, double *out)
{
  if (!in || !out || is < 0 || is >= in->screens.n)
    return fail(SPIFFE_ERR_INVALID, "bad screen index");
  if (!in->d_moments)
    CUDA_TRY(cudaMalloc(&in->d_moments, sizeof(double) * (148 * 9 + 64)));
  const int rc = spiffe_screen_moments_device(&in->screens.s[is], &in->cnt->screen_nb[is], in->d_moments, out,
                                              in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "screen moments failed: %s", cudaGetErrorString((cudaError_t)rc));
  return 0;
}

// The device log of lost particles runs while the caller asked for the rows
// or secondary emission needs them; capacity: rows between fetches.
static int lost_log_size(spiffe_gpu_instance *in, long long capacity)
{
  if (capacity == in->lost_cap)
    return 0;
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  cudaFree(in->d_lost);
  in->d_lost = nullptr;
  in->d_lost_n = nullptr;
  in->lost_cap = 0;
  if (capacity == 0)
    return 0;
  if (cudaMalloc(&in->d_lost, sizeof(LostRecord) * (size_t)capacity + 256) != cudaSuccess)
    return fail(SPIFFE_ERR_NOMEM, "lost-particle log of %lld rows does not fit", capacity);
  in->d_lost_n = (unsigned long long *)((char *)in->d_lost + sizeof(LostRecord) * (size_t)capacity);
  CUDA_TRY(cudaMemsetAsync(in->d_lost_n, 0, sizeof(unsigned long long), in->stream));
  in->lost_cap = capacity;
  return 0;
}

// Moves the device's rows to lost_host, in the reference's order within each
// step (advance_particles.c:437-440: ascending particle index).
static int fetch_lost(spiffe_gpu_instance *in)
{
  if (!in->d_lost)
    return 0;
  unsigned long long n = 0;
  CUDA_TRY(cudaMemcpyAsync(&n, in->d_lost_n, sizeof(n), cudaMemcpyDeviceToHost, in->stream));
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  if (!n)
    return 0;
  if ((long long)n > in->lost_cap)
    return fail(SPIFFE_ERR_CAPACITY, "%llu particles were lost since the last download, more than the log's %lld",
                n, in->lost_cap);
  const size_t first = in->lost_host.size();
  in->lost_host.resize(first + n);
  CUDA_TRY(cudaMemcpy(in->lost_host.data() + first, in->d_lost, sizeof(LostRecord) * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemsetAsync(in->d_lost_n, 0, sizeof(unsigned long long), in->stream));
  std::sort(in->lost_host.begin() + (long)first, in->lost_host.end(), [](const LostRecord &a, const LostRecord &b) {
    return a.step != b.step ? a.step < b.step : a.ip < b.ip;
  });
  return 0;
}

extern "C" int spiffe_gpu_set_lost_log(spiffe_gpu_instance *in, int64_t capacity)
{
  if (!in || capacity < 0)
    return fail(SPIFFE_ERR_INVALID, "bad argument");
  in->lost_user = capacity > 0;
  if (!in->lost_user)
    in->lost_host.clear();
  const long long need = in->lost_user ? capacity : (in->secondaries.empty() ? 0 : in->capacity);
  return lost_log_size(in, std::max<long long>(need, in->secondaries.empty() ? 0 : in->capacity));
}

extern "C" int spiffe_gpu_download_lost(spiffe_gpu_instance *in, spiffe_lost_set *h)
{
  if (!in || !h)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  h->nb = 0;
  RC_TRY(fetch_lost(in));
  const size_t n = in->lost_host.size();
  if ((long long)n > h->capacity)
    return fail(SPIFFE_ERR_CAPACITY, "%zu lost-particle rows do not fit the %lld of the host buffer", n,
                (long long)h->capacity);
  for (size_t k = 0; k < n; k++) {
    const LostRecord &r = in->lost_host[k];
    h->t[k] = r.t;
    h->rLost[k] = r.rLost;
    h->zLost[k] = r.zLost;
    h->pz[k] = r.pz;
    h->pr[k] = r.pr;
    h->z0[k] = r.z0;
    h->r0[k] = r.r0;
    h->q[k] = r.q;
    h->generation[k] = r.gen;
    h->particleID[k] = r.id;
    if (h->step)
      h->step[k] = r.step;
    if (h->p)
      h->p[k] = r.p;
    if (h->direction)
      h->direction[k] = r.code;
  }
  h->nb = (int64_t)n;
  in->lost_host.clear();
  return 0;
}

static int ensure_points(spiffe_gpu_instance *in, size_t n)
{
  if (n <= in->points_cap)
    return 0;
  cudaFree(in->d_points);
  in->d_points = nullptr;
  const size_t cap = std::max<size_t>(n, 1024);
  CUDA_TRY(cudaMalloc(&in->d_points, sizeof(double) * 4 * cap));
  in->points_cap = cap;
  return 0;
}

// queueSecondaryEmission (secondaryEmission.c:120-237) for the lost rows from
// index `first` of lost_host (this push's, in the reference's order)
static int queue_secondaries(spiffe_gpu_instance *in, size_t first)
{
  const spiffe_mesh &m = in->mesh;
  const int nz = m.nz, nr = m.nr, P = nr + 1;
  const int16_t *fl = in->h_flags.data();
  const int16_t *mat = in->h_material.empty() ? nullptr : in->h_material.data();
  struct Cand {
    size_t row;
    int im;
  };
  std::vector<Cand> cand;
  for (size_t k = first; k < in->lost_host.size(); k++) {
    const LostRecord &L = in->lost_host[k];
    const double z = L.zLost, r = L.rLost;
    if ((z + m.dz) >= m.zmax)
      continue;
    const long iz = (long)((z - m.zmin) / m.dz), ir = (long)(std::fabs(r) / m.dr), iz1 = iz + 1, ir1 = ir + 1;
    if (iz >= nz || ir >= nr || iz < 0 || ir < 0)
      continue;
    const int16_t f0 = fl[iz * P + ir];
    if (f0 & SPIFFE_FL_IS_INSIDE)
      continue;
    if (f0 & SPIFFE_FL_IS_SURFACE) {
      if (iz1 > nz || ir1 > nr)
        continue;
      if (fl[iz1 * P + ir1] & SPIFFE_FL_IS_METAL && fl[iz * P + ir1] & SPIFFE_FL_IS_METAL &&
          fl[iz1 * P + ir] & SPIFFE_FL_IS_METAL)
        continue;
    }
    int material = 0;
    if (mat) {
      const long at[4][2] = {{iz, ir}, {iz1, ir}, {iz, ir1}, {iz1, ir1}};
      for (int q = 0; q < 4 && material < 1; q++)
        material = mat[at[q][0] * P + at[q][1]];
    }
    if (material < 1)
      continue; // no secondary emission here
    int im = -1;
    for (size_t q = 0; q < in->secondaries.size(); q++)
      if (in->secondaries[q].material == material) {
        im = (int)q;
        break;
      }
    if (im < 0)
      return fail(SPIFFE_ERR_INVALID, "no match for material %d for r=%e, z=%e, (ir=%ld, iz=%ld)", material, r, z, ir,
                  iz);
    const HostSecondary &SE = in->secondaries[(size_t)im];
    if (SE.pMin > L.p || SE.pMax < L.p)
      continue;
    cand.push_back(Cand{k, im});
  }
  if (cand.empty())
    return 0;
  // the fields at the loss point, as the reference asks interpolateFields
  // for them: with z and r exchanged (secondaryEmission.c:195)
  RC_TRY(ensure_points(in, cand.size()));
  std::vector<double> pts(2 * cand.size()), E(2 * cand.size());
  for (size_t c = 0; c < cand.size(); c++) {
    pts[2 * c] = in->lost_host[cand[c].row].rLost;
    pts[2 * c + 1] = in->lost_host[cand[c].row].zLost;
  }
  double *d_pts = in->d_points, *d_E = in->d_points + 2 * in->points_cap;
  CUDA_TRY(cudaMemcpyAsync(d_pts, pts.data(), sizeof(double) * pts.size(), cudaMemcpyHostToDevice, in->stream));
  const int rc = in->s32 ? s32_gather_points(&in->dm, &in->s32->f, d_pts, (int)cand.size(), 2, d_E, in->stream)
                         : spiffe_gather_points64(&in->dm, &in->f, d_pts, (int)cand.size(), 2, d_E, in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "field gather failed: %s", cudaGetErrorString((cudaError_t)rc));
  CUDA_TRY(cudaMemcpyAsync(E.data(), d_E, sizeof(double) * E.size(), cudaMemcpyDeviceToHost, in->stream));
  RC_TRY(read_counts(in)); // synchronises; the beam's next particle ID
  long long next_id = in->h_cnt->nextParticleID;
  const long long id0 = next_id;
  for (size_t c = 0; c < cand.size(); c++) {
    const LostRecord &L = in->lost_host[cand[c].row];
    HostSecondary &SE = in->secondaries[(size_t)cand[c].im];
    const double Ez = E[2 * c], Er = E[2 * c + 1];
    const double K = SPIFFE_ME_MEV * 1e6 * (std::sqrt(SE.em * SE.em + 1) - 1);
    if ((L.code == SPIFFE_GOING_LEFT && (Ez * m.dz * 1e-9) > K) ||
        (L.code == SPIFFE_GOING_RIGHT && (-1 * Ez * m.dz * 1e-9) > K) ||
        (L.code == SPIFFE_GOING_DOWN && (Er * m.dr * 1e-9) > K) ||
        (L.code == SPIFFE_GOING_UP && (-1 * Er * m.dr * 1e-9) > K))
      continue;
    SE.qz.push_back(L.zLost);
    SE.qr.push_back(L.rLost);
    SE.qp.push_back(L.p);
    SE.qQ.push_back(L.q);
    SE.qdir.push_back(L.code);
    SE.qgen.push_back(L.gen);
    SE.qid.push_back((int32_t)next_id++);
  }
  if (next_id != id0) {
    in->h_cnt->nextParticleID = next_id;
    CUDA_TRY(cudaMemcpyAsync(&in->cnt->nextParticleID, &in->h_cnt->nextParticleID, sizeof(long long),
                             cudaMemcpyHostToDevice, in->stream));
    CUDA_TRY(cudaStreamSynchronize(in->stream));
  }
  return 0;
}

// After a push: the lost rows feed the secondary-emission queue.
static int after_push(spiffe_gpu_instance *in)
{
  if (in->secondaries.empty())
    return 0;
  const size_t first = in->lost_host.size();
  RC_TRY(fetch_lost(in));
  RC_TRY(queue_secondaries(in, first));
  if (!in->lost_user)
    in->lost_host.clear();
  return 0;
}

// inversePoissonCDF (secondaryEmission.c:586-601)
static long inverse_poisson_cdf(double mu, double C)
{
  long r = 0, rMax = (long)(10 * mu);
  const double expMinusMu = std::exp(-mu);
  double sum = expMinusMu, term = 1;
  while (r <= rMax && C > sum) {
    term *= mu / (++r);
    sum += term * expMinusMu;
  }
  return r;
}

static double rng_next(spiffe_gpu_instance *in);

// Particles the host composed (BIRTH_LIST_COLS columns of equal length)
// appended to the beam on the device, the beam grown first if they do not fit.
static int list_births(spiffe_gpu_instance *in, const std::vector<double> *col, double qmax)
{
  const size_t total = col[0].size();
  if (!total)
    return 0;
  if (in->np_upper + (long long)total > in->capacity) {
    RC_TRY(read_counts(in));
    RC_TRY(grow_beam(in, in->h_cnt->np + (long long)total));
  }
  if (in->list_cap < total) {
    cudaFree(in->d_list);
    in->d_list = nullptr;
    in->list_cap = std::max<size_t>(total, 1024);
    CUDA_TRY(cudaMalloc(&in->d_list, sizeof(double) * BIRTH_LIST_COLS * in->list_cap));
  }
  std::vector<double> flat;
  flat.reserve(BIRTH_LIST_COLS * total);
  for (int c = 0; c < BIRTH_LIST_COLS; c++)
    flat.insert(flat.end(), col[c].begin(), col[c].end());
  CUDA_TRY(cudaMemcpyAsync(in->d_list, flat.data(), sizeof(double) * flat.size(), cudaMemcpyHostToDevice, in->stream));
  BirthParams p{};
  p.total = (long long)total;
  p.mode = SPIFFE_BIRTH_LIST;
  p.list = in->d_list;
  p.time = in->mesh.time;
  int rc;
  if (in->s32) {
    S32State &S = *in->s32;
    RC_TRY(s32_cover_charge(in, qmax));
    rc = s32_births(&in->dm, &S.f, &S.b, &p, in->cnt, &S.sc, in->space_charge && S.j_state == S32_J_DEPOSITED ? 1 : 0,
                    in->stream);
  } else {
    rc = spiffe_births64(&in->dm, &in->f, &in->b, &p, in->cnt, in->stream);
  }
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "birth launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  in->np_upper += (long long)total;
  CUDA_TRY(cudaStreamSynchronize(in->stream)); // the host list is freed on return
  return 0;
}

// emitSecondaryElectrons (secondaryEmission.c:374-584): each material's queue
// in order, the number of secondaries of each source from its mean yield
// (a Poisson draw), each with a random direction away from the surface it
// hit; the births go to the device as a list.
static int emit_secondaries(spiffe_gpu_instance *in)
{
  const spiffe_mesh &m = in->mesh;
  for (HostSecondary &SE : in->secondaries) {
    if (SE.qz.empty())
      continue;
    if (SE.verbosity > 0) {
      printf("%ld secondary emission sources for material %hd\n", (long)SE.qz.size(), (short)SE.material);
      fflush(stdout);
    }
    std::vector<double> col[BIRTH_LIST_COLS];
    double qmax = 0;
    long long log_id = 0, logged = 0; // the log takes particle IDs (secondaryEmission.c:541)
    if (SE.log) {
      RC_TRY(read_counts(in));
      log_id = in->h_cnt->nextParticleID;
    }
    for (size_t s0 = 0; s0 < SE.qz.size(); s0++) {
      double gamma = std::sqrt(SE.qp[s0] * SE.qp[s0] + 1);
      const double K = (gamma - 1) * SPIFFE_ME_MEV * 1e6;
      // interp(yieldData, energyData, n, K, 0, 1, &code): linear, code 0 outside the table
      const std::vector<double> &x = SE.E, &y = SE.Y;
      const long n = (long)x.size();
      bool ok = true;
      double Y;
      if (K <= x[0]) {
        ok = !(K < x[0]);
        Y = y[0];
      } else if (K >= x[(size_t)n - 1]) {
        ok = !(K > x[(size_t)n - 1]);
        Y = y[(size_t)n - 1];
      } else {
        long lo = 0, hi = n - 1;
        while (hi - lo > 1) {
          const long mid = (lo + hi) / 2;
          if (x[(size_t)mid] <= K)
            lo = mid;
          else
            hi = mid;
        }
        Y = y[(size_t)lo] + (y[(size_t)hi] - y[(size_t)lo]) / (x[(size_t)hi] - x[(size_t)lo]) * (K - x[(size_t)lo]);
      }
      if (!ok) {
        if (SE.verbosity > 0) {
          printf("Secondary yield curve interpolation failed for K=%e eV\n", K);
          fflush(stdout);
        }
        continue;
      }
      long total = inverse_poisson_cdf(Y, rng_next(in));
      if (SE.limit > 0 && total > SE.limit)
        total = (long)SE.limit;
      for (long q = 0; q < total; q++) {
        double theta;
        switch (SE.qdir[s0]) {
        case SPIFFE_GOING_RIGHT: // the secondary goes left
          theta = -rng_next(in) * SPIFFE_PI;
          break;
        case SPIFFE_GOING_LEFT:
          theta = rng_next(in) * SPIFFE_PI;
          break;
        case SPIFFE_GOING_UP:
          theta = rng_next(in) * SPIFFE_PI + SPIFFE_PI / 2;
          break;
        case SPIFFE_GOING_DOWN:
          theta = rng_next(in) * SPIFFE_PI - SPIFFE_PI / 2;
          break;
        default:
          theta = rng_next(in) * SPIFFE_PIx2;
          break;
        }
        const double pz = SE.em * std::sin(theta), pr = SE.em * std::cos(theta);
        gamma = std::sqrt(pz * pz + pr * pr + 1);
        const double v[BIRTH_LIST_COLS] = {SE.qz[s0], SE.qr[s0], pz, pr, SPIFFE_C_MKS * pz / gamma,
                                           SPIFFE_C_MKS * pr / gamma, SE.qQ[s0], m.time, (double)(SE.qgen[s0] + 1),
                                           (double)SE.qid[s0]};
        for (int c = 0; c < BIRTH_LIST_COLS; c++)
          col[c].push_back(v[c]);
        qmax = std::max(qmax, std::fabs(SE.qQ[s0]));
      }
      if (SE.log && total > 0) {
        const double row[SPIFFE_SECONDARY_LOG_COLS] = {(double)m.time_step, SE.qz[s0], SE.qr[s0], m.time, K, Y,
                                                       (double)total, (double)SE.qdir[s0], (double)(SE.qgen[s0] + 1),
                                                       (double)(log_id + logged)};
        SE.log_rows.insert(SE.log_rows.end(), row, row + SPIFFE_SECONDARY_LOG_COLS);
        logged++;
      }
    }
    if (logged) {
      in->h_cnt->nextParticleID = log_id + logged;
      CUDA_TRY(cudaMemcpyAsync(&in->cnt->nextParticleID, &in->h_cnt->nextParticleID, sizeof(long long),
                               cudaMemcpyHostToDevice, in->stream));
      CUDA_TRY(cudaStreamSynchronize(in->stream));
    }
    const size_t total = col[0].size();
    RC_TRY(list_births(in, col, qmax));
    if (SE.verbosity > 0) {
      RC_TRY(read_counts(in));
      printf("Secondary emission increased number of particles from %lld to %lld\n",
             (long long)(in->h_cnt->np - (long long)total), (long long)in->h_cnt->np);
      fflush(stdout);
    }
    SE.qz.clear();
    SE.qr.clear();
    SE.qp.clear();
    SE.qQ.clear();
    SE.qdir.clear();
    SE.qgen.clear();
    SE.qid.clear();
  }
  return 0;
}

extern "C" int spiffe_gpu_set_materials(spiffe_gpu_instance *in, const int16_t *material)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (material)
    in->h_material.assign(material, material + in->nodes);
  else
    in->h_material.clear();
  return 0;
}

extern "C" int spiffe_gpu_add_secondary_emission(spiffe_gpu_instance *in, const spiffe_secondary_options *o)
{
  if (!in || !o)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  // processSecondaryEmissionDefinition (secondaryEmission.c:21-118)
  if (o->emitted_momentum < 0)
    return fail(SPIFFE_ERR_INVALID, "emitted_momentum < 0");
  if (o->n_data <= 0 || !o->energy || !o->yield)
    return fail(SPIFFE_ERR_INVALID, "no data in yield file");
  HostSecondary SE;
  SE.material = o->material_id;
  SE.em = o->emitted_momentum;
  SE.limit = o->yield_limit;
  SE.verbosity = o->verbosity;
  SE.E.assign(o->energy, o->energy + o->n_data);
  SE.Y.assign(o->yield, o->yield + o->n_data);
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (double e : SE.E) {
    lo = e < lo ? e : lo;
    hi = e > hi ? e : hi;
  }
  SE.pMin = std::sqrt((lo / SPIFFE_ME_MEV / 1e6 + 1) * (lo / SPIFFE_ME_MEV / 1e6 + 1) - 1);
  SE.pMax = std::sqrt((hi / SPIFFE_ME_MEV / 1e6 + 1) * (hi / SPIFFE_ME_MEV / 1e6 + 1) - 1);
  for (size_t i = 1; i < SE.E.size(); i++)
    if (SE.E[i - 1] >= SE.E[i])
      return fail(SPIFFE_ERR_INVALID, "secondary emission data is not ordered by increasing energy values");
  SE.log = o->log != 0;
  in->secondaries.push_back(std::move(SE));
  return lost_log_size(in, std::max<long long>(in->lost_cap, in->capacity));
}

extern "C" int spiffe_gpu_secondary_log(spiffe_gpu_instance *in, int32_t index, int64_t max_rows, double *rows,
                                        int64_t *n_rows)
{
  if (!in || !n_rows || index < 0 || (size_t)index >= in->secondaries.size())
    return fail(SPIFFE_ERR_INVALID, "bad argument");
  std::vector<double> &L = in->secondaries[(size_t)index].log_rows;
  const int64_t n = (int64_t)(L.size() / SPIFFE_SECONDARY_LOG_COLS);
  *n_rows = n;
  if (!rows)
    return 0;
  if (n > max_rows)
    return fail(SPIFFE_ERR_CAPACITY, "%lld emission-log rows do not fit the %lld of the host buffer", (long long)n,
                (long long)max_rows);
  std::copy(L.begin(), L.end(), rows);
  L.clear();
  return 0;
}

extern "C" int spiffe_gpu_download_screen(spiffe_gpu_instance *in, int32_t is, spiffe_screen_set *h)
{
  int64_t nb = 0;
  RC_TRY(spiffe_gpu_screen_count(in, is, &nb));
  if (nb > h->capacity)
    return fail(SPIFFE_ERR_CAPACITY, "host screen buffer holds %lld records, device has %lld", (long long)h->capacity,
                (long long)nb);
  const DevScreen &sc = in->screens.s[is];
  cudaStream_t s = in->stream;
  const size_t n = (size_t)nb;
  if (n) {
    for (int c = 0; c < SPIFFE_SCREEN_QUANS; c++)
      if (h->col[c])
        CUDA_TRY(cudaMemcpyAsync(h->col[c], sc.col[c], n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->rmin) CUDA_TRY(cudaMemcpyAsync(h->rmin, sc.rmin, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->rmax) CUDA_TRY(cudaMemcpyAsync(h->rmax, sc.rmax, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->zmin) CUDA_TRY(cudaMemcpyAsync(h->zmin, sc.zmin, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->zmax) CUDA_TRY(cudaMemcpyAsync(h->zmax, sc.zmax, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->generation)
      CUDA_TRY(cudaMemcpyAsync(h->generation, sc.generation, n * sizeof(int16_t), cudaMemcpyDeviceToHost, s));
    if (h->particleID)
      CUDA_TRY(cudaMemcpyAsync(h->particleID, sc.particleID, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  }
  std::vector<long long> order(n);
  if (n > 1)
    CUDA_TRY(cudaMemcpyAsync(order.data(), sc.order, n * sizeof(long long), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  // the pushes append crossings as they happen; the reference records them
  // step by step in particle order (advance_particles.c:362-434)
  if (n > 1 && !std::is_sorted(order.begin(), order.end())) {
    std::vector<size_t> perm(n);
    for (size_t i = 0; i < n; i++)
      perm[i] = i;
    std::sort(perm.begin(), perm.end(), [&](size_t a, size_t b) { return order[a] < order[b]; });
    auto apply = [&](auto *p) {
      if (!p)
        return;
      using T = std::remove_pointer_t<decltype(p)>;
      std::vector<T> tmp(p, p + n);
      for (size_t i = 0; i < n; i++)
        p[i] = tmp[perm[i]];
    };
    for (int c = 0; c < SPIFFE_SCREEN_QUANS; c++)
      apply(h->col[c]);
    apply(h->rmin);
    apply(h->rmax);
    apply(h->zmin);
    apply(h->zmax);
    apply(h->generation);
    apply(h->particleID);
  }
  h->nb = nb;
  h->z_position = sc.z_position;
  h->direction = sc.direction;
  return 0;
}

extern "C" int spiffe_gpu_clear_screens(spiffe_gpu_instance *in)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  RC_TRY(read_counts(in));
  for (int k = 0; k < SPIFFE_MAX_SCREENS; k++)
    in->h_cnt->screen_nb[k] = 0;
  in->h_cnt->screen_overflow = 0;
  CUDA_TRY(cudaMemcpyAsync(in->cnt, in->h_cnt, sizeof(DevCounts), cudaMemcpyHostToDevice, in->stream));
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  return 0;
}

// ---------------------------------------------------------------- cathodes

// The checks of process_cathode_definition (cathode.c:43-81) that concern
// the options the device loop uses.
extern "C" int spiffe_cathode_check(const spiffe_mesh *mesh, const spiffe_cathode_options *o)
{
  if (!mesh || !o)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  const spiffe_mesh &m = *mesh;
  if (o->z_position < m.zmin || o->z_position > m.zmax)
    return fail(SPIFFE_ERR_INVALID, "cathode is outside of simulation region");
  if (o->inner_radius > o->outer_radius)
    return fail(SPIFFE_ERR_INVALID, "cathode has negative radial extent");
  if (o->inner_radius == o->outer_radius && o->current_density != 0)
    return fail(SPIFFE_ERR_INVALID, "cathode has zero radial extent--specify electrons_per_macroparticle instead of current_density");
  if (o->inner_radius < 0 || o->outer_radius > m.rmax)
    return fail(SPIFFE_ERR_INVALID, "all or part of cathode is outside of simulation region");
  if (!o->field_emission && o->current_density <= 0 && o->electrons_per_macroparticle == 0 && o->temperature <= 0)
    return fail(SPIFFE_ERR_INVALID, "either field_emission, current_density, electrons_per_macroparticle, or temperature must be non-zero");
  if (o->current_density < 0)
    return fail(SPIFFE_ERR_INVALID, "the current density should be a positive quantity");
  if (o->electrons_per_macroparticle < 0)
    return fail(SPIFFE_ERR_INVALID, "electrons_per_macroparticle should be a positive quantity");
  if (o->stop_time && o->start_time > o->stop_time)
    return fail(SPIFFE_ERR_INVALID, "stop_time is non-zero and less than start_time");
  if (o->distribution_correction_interval < 0)
    return fail(SPIFFE_ERR_INVALID, "distribution_correction_interval < 0");
  if (o->distribution_correction_interval && o->discretize_radii)
    return fail(SPIFFE_ERR_INVALID, "distribution correction and discrete radii are incompatible");
  if (o->stiffness <= 0)
    return fail(SPIFFE_ERR_INVALID, "stiffness <= 0");
  if (std::fabs(o->initial_omega * o->outer_radius) >= SPIFFE_C_MKS)
    return fail(SPIFFE_ERR_INVALID, "initial_omega*outer_radius >= c---unphysical");
  if (o->random_number_seed == 0)
    return fail(SPIFFE_ERR_INVALID, "random_number_seed must be non-zero (a clock seed is not reproducible)");
  if (o->n_profile) {
    if (o->distribution_correction_interval)
      return fail(SPIFFE_ERR_INVALID, "can't do distribution correction with an emission profile");
    for (int i = 1; i < o->n_profile; i++)
      if (o->profile_t[i - 1] >= o->profile_t[i])
        return fail(SPIFFE_ERR_INVALID, "profile data is not ordered by increasing time values");
  }
  return 0;
}

// process_cathode_definition, cathode.c:21-237.
extern "C" int spiffe_gpu_add_cathode(spiffe_gpu_instance *in, const spiffe_cathode_options *o)
{
  if (!in || !o)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  const spiffe_mesh &m = in->mesh;
  RC_TRY(spiffe_cathode_check(&m, o));
  long n = 1;
  if (o->field_emission) {
    if (o->inner_radius != 0)
      n = (long)((o->outer_radius - o->inner_radius) / m.dr);
    else
      n = (long)((o->outer_radius - o->inner_radius + m.dr / 2) / m.dr);
  }
  const long seed = o->random_number_seed < 0 ? -(long)o->random_number_seed : o->random_number_seed;
  in->rng_key = spiffe_rng_key((uint64_t)seed); // random_1(-abs(seed)), cathode.c:90
  in->rng_counter = 0;
  for (long i = 0; i < n; i++) {
    HostCathode c;
    c.o = *o;
    if (o->n_profile) {
      c.prof_t.assign(o->profile_t, o->profile_t + o->n_profile);
      c.prof_A.assign(o->profile_A, o->profile_A + o->n_profile);
    }
    c.o.profile_t = c.o.profile_A = nullptr;
    if (o->field_emission) {
      c.o.outer_radius = (i + 0.5) * m.dr;
      if ((c.o.inner_radius = c.o.outer_radius - m.dr) < 0)
        c.o.inner_radius = 0;
      if (i == n - 1)
        c.o.outer_radius = o->outer_radius;
      if (c.o.outer_radius > o->outer_radius)
        c.o.outer_radius = o->outer_radius;
      if (c.o.inner_radius < o->inner_radius)
        c.o.inner_radius = o->inner_radius;
    }
    c.initial_vz = o->initial_pz / std::sqrt(1 + o->initial_pz * o->initial_pz) * SPIFFE_C_MKS;
    c.current_density = o->current_density;
    c.start_time = o->start_time;
    c.stop_time = o->stop_time;
    c.number_per_step = o->number_per_step;
    c.QoMC = -SPIFFE_E_MKS / (SPIFFE_ME_MKS * SPIFFE_C_MKS);
    c.correction_interval = o->distribution_correction_interval;
    c.electrons_per_macroparticle = o->electrons_per_macroparticle;
    c.zoned_emission = o->zoned_emission;
    if (o->discretize_radii)
      c.correction_interval = 0;
    if (o->field_emission)
      c.zoned_emission = 0;
    if (!c.zoned_emission)
      c.correction_interval = 0;
    in->cathodes.push_back(std::move(c));
  }
  return 0;
}

// interp(A, t, n, x, ...) of an ascending table: linear inside, the end
// values outside
static double interp_table(const std::vector<double> &A, const std::vector<double> &T, double t)
{
  const long n = (long)T.size();
  long lo = 0, hi = n - 1;
  if (t <= T[0])
    return A[0];
  if (t >= T[(size_t)hi])
    return A[(size_t)hi];
  while (hi - lo > 1) {
    const long mid = (lo + hi) / 2;
    if (T[(size_t)mid] <= t)
      lo = mid;
    else
      hi = mid;
  }
  return A[(size_t)lo] + (A[(size_t)hi] - A[(size_t)lo]) / (T[(size_t)hi] - T[(size_t)lo]) * (t - T[(size_t)lo]);
}

static double profile_value(const HostCathode &c, double t) { return interp_table(c.prof_A, c.prof_t, t); }

static double rng_next(spiffe_gpu_instance *in) { return spiffe_rng_uniform(in->rng_key, ++in->rng_counter); }

static int ensure_bins(spiffe_gpu_instance *in, size_t n)
{
  if (in->bins_n >= n)
    return 0;
  cudaFree(in->d_bins);
  if (in->h_bins)
    cudaFreeHost(in->h_bins);
  CUDA_TRY(cudaMalloc(&in->d_bins, n * sizeof(BirthBin)));
  CUDA_TRY(cudaMallocHost(&in->h_bins, n * sizeof(BirthBin)));
  in->bins_n = n;
  return 0;
}

// emit_electrons_from_cathode, cathode.c:239-671: counts on the host, births on the device.
static int emit(spiffe_gpu_instance *in)
{
  PhaseScope ps(in, PH_EMIT);
  RC_TRY(emit_secondaries(in)); // integrate.c:159-163: before the cathodes
  const spiffe_mesh &m = in->mesh;
  for (HostCathode &c : in->cathodes) {
    if (c.number_per_step == 0 && c.electrons_per_macroparticle == 0)
      continue;
    if (c.start_step == -1) {
      if (c.current_density <= 1. / std::sqrt(1.7976931348623157e308))
        continue;
      c.ref_current_density = c.current_density;
      if (c.o.autophase) {
        c.stop_time = (c.stop_time - c.start_time) + m.time + c.o.time_offset;
        c.start_time = m.time + c.o.time_offset;
      }
      if (m.dt <= 0)
        return fail(SPIFFE_ERR_INVALID, "integration step size is not defined (emit_electrons_from_cathode)");
      c.inner_r2 = c.o.inner_radius * c.o.inner_radius;
      c.outer_r2 = c.o.outer_radius * c.o.outer_radius;
      double area;
      if ((area = SPIFFE_PI * (c.outer_r2 - c.inner_r2)) != 0) {
        if (c.electrons_per_macroparticle) {
          c.number_per_step = area * m.dt * c.current_density / (SPIFFE_E_MKS * c.electrons_per_macroparticle);
          if (c.number_per_step == 0)
            continue;
        } else
          c.electrons_per_macroparticle = area * m.dt * c.current_density / (SPIFFE_E_MKS * c.number_per_step);
      } else {
        c.correction_interval = 0;
        c.n_bins = 1;
      }
      c.start_step = (long long)((c.start_time - m.start_time) / m.dt);
      if (c.stop_time && c.stop_time > m.start_time)
        c.stop_step = (long long)((c.stop_time - m.start_time) / m.dt);
      else
        c.stop_step = 0x7fffffffffffffffLL;
      c.Q = -SPIFFE_E_MKS * c.electrons_per_macroparticle;
      c.n_bins = (long long)((c.o.outer_radius - c.o.inner_radius) / m.dr + 1);
      c.distribution.assign((size_t)c.n_bins, 0);
      c.deficit.assign((size_t)c.n_bins, 0);
      c.area.assign((size_t)c.n_bins, 0);
      c.rmin.assign((size_t)c.n_bins, 0);
      c.totalArea = 0;
      for (long long ib = 0; ib < c.n_bins; ib++) {
        const long ir = (long)(c.o.inner_radius / m.dr + ib);
        if (ir == 0) {
          const double r_max = m.dr / 2;
          c.area[ib] = r_max * r_max * SPIFFE_PI;
          c.rmin[ib] = 0;
        } else {
          const double r_min = m.dr * (ir - 0.5), r_max = m.dr * (ir + 0.5);
          c.area[ib] = SPIFFE_PI * (r_max * r_max - r_min * r_min);
          c.rmin[ib] = r_min;
          c.totalArea += c.area[ib];
        }
      }
    }
    double profile_factor = 1;
    if (!c.prof_t.empty()) {
      if (m.time >= c.prof_t.front() && m.time <= c.prof_t.back())
        profile_factor = profile_value(c, m.time);
      else
        profile_factor = 0;
    }
    if (c.start_step > m.time_step || c.stop_step < m.time_step)
      continue;
    if (c.step_emission_started < 0)
      c.step_emission_started = m.time_step;
    const double dr2 = (c.outer_r2 - c.inner_r2) / c.number_per_step;
    const double total_area = c.totalArea;
    const double totalNominal = c.number_per_step * (c.current_density / c.ref_current_density);
    long long total;
    if (c.correction_interval && m.time_step % c.correction_interval == 0) {
      total = 0;
      for (long long ib = 0; ib < c.n_bins; ib++) {
        if ((c.deficit[ib] = (long)((m.time_step - c.step_emission_started + 1) * (c.area[ib] / total_area) *
                                        totalNominal +
                                    0.5) -
                             c.distribution[ib]) <= 0)
          c.deficit[ib] = 0;
        total += c.deficit[ib];
      }
    } else if (c.zoned_emission) {
      total = 0;
      for (long long ib = 0; ib < c.n_bins; ib++) {
        if (total_area) {
          double fnumber = profile_factor * (c.area[ib] / total_area) * totalNominal;
          if (fnumber > 1) {
            c.deficit[ib] = (long)fnumber;
            fnumber -= c.deficit[ib];
          } else
            c.deficit[ib] = 0;
          if (fnumber && fnumber > rng_next(in))
            c.deficit[ib] += 1;
          total += c.deficit[ib];
        }
      }
    } else {
      double fnumber = totalNominal * profile_factor;
      total = (long)fnumber;
      fnumber -= (long)fnumber;
      if (fnumber && fnumber > rng_next(in))
        total += 1;
    }
    if (total < 0)
      return fail(SPIFFE_ERR_INVALID, "negative number of particles created!");
    if (!total)
      continue;
    // make room: the bound is exact enough unless many particles were lost
    if (in->np_upper + total > in->capacity) {
      RC_TRY(read_counts(in));
      RC_TRY(grow_beam(in, in->h_cnt->np + total));
    }
    BirthParams p{};
    p.total = total;
    p.key = in->rng_key;
    p.counter_base = in->rng_counter;
    p.spread = c.o.spread_over_dt;
    p.z_position = c.o.z_position;
    p.inner_radius = c.o.inner_radius;
    p.outer_radius = c.o.outer_radius;
    p.inner_r2 = c.inner_r2;
    p.dr2 = dr2;
    p.initial_vz = c.initial_vz;
    p.initial_omega = c.o.initial_omega;
    p.Q = c.Q;
    p.time = m.time;
    p.dt = m.dt;
    p.QoMC = c.QoMC;
    p.stiffness = c.o.stiffness;
    if (c.correction_interval) {
      RC_TRY(ensure_bins(in, (size_t)c.n_bins));
      CUDA_TRY(cudaStreamSynchronize(in->stream)); // the pinned bin table may still be in flight
      long long start = 0;
      for (long long ib = 0; ib < c.n_bins; ib++) {
        in->h_bins[ib] = BirthBin{start, c.deficit[ib], c.area[ib], c.rmin[ib]};
        start += c.deficit[ib];
        c.distribution[ib] += c.deficit[ib];
      }
      CUDA_TRY(cudaMemcpyAsync(in->d_bins, in->h_bins, (size_t)c.n_bins * sizeof(BirthBin), cudaMemcpyHostToDevice,
                               in->stream));
      p.mode = 1;
      p.bins = in->d_bins;
      p.n_bins = (int)c.n_bins;
      in->rng_counter += (uint64_t)total;
    } else if (!c.o.discretize_radii) {
      p.mode = 0;
      in->rng_counter += (uint64_t)total;
    } else {
      p.mode = 2;
    }
    int rc;
    if (in->s32) {
      S32State &S = *in->s32;
      RC_TRY(s32_cover_charge(in, std::fabs(c.Q)));
      rc = s32_births(&in->dm, &S.f, &S.b, &p, in->cnt, &S.sc,
                      in->space_charge && S.j_state == S32_J_DEPOSITED ? 1 : 0, in->stream);
    } else {
      rc = spiffe_births64(&in->dm, &in->f, &in->b, &p, in->cnt, in->stream);
    }
    if (rc)
      return fail(SPIFFE_ERR_CUDA, "birth launch failed: %s", cudaGetErrorString((cudaError_t)rc));
    in->np_upper += total;
    in->QoMC = c.QoMC; // cathode.c:661-663
    in->stiffness = c.o.stiffness;
  }
  RC_TRY(emit_emitters(in)); // integrate.c:164-165: after the cathodes
  return 0;
}

// emit_test_particles, test_beam.c:57-104
static int emit_test(spiffe_gpu_instance *in)
{
  HostTestBeam &t = in->test_beam;
  if (t.o.electrons_per_macroparticle == 0)
    return 0;
  PhaseScope ps(in, PH_EMIT);
  const spiffe_mesh &m = in->mesh;
  if (t.start_step == -1) {
    if (m.dt <= 0)
      return fail(SPIFFE_ERR_INVALID, "integration step size is not defined (emit_test_particles)");
    t.start_step = (long long)((t.o.start_time - m.start_time) / m.dt);
    t.stop_step = (long long)((t.o.stop_time - m.start_time) / m.dt);
    in->QoMC = -SPIFFE_E_MKS / (SPIFFE_ME_MKS * SPIFFE_C_MKS);
  }
  if (!(t.start_step <= m.time_step && t.stop_step >= m.time_step))
    return 0;
  if (in->np_upper + 1 > in->capacity) {
    RC_TRY(read_counts(in));
    RC_TRY(grow_beam(in, in->h_cnt->np + 1));
  }
  BirthParams p{};
  p.total = 1;
  p.mode = SPIFFE_BIRTH_TEST;
  p.z_position = t.o.initial_z;
  p.inner_radius = t.o.initial_r;
  p.pz0 = t.o.initial_pz;
  p.pr0 = t.o.initial_pr;
  p.rpphi0 = t.o.initial_rpphi;
  p.Q = -SPIFFE_E_MKS * t.o.electrons_per_macroparticle;
  p.time = m.time;
  p.dt = m.dt;
  int rc;
  if (in->s32) {
    S32State &S = *in->s32;
    RC_TRY(s32_cover_charge(in, std::fabs(p.Q)));
    rc = s32_births(&in->dm, &S.f, &S.b, &p, in->cnt, &S.sc, 0, in->stream);
  } else {
    rc = spiffe_births64(&in->dm, &in->f, &in->b, &p, in->cnt, in->stream);
  }
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "test-beam launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  in->np_upper += 1;
  return 0;
}

extern "C" int spiffe_gpu_set_test_beam(spiffe_gpu_instance *in, const spiffe_test_beam_options *o)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  in->test_beam = HostTestBeam{};
  if (!o || o->electrons_per_macroparticle == 0)
    return 0;
  const spiffe_mesh &m = in->mesh;
  // test_beam.c:32-41
  if (o->initial_z < m.zmin || o->initial_z > m.zmax)
    return fail(SPIFFE_ERR_INVALID, "test beam initial_z is outside of simulation region");
  if (o->initial_r < 0 || o->initial_r > m.rmax)
    return fail(SPIFFE_ERR_INVALID, "test beam initial_r is outside of simulation region");
  if (o->start_time >= o->stop_time)
    return fail(SPIFFE_ERR_INVALID, "start_time >= stop_time for test beam");
  if (o->electrons_per_macroparticle < 0)
    return fail(SPIFFE_ERR_INVALID, "electrons_per_macroparticle <= 0 for test beam");
  in->test_beam.o = *o;
  return 0;
}

// process_on_axis_field_definition, onAxisFields.c:18-172, without the file
// reading: the tables are prepared on the host and copied to the device once.
extern "C" int spiffe_gpu_add_on_axis_field(spiffe_gpu_instance *in, const double *z, const double *Ez, int64_t n,
                                            double z_offset, double Ez_peak, double frequency, double phase,
                                            int32_t expansion_order)
{
  if (!in || !z || !Ez)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (Ez_peak == 0)
    return 0; // ignored, onAxisFields.c:45-49
  if (in->onaxis.size() >= SPIFFE_MAX_ON_AXIS)
    return fail(SPIFFE_ERR_UNSUPPORTED, "more than %d on-axis fields", SPIFFE_MAX_ON_AXIS);
  OnAxisProfile p;
  const std::string err = onaxis_prepare(p, z, Ez, n, z_offset, Ez_peak, frequency, phase, expansion_order);
  if (!err.empty())
    return fail(SPIFFE_ERR_INVALID, "%s", err.c_str());
  in->onaxis.push_back(std::move(p));
  size_t total = 0;
  for (const OnAxisProfile &q : in->onaxis)
    total += q.z.size();
  CUDA_TRY(cudaStreamSynchronize(in->stream)); // the old tables may still be read
  cudaFree(in->d_onaxis_data);
  cudaFree(in->d_onaxis);
  in->d_onaxis_data = nullptr;
  in->d_onaxis = nullptr;
  CUDA_TRY(cudaMalloc(&in->d_onaxis_data, 5 * total * sizeof(double)));
  CUDA_TRY(cudaMalloc(&in->d_onaxis, in->onaxis.size() * sizeof(OnAxisField)));
  std::vector<OnAxisField> views;
  double *d = in->d_onaxis_data;
  for (const OnAxisProfile &q : in->onaxis) {
    const size_t k = q.z.size();
    OnAxisField v = q.view();
    const std::vector<double> *src[5] = {&q.z, &q.Ez, &q.D1, &q.D2, &q.D3};
    const double **dst[5] = {&v.z, &v.Ez, &v.D1, &v.D2, &v.D3};
    for (int a = 0; a < 5; a++) {
      CUDA_TRY(cudaMemcpy(d, src[a]->data(), k * sizeof(double), cudaMemcpyHostToDevice));
      *dst[a] = d;
      d += k;
    }
    views.push_back(v);
  }
  CUDA_TRY(cudaMemcpy(in->d_onaxis, views.data(), views.size() * sizeof(OnAxisField), cudaMemcpyHostToDevice));
  set_devmesh(in);
  return 0;
}

// setup_translation, translate.c:21-38; the region reduction of z_lower and
// z_upper (translate.c:59-121) is the caller's to reject
extern "C" int spiffe_gpu_set_translation(spiffe_gpu_instance *in, int32_t enable, double z_trigger)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  const spiffe_mesh &m = in->mesh;
  if (enable && (z_trigger < m.zmin + m.dz || z_trigger > m.zmax - m.dz))
    return fail(SPIFFE_ERR_INVALID, "z_trigger is not in range [zmin+dz, zmax-dz]");
  if (enable && !in->d_tr_flag) {
    CUDA_TRY(cudaMalloc(&in->d_tr_flag, sizeof(int)));
    CUDA_TRY(cudaMalloc(&in->d_tr_scratch, (size_t)m.nz * in->dm.pitch * sizeof(double)));
  }
  in->tr_on = enable != 0;
  in->tr_trigger = z_trigger;
  return 0;
}

// translate_problem, translate.c:40-197 (without the region reduction):
// *translated = 1 when the problem moved by one dz
static int translate(spiffe_gpu_instance *in, int32_t *translated)
{
  if (translated)
    *translated = 0;
  if (!in->tr_on)
    return 0;
  spiffe_mesh &m = in->mesh;
  cudaStream_t s = in->stream;
  S32State *S = in->s32;
  int *h = (int *)in->h_probe;
  CUDA_TRY(cudaMemsetAsync(in->d_tr_flag, 0, sizeof(int), s));
  const int rc = S ? s32_beyond(S->b.cell, S->b.fz, in->cnt, in->np_upper, m.zmin, m.dz, in->tr_trigger, in->d_tr_flag, s)
                   : spiffe_beyond64(in->b.z, in->cnt, in->np_upper, in->tr_trigger, in->d_tr_flag, s);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "translation test launch failed");
  CUDA_TRY(cudaMemcpyAsync(h, in->d_tr_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (!*h)
    return 0;
  const int P = in->dm.pitch;
  std::vector<std::pair<void *, size_t>> rows;
  if (S) {
    const DevFields32 &F = S->f;
    if (m.modes & SPIFFE_FL_TM_FIELDS)
      rows.insert(rows.end(), {{F.Ez, 4}, {F.Jz, 8}, {F.Er, 4}, {F.Jr, 8}, {F.Bphi, 4}, {F.Bphi2, 4}});
    if (m.modes & SPIFFE_FL_TE_FIELDS)
      rows.insert(rows.end(), {{F.Ephi, 4}, {F.Jphi, 8}, {F.Br, 4}, {F.Br2, 4}, {F.Bz, 4}, {F.Bz2, 4}});
  } else {
    const DevFields<double> &F = in->f;
    if (m.modes & SPIFFE_FL_TM_FIELDS)
      rows.insert(rows.end(), {{F.Ez, 8}, {F.Jz, 8}, {F.Er, 8}, {F.Jr, 8}, {F.Bphi, 8}, {F.Bphi2, 8}});
    if (m.modes & SPIFFE_FL_TE_FIELDS)
      rows.insert(rows.end(), {{F.Ephi, 8}, {F.Jphi, 8}, {F.Br, 8}, {F.Br2, 8}, {F.Bz, 8}, {F.Bz2, 8}});
  }
  for (auto &a : rows)
    if (spiffe_rows_down(a.first, a.second * (size_t)P, m.nz, in->d_tr_scratch, s))
      return fail(SPIFFE_ERR_CUDA, "translation copy failed");
  if (S && s32_cells_down(S->b.cell, S->f.jbox, in->cnt, in->np_upper, s))
    return fail(SPIFFE_ERR_CUDA, "translation launch failed");
  // a screen's cell moves with the particles' cells (the split push finds
  // crossings by cell)
  for (int k = 0; k < in->screens.n; k++)
    in->screens.s[k].cell -= 1;
  m.zmin += m.dz;
  m.zmax += m.dz;
  in->tr_zt += m.dz;
  in->tr_trigger += m.dz;
  set_devmesh(in);
  if (translated)
    *translated = 1;
  return 0;
}

extern "C" int spiffe_gpu_translate_problem(spiffe_gpu_instance *in, int32_t *translated, double *total)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  RC_TRY(translate(in, translated));
  if (total)
    *total = in->tr_zt;
  return 0;
}

// computeMoments as the checker's SDDS stand-in defines it: mean, rms about
// zero, standard deviation with n-1 (SDDS's mdbmth, absent here)
extern "C" int spiffe_status_device(const DevMesh *m, bool split, const void *fields, const int16_t *flags,
                                    int fpitch, const void *beam, const DevCounts *cnt, double stiffness,
                                    double *scratch, double *host_out, cudaStream_t s);

// do_status_printouts, status_pr.c:18-356; kinetic_energy and field_energy,
// :358-452.  The sums run on the device in the reference's order (reduce.cu);
// only the row's values come back.
extern "C" int spiffe_gpu_status_report(spiffe_gpu_instance *in, spiffe_status_row *st)
{
  if (!in || !st)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  const spiffe_mesh &m = in->mesh;
  memset(st, 0, sizeof(*st));
  st->t = m.time;
  st->JCathode = in->cathodes.empty() ? 0 : in->cathodes[0].current_density;
  if (!in->d_status) {
    CUDA_TRY(cudaMalloc(&in->d_status, sizeof(double) * (10 * (size_t)m.nr + 64)));
  }
  CUDA_TRY(cudaMemsetAsync(in->d_status, 0, sizeof(double) * (10 * (size_t)m.nr + 64), in->stream));
  double v[4 + 23];
  int rc;
  if (in->s32)
    rc = spiffe_status_device(&in->dm, true, &in->s32->f, in->d_flags, in->dm.pitch, &in->s32->b, in->cnt,
                              in->stiffness, in->d_status, v, in->stream);
  else
    rc = spiffe_status_device(&in->dm, false, &in->f, in->d_flags, m.nr + 1, &in->b, in->cnt, in->stiffness,
                              in->d_status, v, in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "status reductions failed: %s", cudaGetErrorString((cudaError_t)rc));
  RC_TRY(read_counts(in));
  const double *b = v + 4;
  st->Particles = in->h_cnt->np;
  st->ActiveParticles = in->h_cnt->npActive;
  if (st->Particles) {
    st->Charge = b[0];
    st->SecondaryParticles = (int64_t)b[1];
    st->KineticEnergy = b[2];
    st->zAve = b[3], st->zRMS = b[4], st->zStDev = b[5];
    st->rAve = b[6], st->rRMS = b[7], st->rStDev = b[8];
    st->pzAve = b[9], st->pzRMS = b[10], st->pzStDev = b[11];
    st->prAve = b[12], st->prRMS = b[13], st->prStDev = b[14];
    st->zMin = b[15], st->zMax = b[16], st->rMin = b[17], st->rMax = b[18];
    st->pzMin = b[19], st->pzMax = b[20], st->prMin = b[21], st->prMax = b[22];
  }
  st->ElectricEnergy = v[0];
  st->MagneticEnergy = v[1];
  st->EzAbsMax = v[2];
  st->ErAbsMax = v[3];
  st->FieldEnergy = v[0] + v[1];
  st->TotalEnergy = st->KineticEnergy + st->FieldEnergy;
  st->EzOOEMin = in->h_cnt->oa_min;
  st->EzOOEMax = in->h_cnt->oa_max;
  return 0;
}

extern "C" int spiffe_gpu_on_axis_fields_at(spiffe_gpu_instance *in, double z, double r, double t, int32_t profile,
                                            double *EzErBphi)
{
  if (!in || !EzErBphi)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  EzErBphi[0] = EzErBphi[1] = EzErBphi[2] = 0;
  onaxis_eval(in->onaxis, z, r, t, profile != 0, EzErBphi[0], EzErBphi[1], EzErBphi[2]);
  return 0;
}

// Richardson-Schottky emission (cathode.c:694-706, emitter.c:424-436) with
// the reference's grouping of the products
static double schottky_density(double T, double wf, double Ez)
{
  double c = 0.012 * std::sqrt(std::fabs(Ez * 1e-5));
  if (c > wf)
    c = wf;
  return 60e4 * (T * T) * std::exp(-(wf - c) / (T * SPIFFE_KB_MKS / SPIFFE_E_MKS));
}

// fieldEmissionCurrentDensity, cathode.c:799-810
static double field_emission_density(double E, double beta, double wf)
{
  E = std::fabs(E) * beta;
  const double y = 3.79e-5 * std::sqrt(E) / wf;
  const double t = ((-0.0020 * y + 0.0131) * y + 0.1091) * y + 0.9899;
  const double v = ((0.0445 * y - 0.6782) * y - 0.4091) * y + 1.0437;
  return 1.54e-6 * (E * E) / (wf * (t * t)) * std::exp(-6.83e9 * v * std::pow(wf, 1.5) / E);
}

// set_current_density, cathode.c:673-715
static int set_current_density(spiffe_gpu_instance *in)
{
  const spiffe_mesh &m = in->mesh;
  for (HostCathode &c : in->cathodes) {
    const bool schottky = c.o.temperature > 0 && c.o.work_function;
    if (!schottky && !c.o.field_emission)
      continue;
    long iz = (long)((c.o.z_position - m.zmin) / m.dz + 1.5), ir = (long)((c.o.inner_radius + c.o.outer_radius) / 2 / m.dr);
    if (iz <= 0)
      iz = 1;
    if (iz > m.nz)
      iz = m.nz; // a cathode at zmax would probe one row past the mesh
    double Ez = m.constant_E[0];
    if ((m.modes & SPIFFE_FL_TM_FIELDS) && in->s32) {
      const size_t i = node((int)iz, (int)ir, in->dm.pitch);
      float *pf = (float *)in->h_probe;
      CUDA_TRY(cudaMemcpyAsync(pf, in->s32->f.Ez + i, sizeof(float), cudaMemcpyDeviceToHost, in->stream));
      CUDA_TRY(cudaMemcpyAsync(pf + 1, in->s32->f.EzImposed + i, sizeof(float), cudaMemcpyDeviceToHost, in->stream));
      CUDA_TRY(cudaStreamSynchronize(in->stream));
      Ez += (double)pf[0] + (double)pf[1];
    } else if (m.modes & SPIFFE_FL_TM_FIELDS) {
      const size_t i = node((int)iz, (int)ir, m.nr + 1);
      CUDA_TRY(cudaMemcpyAsync(in->h_probe, in->f.Ez + i, sizeof(double), cudaMemcpyDeviceToHost, in->stream));
      CUDA_TRY(cudaMemcpyAsync(in->h_probe + 1, in->f.EzImposed + i, sizeof(double), cudaMemcpyDeviceToHost, in->stream));
      CUDA_TRY(cudaStreamSynchronize(in->stream));
      Ez += in->h_probe[0] + in->h_probe[1];
    }
    if (!in->onaxis.empty()) {
      double dummy = 0;
      onaxis_eval(in->onaxis, c.o.z_position, (c.o.inner_radius + c.o.outer_radius) / 2.0, m.time, false, Ez, dummy,
                  dummy);
    }
    if (Ez >= 0 && c.initial_vz <= 0)
      continue;
    if (schottky) {
      if (0.012 * std::sqrt(std::fabs(Ez * 1e-5)) > c.o.work_function)
        printf("Warning: Schottky correction exceeds work function.  Set equal to work function.\n");
      c.current_density = schottky_density(c.o.temperature, c.o.work_function, Ez);
    } else {
      c.current_density = field_emission_density(Ez, c.o.field_emission_beta, c.o.work_function);
    }
  }
  return 0;
}

// The node values of Ez + EzImposed at `ez` and of Er + ErImposed at `er`
// (flat indices of the reference's layout), read on the device for the host.
template <typename T>
__global__ void k_node_sums(const T *a, const T *ai, const T *b, const T *bi, const long long *idx, int n, int pitch,
                            int P, double *out)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 2 * n)
    return;
  const long long f = idx[k];
  const size_t i = (size_t)(f / P) * (size_t)pitch + (size_t)(f % P);
  out[k] = k < n ? (double)a[i] + (double)ai[i] : (double)b[i] + (double)bi[i];
}

static int node_sums(spiffe_gpu_instance *in, const std::vector<long long> &ez, const std::vector<long long> &er,
                     std::vector<double> &Ez, std::vector<double> &Er)
{
  const size_t n = ez.size();
  Ez.assign(n, 0);
  Er.assign(n, 0);
  if (!n)
    return 0;
  if (in->nodes_cap < n) {
    cudaFree(in->d_nodes);
    cudaFree(in->d_node_vals);
    in->d_nodes = nullptr;
    in->d_node_vals = nullptr;
    in->nodes_cap = std::max<size_t>(n, 256);
    CUDA_TRY(cudaMalloc(&in->d_nodes, sizeof(long long) * 2 * in->nodes_cap));
    CUDA_TRY(cudaMalloc(&in->d_node_vals, sizeof(double) * 2 * in->nodes_cap));
  }
  std::vector<long long> idx(ez);
  idx.insert(idx.end(), er.begin(), er.end());
  CUDA_TRY(cudaMemcpyAsync(in->d_nodes, idx.data(), sizeof(long long) * 2 * n, cudaMemcpyHostToDevice, in->stream));
  const int P = in->mesh.nr + 1, blocks = (int)((2 * n + 255) / 256);
  if (in->s32) {
    const DevFields32 &f = in->s32->f;
    k_node_sums<float><<<blocks, 256, 0, in->stream>>>(f.Ez, f.EzImposed, f.Er, f.ErImposed, in->d_nodes, (int)n,
                                                       in->dm.pitch, P, in->d_node_vals);
  } else {
    const DevFields<double> &f = in->f;
    k_node_sums<double><<<blocks, 256, 0, in->stream>>>(f.Ez, f.EzImposed, f.Er, f.ErImposed, in->d_nodes, (int)n, P, P,
                                                        in->d_node_vals);
  }
  CUDA_TRY(cudaGetLastError());
  std::vector<double> v(2 * n);
  CUDA_TRY(cudaMemcpyAsync(v.data(), in->d_node_vals, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, in->stream));
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  std::copy(v.begin(), v.begin() + (long)n, Ez.begin());
  std::copy(v.begin() + (long)n, v.end(), Er.begin());
  return 0;
}

// The fields an emitter segment sees at its nodes (emitter.c:210-222,
// :405-417): constant plus (TM) node value plus on-axis expansion.
static int segment_fields(spiffe_gpu_instance *in, const HostEmitter &e, bool shifted, std::vector<double> &Ez,
                          std::vector<double> &Er)
{
  const spiffe_mesh &m = in->mesh;
  const size_t nseg = e.iz.size() - 1;
  const long long P = m.nr + 1;
  std::vector<double> a, b;
  if (m.modes & SPIFFE_FL_TM_FIELDS) {
    std::vector<long long> ez(nseg), er(nseg);
    for (size_t k = 0; k < nseg; k++) {
      ez[k] = (e.iz[k] + (shifted ? 1 : 0)) * P + e.ir[k];
      er[k] = e.iz[k] * P + e.ir[k] + (shifted ? 1 : 0);
    }
    RC_TRY(node_sums(in, ez, er, a, b));
  }
  Ez.assign(nseg, 0);
  Er.assign(nseg, 0);
  for (size_t k = 0; k < nseg; k++) {
    Ez[k] = m.constant_E[0];
    Er[k] = m.constant_E[1];
    if (m.modes & SPIFFE_FL_TM_FIELDS) {
      Ez[k] += a[k];
      Er[k] += b[k];
    }
    if (!in->onaxis.empty()) {
      double dummy = 0;
      onaxis_eval(in->onaxis, e.iz[k] * m.dz + m.zmin, e.ir[k] * m.dr, m.time, false, Ez[k], Er[k], dummy);
    }
  }
  return 0;
}

// setEmitterCurrentDensity, emitter.c:392-440
static int set_emitter_current_density(spiffe_gpu_instance *in)
{
  for (HostEmitter &e : in->emitters) {
    const size_t nseg = e.iz.size() - 1;
    e.J.assign(nseg, e.o.current_density);
    const bool schottky = e.o.temperature > 0 && e.o.work_function;
    if (!schottky && !e.o.field_emission)
      continue;
    std::vector<double> Ez, Er;
    RC_TRY(segment_fields(in, e, false, Ez, Er));
    for (size_t k = 0; k < nseg; k++)
      e.J[k] = schottky ? schottky_density(e.o.temperature, e.o.work_function, Ez[k])
                        : field_emission_density(std::sqrt(Ez[k] * Ez[k] + Er[k] * Er[k]), e.o.field_emission_beta,
                                                 e.o.work_function);
  }
  return 0;
}

static double rng2_next(spiffe_gpu_instance *in) { return spiffe_rng_uniform(in->rng2_key, ++in->rng2_counter); }

// emit_electrons_from_emitter, emitter.c:169-390: per segment, the count
// from area, current density and profile with random rounding, then each
// particle spread over the segment (random_2), offset from the surface and
// launched along its normal at initial_p; one list per emitter.
static int emit_emitters(spiffe_gpu_instance *in)
{
  const spiffe_mesh &m = in->mesh;
  for (HostEmitter &e : in->emitters) {
    if (m.dt <= 0)
      return fail(SPIFFE_ERR_INVALID, "integration step size is not defined (emit_electrons_from_emitter)");
    if (e.start_step > m.time_step || e.stop_step < m.time_step)
      continue;
    double profile_factor = 1;
    if (!e.prof_t.empty()) {
      if (m.time >= e.prof_t.front() && m.time <= e.prof_t.back())
        profile_factor = interp_table(e.prof_A, e.prof_t, m.time);
      else
        profile_factor = 0;
    }
    if (profile_factor <= 0)
      continue;
    e.start_step = (long long)((e.o.start_time - m.start_time) / m.dt);
    if (e.o.stop_time && e.o.stop_time > m.start_time)
      e.stop_step = (long long)((e.o.stop_time - m.start_time) / m.dt);
    else
      e.stop_step = 0x7fffffffffffffffLL;
    if (e.start_step > m.time_step || e.stop_step < m.time_step)
      continue;
    const size_t nseg = e.iz.size() - 1;
    std::vector<double> Ez, Er;
    if (e.o.field_emission)
      RC_TRY(segment_fields(in, e, true, Ez, Er));
    std::vector<double> col[BIRTH_LIST_COLS];
    for (size_t k = 0; k < nseg; k++) {
      const long iz = e.iz[k], ir = e.ir[k], iz1 = e.iz[k + 1], ir1 = e.ir[k + 1];
      const double z = iz * m.dz + m.zmin, r = ir * m.dr;
      double nps = 0;
      if (e.o.field_emission)
        e.J[k] = field_emission_density(std::sqrt(Ez[k] * Ez[k] + Er[k] * Er[k]), e.o.field_emission_beta,
                                        e.o.work_function);
      const bool axial = e.dir[k] == SPIFFE_EMITS_RIGHT || e.dir[k] == SPIFFE_EMITS_LEFT;
      const double area = axial ? SPIFFE_PI * ((r + m.dr) * (r + m.dr) - r * r) : SPIFFE_PIx2 * r * m.dz;
      if (area > 0 && e.o.electrons_per_macroparticle)
        nps = area * m.dt * e.J[k] / (SPIFFE_E_MKS * e.o.electrons_per_macroparticle);
      if (e.step_emission_started < 0)
        e.step_emission_started = m.time_step;
      double fnumber = nps * profile_factor;
      long total = (long)fnumber;
      fnumber -= (long)fnumber;
      if (fnumber && fnumber > rng2_next(in))
        total += 1;
      for (long q = 0; q < total; q++) {
        double pz_, pr_, vz = 0, vr = 0, zp = z, rp = r;
        if (axial) {
          const double rn = rng2_next(in);
          if (ir1 > ir)
            rp = std::sqrt(rn * ((r + m.dr) * (r + m.dr) - r * r) + r * r);
          else
            rp = std::sqrt(rn * ((r + m.dr) * (r + m.dr) - r * r) + (r - m.dr) * (r - m.dr));
          if (e.dir[k] == SPIFFE_EMITS_RIGHT) {
            vz = e.initial_v;
            zp += m.dz * e.o.offset_factor;
          } else {
            vz = -e.initial_v;
            zp -= m.dz * e.o.offset_factor;
          }
        } else {
          const double rn = rng2_next(in);
          if (iz1 > iz)
            zp = z + rn * m.dz;
          else
            zp = z - rn * m.dz;
          if (e.dir[k] == SPIFFE_EMITS_UP) {
            vr = e.initial_v;
            rp += m.dr * e.o.offset_factor;
          } else {
            vr = -e.initial_v;
            rp -= m.dr * e.o.offset_factor;
          }
        }
        const double gamma = 1 / std::sqrt(1 - (vz / SPIFFE_C_MKS) * (vz / SPIFFE_C_MKS) -
                                           (vr / SPIFFE_C_MKS) * (vr / SPIFFE_C_MKS) - 0.0);
        pz_ = vz / SPIFFE_C_MKS * gamma;
        pr_ = vr / SPIFFE_C_MKS * gamma;
        const double v[BIRTH_LIST_COLS - 1] = {zp, rp, pz_, pr_, vz, vr, e.Q, m.time, 0.0};
        for (int c = 0; c < BIRTH_LIST_COLS - 1; c++)
          col[c].push_back(v[c]);
      }
    }
    const size_t total = col[0].size();
    if (!total)
      continue;
    // particle IDs in emission order from the beam's counter (emitter.c:300)
    RC_TRY(read_counts(in));
    const long long id0 = in->h_cnt->nextParticleID;
    for (size_t q = 0; q < total; q++)
      col[BIRTH_LIST_COLS - 1].push_back((double)(id0 + (long long)q));
    RC_TRY(list_births(in, col, std::fabs(e.Q)));
    in->h_cnt->nextParticleID = id0 + (long long)total;
    CUDA_TRY(cudaMemcpyAsync(&in->cnt->nextParticleID, &in->h_cnt->nextParticleID, sizeof(long long),
                             cudaMemcpyHostToDevice, in->stream));
    CUDA_TRY(cudaStreamSynchronize(in->stream));
    in->QoMC = e.QoMC; // emitter.c:381-383
    in->stiffness = 1;
  }
  return 0;
}

// ------------------------------------------------------------ field sampling

// node reads of the sampled arrays: a[i] + (b ? b[i] : 0.0), field_sampling.c:331
__global__ void k_sample_nodes(const double *a, const double *b, const long long *idx, int n, double *out)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n)
    return;
  const long long i = idx[k];
  out[k] = a[i] + (b ? b[i] : 0.0);
}

// Room for `need` more values in the sample buffer; a larger buffer keeps
// the values not yet downloaded.
static int sample_room(spiffe_gpu_instance *in, size_t need)
{
  if (in->samples_used + need <= in->samples_cap)
    return 0;
  const size_t cap = std::max<size_t>(2 * (in->samples_used + need), 4096);
  double *p = nullptr;
  CUDA_TRY(cudaMalloc(&p, sizeof(double) * cap));
  if (in->samples_used)
    CUDA_TRY(cudaMemcpyAsync(p, in->d_samples, sizeof(double) * in->samples_used, cudaMemcpyDeviceToDevice,
                             in->stream));
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  cudaFree(in->d_samples);
  in->d_samples = p;
  in->samples_cap = cap;
  return 0;
}

static int sample_staging(spiffe_gpu_instance *in, size_t n)
{
  if (n <= in->sample_pts_cap)
    return 0;
  CUDA_TRY(cudaStreamSynchronize(in->stream)); // the old staging may still be read
  cudaFree(in->d_sample_idx);
  cudaFree(in->d_sample_pts);
  in->d_sample_idx = nullptr;
  in->d_sample_pts = nullptr;
  in->sample_pts_cap = std::max<size_t>(n, 1024);
  CUDA_TRY(cudaMalloc(&in->d_sample_idx, sizeof(long long) * in->sample_pts_cap));
  CUDA_TRY(cudaMalloc(&in->d_sample_pts, sizeof(double) * 2 * in->sample_pts_cap));
  return 0;
}

// interpolateFields at the points (z, r) on the device into a new event
static int sample_gather(spiffe_gpu_instance *in, const std::vector<double> &zr, SampleEvent &ev)
{
  const size_t n = zr.size() / 2;
  ev.gathered = true;
  ev.n = n;
  RC_TRY(sample_room(in, 6 * n));
  ev.offset = in->samples_used;
  if (!n)
    return 0;
  RC_TRY(sample_staging(in, n));
  CUDA_TRY(cudaMemcpyAsync(in->d_sample_pts, zr.data(), sizeof(double) * zr.size(), cudaMemcpyHostToDevice,
                           in->stream));
  // (pageable source: the call returns with the points copied out of `zr`;
  // the next sample's copy into the staging buffer is ordered after this
  // launch on the stream)
  double *out = in->d_samples + ev.offset;
  const int rc = in->s32 ? s32_gather_points(&in->dm, &in->s32->f, in->d_sample_pts, (int)n, 6, out, in->stream)
                         : spiffe_gather_points64(&in->dm, &in->f, in->d_sample_pts, (int)n, 6, out, in->stream);
  if (rc)
    return fail(SPIFFE_ERR_CUDA, "field sampling launch failed: %s", cudaGetErrorString((cudaError_t)rc));
  in->samples_used += 6 * n;
  return 0;
}

// node values data[iz][ir] + data1[iz][ir] at (iz, ir) pairs into a new event
static int sample_nodes(spiffe_gpu_instance *in, const double *data, const double *data1,
                        const std::vector<long long> &izir, SampleEvent &ev)
{
  const size_t n = izir.size() / 2;
  ev.gathered = false;
  ev.n = n;
  RC_TRY(sample_room(in, n));
  ev.offset = in->samples_used;
  if (!n)
    return 0;
  RC_TRY(sample_staging(in, n));
  const long long P = in->s32 ? in->dm.pitch : in->mesh.nr + 1;
  std::vector<long long> idx(n);
  for (size_t k = 0; k < n; k++)
    idx[k] = izir[2 * k] * P + izir[2 * k + 1];
  CUDA_TRY(cudaMemcpyAsync(in->d_sample_idx, idx.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, in->stream));
  k_sample_nodes<<<(unsigned)((n + 255) / 256), 256, 0, in->stream>>>(data, data1, in->d_sample_idx, (int)n,
                                                                     in->d_samples + ev.offset);
  CUDA_TRY(cudaGetLastError());
  spiffe_note_launches(1);
  in->samples_used += n;
  return 0;
}

// sample_fields, field_sampling.c:103-1097.  The reference keeps iz0, iz1,
// ir and data1 as locals of the whole call, so a definition may see what an
// earlier one of the same call left there (the r-direction time sequence
// averages over the z range and radius last set; Jz, Jr and Q add
// PsiImposed after a Phi definition); the call state below carries them the
// same way.
static int sample_fields(spiffe_gpu_instance *in)
{
  if (in->samplings.empty())
    return 0;
  const spiffe_mesh &m = in->mesh;
  const long nz = m.nz, nr = m.nr;
  const double dz = m.dz, dr = m.dr, zmin = m.zmin;
  long iz0 = 0, iz1 = 0, ir = 0, ir0 = 0, ir1 = 0, iz = 0;
  bool data1 = false;
  const double *F = nullptr, *Fimp = nullptr, *Fj[2] = {nullptr, nullptr}, *Fq = nullptr;
  if (in->s32) {
    F = in->s32->f.Psi;
    Fimp = in->s32->f.PsiImposed;
    Fq = in->s32->f.Q;
  } else {
    F = in->f.Psi;
    Fimp = in->f.PsiImposed;
    Fj[0] = in->f.Jz;
    Fj[1] = in->f.Jr;
    Fq = in->f.Q;
  }
  for (HostSampling &S : in->samplings) {
    if (S.sample_index == -1) {
      S.step_interval = (long long)(S.o.time_interval / m.dt + 0.5);
      S.start_step = (long long)((S.o.start_time - m.start_time) / m.dt + 0.5);
      S.sample_index = 0;
    }
    const int c = S.o.component;
    const double *data = nullptr;
    if (c == SPIFFE_SAMPLE_JZ)
      data = Fj[0];
    else if (c == SPIFFE_SAMPLE_JR)
      data = Fj[1];
    else if (c == SPIFFE_SAMPLE_PHI) {
      data = F;
      data1 = true;
    } else if (c == SPIFFE_SAMPLE_Q)
      data = Fq;
    if (!(m.time_step >= S.start_step &&
          (S.step_interval == 0 || (m.time_step - S.start_step) % S.step_interval == 0)))
      continue;
    const bool field = c <= SPIFFE_SAMPLE_BPHI || c == SPIFFE_SAMPLE_E || c == SPIFFE_SAMPLE_B;
    const bool zdir = S.o.direction == 0;
    SampleEvent ev;
    char pbuf[64];
    auto fixed = [&](const char *fmt, double v) { // the parameter as its header text reads back
      snprintf(pbuf, sizeof(pbuf), fmt, v);
      return std::strtod(pbuf, nullptr);
    };
    if (!S.o.time_sequence) {
      ev.t = m.time;
      std::vector<double> zr;
      std::vector<long long> nodes;
      if (field) {
        if (zdir) {
          if ((ir = (long)(S.o.position / dr)) < 0 || ir > nr - 1)
            return fail(SPIFFE_ERR_INVALID, "sampling position out of range for Ez, Er, Ephi, Bz, Br, or Bphi samples vs z");
          if ((iz0 = (long)((S.o.min_coord - zmin) / dz + 0.5)) <= 0 || iz0 > nz - 1)
            iz0 = iz0 <= 0 ? 1 : nz - 1;
          if ((iz1 = (long)((S.o.max_coord - zmin) / dz + 0.5)) <= 0 || iz1 > nz - 1)
            iz1 = iz1 <= 0 ? 1 : nz - 1;
          ev.param[0] = fixed("%21.15e", ir * dr);
          for (iz = iz0; iz <= iz1; iz++) {
            ev.x.push_back(zmin + iz * dz);
            zr.push_back(zmin + iz * dz);
            zr.push_back(ir * dr);
          }
        } else {
          iz = (long)((S.o.position - zmin) / dz + 0.5);
          if (iz <= 0 || iz > nz)
            return fail(SPIFFE_ERR_INVALID, "sampling position out of range for Ez, Er, Ephi, Bz, Br, or Bphi samples vs z");
          if ((ir0 = (long)(S.o.min_coord / dr)) < 0 || ir0 >= nr)
            ir0 = ir0 < 0 ? 0 : nr - 1;
          if ((ir1 = (long)(S.o.max_coord / dr)) < 0 || ir1 >= nr)
            ir1 = ir1 < 0 ? 0 : nr - 1;
          ev.param[0] = fixed("%21.15e", zmin + (iz - 0.5) * dz);
          for (ir = ir0; ir <= ir1; ir++) {
            ev.x.push_back(ir * dr);
            zr.push_back(zmin + iz * dz);
            zr.push_back(ir * dr);
          }
        }
        RC_TRY(sample_gather(in, zr, ev));
      } else {
        if (!data)
          return fail(SPIFFE_ERR_INVALID, "field sampling: this array is not held in this precision");
        const bool jz = c == SPIFFE_SAMPLE_JZ, jr = c == SPIFFE_SAMPLE_JR;
        if (zdir) {
          if ((ir = (long)(jr ? S.o.position / dr + 0.5 : S.o.position / dr)) < 0 || ir > nr - 1)
            return fail(SPIFFE_ERR_INVALID, jz ? "sampling position out of range for Ez/Jz/Br samples vs z"
                                            : jr ? "sampling position out of range for Er/Jr/Bz samples vs z"
                                                 : "sampling position out of range for potential/Ephi samples vs z");
          if (jz) {
            if ((iz0 = (long)((S.o.min_coord - zmin) / dz + 0.5)) <= 0 || iz0 > nz - 1)
              iz0 = iz0 <= 0 ? 1 : nz - 1;
            if ((iz1 = (long)((S.o.max_coord - zmin) / dz + 0.5)) <= 0 || iz1 > nz - 1)
              iz1 = iz1 <= 0 ? 1 : nz - 1;
          } else {
            if ((iz0 = (long)((S.o.min_coord - zmin) / dz)) < 0 || iz0 > nz - 1)
              iz0 = iz0 < 0 ? 0 : nz - 1;
            if ((iz1 = (long)((S.o.max_coord - zmin) / dz)) < 0 || iz1 > nz - 1)
              iz1 = iz1 < 0 ? 0 : nz - 1;
          }
          ev.param[0] = fixed("%21.15e", jr ? (ir - 0.5) * dr : ir * dr);
          for (iz = iz0; iz <= iz1; iz++) {
            ev.x.push_back(jz ? zmin + (iz - 0.5) * dz : zmin + iz * dz);
            nodes.push_back(iz);
            nodes.push_back(ir);
          }
        } else {
          if (jz) {
            iz = (long)((S.o.position - zmin) / dz + 0.5);
            if (iz <= 0 || iz > nz)
              return fail(SPIFFE_ERR_INVALID, "sampling position out of range for Ez/Jz/Br samples vs r");
          } else {
            iz = (long)((S.o.position - zmin) / dz);
            if (iz < 0 || iz >= nz)
              return fail(SPIFFE_ERR_INVALID, jr ? "sampling position out of range for Er/Jr/Bz samples vs r"
                                                 : "sampling position out of range for potential/Ephi samples vs r");
          }
          if (jr) {
            if ((ir0 = (long)(S.o.min_coord / dr + 0.5)) < 1 || ir0 > nr)
              ir0 = ir0 < 1 ? 1 : nr;
            if ((ir1 = (long)(S.o.max_coord / dr + 0.5)) < 1 || ir1 > nr)
              ir1 = ir1 < 1 ? 1 : nr;
          } else {
            if ((ir0 = (long)(S.o.min_coord / dr)) < 0 || ir0 >= nr)
              ir0 = ir0 < 0 ? 0 : nr - 1;
            if ((ir1 = (long)(S.o.max_coord / dr)) < 0 || ir1 >= nr)
              ir1 = ir1 < 0 ? 0 : nr - 1;
          }
          ev.param[0] = fixed("%21.15e", jz ? zmin + (iz - 0.5) * dz : zmin + iz * dz);
          for (ir = ir0; ir <= ir1; ir++) {
            ev.x.push_back(jr ? dr * (ir - 0.5) : dr * ir);
            nodes.push_back(iz);
            nodes.push_back(ir);
          }
        }
        RC_TRY(sample_nodes(in, data, data1 ? Fimp : nullptr, nodes, ev));
      }
      if (!S.initialized) {
        std::copy(ev.param, ev.param + 3, S.param);
        S.initialized = true;
      }
      S.sample_index++;
    } else {
      // time sequence: the average of the interpolated fields over the range
      if (!field || c == SPIFFE_SAMPLE_B)
        return fail(SPIFFE_ERR_UNSUPPORTED, "time-sequence samples of this component are not supported");
      ev.t = m.time_step * m.dt + m.start_time;
      std::vector<double> zr;
      if (zdir) {
        if ((ir = (long)(S.o.position / dr)) < 0 || ir > nr - 1)
          return fail(SPIFFE_ERR_INVALID, "sampling position out of range for Ez/Jz/Br time-sequence samples vs z");
        if ((iz0 = (long)((S.o.min_coord - zmin) / dz + 0.5)) < 0 || iz0 > nz - 1)
          return fail(SPIFFE_ERR_INVALID, "initial sampling coordinate out of range for Ez/Jz/Br samples vs z");
        if ((iz1 = (long)((S.o.max_coord - zmin) / dz + 0.5)) < 0 || iz1 > nz - 1)
          return fail(SPIFFE_ERR_INVALID, "final sampling coordinate out of range for Ez/Jz/Br time-sequence samples vs z");
        if (iz0 <= 0)
          iz0 = 1;
        if (iz1 <= 0)
          iz1 = 1;
        if (!S.initialized) {
          S.param[0] = fixed("%e", ir * dr);
          S.param[1] = fixed("%e", iz0 * dz + zmin);
          S.param[2] = fixed("%e", iz1 * dz + zmin);
          S.initialized = true;
          S.sample_index = 0;
        }
      } else {
        iz = (long)((S.o.position - zmin) / dz + 0.5);
        if (iz <= 0 || iz > nz)
          return fail(SPIFFE_ERR_INVALID, "sampling position out of range for Ez/Jz/Br samples vs r");
        if ((ir0 = (long)(S.o.min_coord / dr)) < 0 || ir0 >= nr)
          ir0 = ir0 < 0 ? 0 : nr - 1;
        if ((ir1 = (long)(S.o.max_coord / dr)) < 0 || ir1 >= nr)
          ir1 = ir1 < 0 ? 0 : nr - 1;
        if (!S.initialized) {
          S.param[0] = fixed("%e", iz * dz + zmin);
          S.param[1] = fixed("%e", ir0 * dr);
          S.param[2] = fixed("%e", ir1 * dr);
          S.initialized = true;
          S.sample_index = 0;
        }
      }
      // both directions average over iz0..iz1 at radius ir (field_sampling.c:756-767, :793-804)
      for (iz = iz0; iz <= iz1; iz++) {
        zr.push_back(zmin + iz * dz);
        zr.push_back(ir * dr);
      }
      ev.div = iz1 - iz0 + 1;
      RC_TRY(sample_gather(in, zr, ev));
      std::copy(S.param, S.param + 3, ev.param);
      S.sample_index++;
    }
    S.events.push_back(std::move(ev));
  }
  return 0;
}

extern "C" int spiffe_gpu_add_field_sampling(spiffe_gpu_instance *in, const spiffe_sample_options *o, int32_t *index)
{
  if (!in || !o)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  // process_sampling_definition, field_sampling.c:53-101
  if (!in->mesh.nr || !in->mesh.nz)
    return fail(SPIFFE_ERR_INVALID, "you must defined the problem geometry before specifying field sampling");
  if (o->component < 0 || o->component > SPIFFE_SAMPLE_B)
    return fail(SPIFFE_ERR_INVALID, "field component name is not recognized");
  const int c = o->component;
  if (c == SPIFFE_SAMPLE_EPHI || c == SPIFFE_SAMPLE_BPHI || c == SPIFFE_SAMPLE_BZ) { // codes 2, 5, 3
    if (!(in->mesh.modes & SPIFFE_FL_TE_FIELDS))
      return fail(SPIFFE_ERR_INVALID, "can't sample TE fields unless they are enabled in define_geometry namelist");
  } else if (!(in->mesh.modes & SPIFFE_FL_TM_FIELDS)) {
    return fail(SPIFFE_ERR_INVALID, "can't sample TM fields/potential unless they are enabled in define_geometry namelist");
  }
  if (o->direction < 0 || o->direction > 1)
    return fail(SPIFFE_ERR_INVALID, "direction name is not recognized");
  if (o->min_coord > o->max_coord)
    return fail(SPIFFE_ERR_INVALID, "min_coord > max_coord for field samples");
  if (o->time_interval <= 0)
    return fail(SPIFFE_ERR_INVALID, "time_interval <=0 for field samples");
  if (o->time_sequence && (c == SPIFFE_SAMPLE_B || c == SPIFFE_SAMPLE_JZ || c == SPIFFE_SAMPLE_JR ||
                           c == SPIFFE_SAMPLE_PHI || c == SPIFFE_SAMPLE_Q))
    return fail(SPIFFE_ERR_UNSUPPORTED, "time-sequence samples of BAll, Jz, Jr, Phi and Q are not supported");
  if (in->s32 && (c == SPIFFE_SAMPLE_JZ || c == SPIFFE_SAMPLE_JR))
    return fail(SPIFFE_ERR_UNSUPPORTED, "Jz and Jr samples are not available in the split-precision form");
  HostSampling S;
  S.o = *o;
  in->samplings.push_back(S);
  if (index)
    *index = (int32_t)in->samplings.size() - 1;
  return 0;
}

extern "C" int spiffe_gpu_sample_fields(spiffe_gpu_instance *in)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  return sample_fields(in);
}

extern "C" int spiffe_gpu_download_samples(spiffe_gpu_instance *in, int32_t index, spiffe_sample_set *h)
{
  if (!in || !h || index < 0 || (size_t)index >= in->samplings.size())
    return fail(SPIFFE_ERR_INVALID, "bad argument");
  HostSampling &S = in->samplings[(size_t)index];
  const bool seq = S.o.time_sequence != 0;
  const int ncol = S.o.component == SPIFFE_SAMPLE_E || S.o.component == SPIFFE_SAMPLE_B ? 3 : 1;
  int64_t rows = 0;
  for (const SampleEvent &ev : S.events)
    rows += seq ? 1 : (int64_t)ev.x.size();
  h->n_samples = (int64_t)S.events.size();
  h->n_rows = rows;
  if (h->max_samples == 0)
    return 0;
  if (h->n_samples > h->max_samples || rows > h->max_rows)
    return fail(SPIFFE_ERR_CAPACITY, "%lld samples of %lld rows do not fit the host buffers",
                (long long)h->n_samples, (long long)rows);
  // every value of the buffer belongs to some definition: copy it all once
  std::vector<double> v(in->samples_used);
  if (!v.empty()) {
    CUDA_TRY(cudaMemcpyAsync(v.data(), in->d_samples, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, in->stream));
    CUDA_TRY(cudaStreamSynchronize(in->stream));
  }
  // which of interpolateFields' outputs (Ez, Er, Ephi, Bz, Br, Bphi) a column
  // takes (field_sampling.c:233-246, :1035-1088): fieldValue[component]
  int pick[3] = {S.o.component, 0, 0};
  if (S.o.component == SPIFFE_SAMPLE_E)
    pick[0] = 0, pick[1] = 1, pick[2] = 2;
  else if (S.o.component == SPIFFE_SAMPLE_B)
    pick[0] = 3, pick[1] = 4, pick[2] = 5;
  int64_t r = 0;
  for (size_t k = 0; k < S.events.size(); k++) {
    const SampleEvent &ev = S.events[k];
    h->t[k] = ev.t;
    for (int q = 0; q < 3; q++)
      h->param[3 * k + q] = ev.param[q];
    const double *src = v.data() + ev.offset;
    if (seq) {
      double sum[6] = {0, 0, 0, 0, 0, 0};
      for (size_t i = 0; i < ev.n; i++)
        for (int q = 0; q < 6; q++)
          sum[q] += src[6 * i + q];
      h->rows[k] = 1;
      h->x[r] = ev.t;
      for (int q = 0; q < ncol; q++)
        if (h->v[q])
          h->v[q][r] = sum[pick[q]] / (double)ev.div;
      r++;
    } else {
      h->rows[k] = (int64_t)ev.x.size();
      for (size_t i = 0; i < ev.x.size(); i++, r++) {
        h->x[r] = ev.x[i];
        for (int q = 0; q < ncol; q++)
          if (h->v[q])
            h->v[q][r] = ev.gathered ? src[6 * i + pick[q]] : src[i];
      }
    }
  }
  S.events.clear();
  // the buffer empties once no definition holds samples in it
  bool any = false;
  for (const HostSampling &o : in->samplings)
    any = any || !o.events.empty();
  if (!any)
    in->samples_used = 0;
  return 0;
}

extern "C" int spiffe_gpu_add_emitter(spiffe_gpu_instance *in, const spiffe_emitter_options *o)
{
  if (!in || !o)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  // process_emitter_definition, emitter.c:40-167
  if (!o->field_emission && o->current_density <= 0 && o->electrons_per_macroparticle == 0 && o->temperature <= 0)
    return fail(SPIFFE_ERR_INVALID, "either field_emission, current_density, electrons_per_macroparticle, or "
                                    "temperature must be non-zero");
  if (o->current_density < 0)
    return fail(SPIFFE_ERR_INVALID, "the current density should be a positive quantity");
  if (o->electrons_per_macroparticle < 0)
    return fail(SPIFFE_ERR_INVALID, "electrons_per_macroparticle should be a positive quantity");
  if (o->temperature < 0)
    return fail(SPIFFE_ERR_INVALID, "temperature should be a positive quantity");
  if (o->stop_time && o->start_time > o->stop_time)
    return fail(SPIFFE_ERR_INVALID, "stop_time is non-zero and less than start_time");
  if (o->n_points <= 0 || !o->iz || !o->ir || !o->direction)
    return fail(SPIFFE_ERR_INVALID, "No surface elements found with the specified material ID");
  if (o->electrons_per_macroparticle == 0)
    return fail(SPIFFE_ERR_INVALID, "electrons_per_macroparticle must be nonzero");
  HostEmitter e;
  e.o = *o;
  e.iz.assign(o->iz, o->iz + o->n_points);
  e.ir.assign(o->ir, o->ir + o->n_points);
  e.dir.assign(o->direction, o->direction + o->n_points);
  for (int64_t k = 0; k < o->n_points; k++)
    if (e.iz[(size_t)k] < 0 || e.iz[(size_t)k] > in->mesh.nz || e.ir[(size_t)k] < 0 || e.ir[(size_t)k] > in->mesh.nr)
      return fail(SPIFFE_ERR_INVALID, "emitter boundary point outside the mesh");
  if (o->n_profile > 0) {
    e.prof_t.assign(o->profile_t, o->profile_t + o->n_profile);
    e.prof_A.assign(o->profile_A, o->profile_A + o->n_profile);
    for (size_t i = 1; i < e.prof_t.size(); i++)
      if (e.prof_t[i - 1] >= e.prof_t[i])
        return fail(SPIFFE_ERR_INVALID, "profile data is not ordered by increasing time values");
  }
  e.o.iz = e.o.ir = nullptr;
  e.o.direction = nullptr;
  e.o.profile_t = e.o.profile_A = nullptr;
  e.initial_v = std::fabs(o->initial_p / std::sqrt(1 + o->initial_p * o->initial_p) * SPIFFE_C_MKS);
  e.Q = -SPIFFE_E_MKS * o->electrons_per_macroparticle;
  e.QoMC = -SPIFFE_E_MKS / (SPIFFE_ME_MKS * SPIFFE_C_MKS);
  e.J.assign(e.iz.size() > 1 ? e.iz.size() - 1 : 0, o->current_density);
  const long long seed = o->random_number_seed < 0 ? -(long long)o->random_number_seed : o->random_number_seed;
  in->rng2_key = spiffe_rng_key2((uint64_t)seed); // random_2(-abs(seed)), emitter.c:63
  in->rng2_counter = 0;
  in->emitters.push_back(std::move(e));
  return 0;
}

extern "C" int spiffe_gpu_add_antenna(spiffe_gpu_instance *in, int32_t direction, int64_t istart, int64_t iend,
                                      int64_t iposition, double current, double frequency, double phase,
                                      const double *t, const double *W, int64_t n)
{
  if (!in || !t || !W)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (n <= 2)
    return fail(SPIFFE_ERR_INVALID, "SDDS waveform file empty or invalid");
  if (frequency <= 0)
    return fail(SPIFFE_ERR_INVALID, "antenna frequency <= 0");
  if (direction < 0 || direction > 2 || (direction == 2 && !(in->mesh.modes & SPIFFE_FL_TE_FIELDS)))
    return fail(SPIFFE_ERR_INVALID, "bad antenna direction");
  const long lim_a = direction == 1 ? in->mesh.nr : in->mesh.nz, lim_b = direction == 1 ? in->mesh.nz : in->mesh.nr;
  if (istart < 0 || iend > lim_a || iposition < 0 || iposition > lim_b)
    return fail(SPIFFE_ERR_INVALID, "antenna indices out of range");
  for (int64_t i = 1; i < n; i++)
    if (t[i - 1] >= t[i])
      return fail(SPIFFE_ERR_INVALID, "waveform data is not ordered by increasing time index");
  HostAntenna a;
  a.direction = direction;
  a.istart = (long)istart;
  a.iend = (long)iend;
  a.iposition = (long)iposition;
  a.current = current;
  a.frequency = frequency;
  a.phase = phase;
  a.t.assign(t, t + n);
  a.W.assign(W, W + n);
  in->antennas.push_back(std::move(a));
  return 0;
}

// add_antenna_excitation, antenna.c:374-418
static int antennas(spiffe_gpu_instance *in, double time)
{
  for (HostAntenna &a : in->antennas) {
    const long n_pts = (long)a.t.size();
    double J;
    if (time <= a.t[0])
      J = a.W[0];
    else if (time > a.t[n_pts - 1] || a.last_index >= (n_pts - 1))
      J = a.W[n_pts - 1];
    else {
      long i = a.last_index;
      while (i < n_pts - 2 && time >= a.t[i + 1])
        i++;
      a.last_index = i;
      J = (a.W[i + 1] - a.W[i]) / (a.t[i + 1] - a.t[i]) * (time - a.t[i]) + a.W[i];
    }
    J *= a.current * std::sin(SPIFFE_PIx2 * a.frequency * time + a.phase);
    int rc;
    if (in->s32) {
      const DevFields32 &F = in->s32->f;
      long long *arr = a.direction == 0 ? F.Jz : (a.direction == 1 ? F.Jr : F.Jphi);
      rc = s32_antenna(arr, F.jbox, in->dm.pitch, a.direction, a.istart, a.iend, a.iposition, J, in->s32->sc.qJ, in->stream);
    } else {
      double *arr = a.direction == 0 ? in->f.Jz : (a.direction == 1 ? in->f.Jr : in->f.Jphi);
      rc = spiffe_antenna64(arr, in->dm.pitch, a.direction, a.istart, a.iend, a.iposition, J, in->stream);
    }
    if (rc)
      return fail(SPIFFE_ERR_CUDA, "antenna launch failed");
  }
  return 0;
}

extern "C" int spiffe_gpu_configure_run(spiffe_gpu_instance *in, int32_t space_charge, const spiffe_push_options *push,
                                        const spiffe_poisson_options *pc)
{
  if (!in || !push)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  in->space_charge = space_charge;
  in->push = *push;
  if (pc)
    in->pc = *pc;
  else
    memset(&in->pc, 0, sizeof(in->pc));
  if (space_charge)
    in->mesh.modes |= SPIFFE_FL_SPACE_CHARGE;
  set_devmesh(in);
  // the solver's set-up (for the split form the multigrid hierarchy, built
  // on the host in about 0.2 s for a 2.5M-node mesh) belongs to the
  // configuration, not to the first step that corrects
  if (pc && pc->maximum_iterations > 0 && pc->step_interval > 0)
    RC_TRY(in->s32 ? s32_ensure_poisson(in) : ensure_poisson(in));
  return 0;
}

// setup before the loop, integrate.c:125-133
extern "C" int spiffe_gpu_run_begin(spiffe_gpu_instance *in, spiffe_poisson_report *rep)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  RC_TRY(imposed_efield(in, &in->pc, 1));
  const int ran = poisson_correction(in, in->space_charge, &in->pc);
  if (ran < 0)
    return ran;
  if (rep) {
    memset(rep, 0, sizeof(*rep));
    if (ran)
      RC_TRY(in->s32 ? s32_poisson_report(&in->s32->pcw, rep, in->stream)
                     : spiffe_poisson64_report(&in->pcw, rep, in->stream));
  }
  RC_TRY(set_current_density(in));
  RC_TRY(set_emitter_current_density(in));
  return 0;
}

// The perform_integration loop body, integrate.c:136-193.
extern "C" int spiffe_gpu_run_steps(spiffe_gpu_instance *in, int64_t n_steps)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  spiffe_mesh &m = in->mesh;
  for (int64_t k = 0; k < n_steps; k++) {
    if (m.imposed_ramp_time > 0)
      RC_TRY(imposed_efield(in, &in->pc, 0));
    m.time = m.time_step * m.dt + m.start_time;
    RC_TRY(sample_fields(in)); // integrate.c:149
    RC_TRY(emit(in));
    RC_TRY(emit_test(in));
    S32State *S = in->s32;
    if (!S) {
      RC_TRY(spiffe_gpu_zero_current_arrays(in));
      if (in->space_charge)
        RC_TRY(spiffe_gpu_add_particle_currents(in));
    } else if (!(in->space_charge && S->j_state == S32_J_DEPOSITED)) {
      // J holds the previous push's deposit only when that push ran inside this loop
      if (S->j_state != S32_J_ZERO)
        RC_TRY(s32_zero_j(in));
      if (in->space_charge) {
        RC_TRY(s32_deposit_all(in));
        S->j_state = S32_J_DEPOSITED;
      }
    }
    RC_TRY(antennas(in, m.time + m.dt / 2));
    const int ran = poisson_correction(in, in->space_charge, &in->pc);
    if (ran < 0)
      return ran;
    if (!S) {
      RC_TRY(spiffe_gpu_advance_field_solutions(in));
      RC_TRY(spiffe_gpu_advance_particles(in, &in->push));
    } else {
      // particles by cell before the push, every sort_interval steps and on
      // the first step after an upload
      if (S->sort_interval > 0 && S->since_sort >= S->sort_interval) {
        S->since_sort = 0;
        PhaseScope ps(in, PH_PUSH);
        RC_TRY(s32_sort(&in->dm, &S->b, in->cnt, in->np_upper, &S->pw, in->stream));
      }
      RC_TRY(s32_fdtd(in, 1)); // reads J and leaves it zero
      RC_TRY(s32_push_step(in, &in->push, in->space_charge)); // deposits J for the next step
      if (!in->space_charge)
        S->j_state = S32_J_ZERO;
      S->since_sort++;
    }
    RC_TRY(translate(in, nullptr));
    RC_TRY(set_current_density(in));
    RC_TRY(set_emitter_current_density(in));
    m.time_step++;
  }
  return 0;
}

extern "C" int spiffe_gpu_synchronize(spiffe_gpu_instance *in)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  RC_TRY(read_counts(in));
  return 0;
}

extern "C" int spiffe_gpu_counts(spiffe_gpu_instance *in, int64_t *np, int64_t *np_active)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  RC_TRY(read_counts(in));
  if (np)
    *np = in->h_cnt->np;
  if (np_active)
    *np_active = in->h_cnt->npActive;
  return 0;
}

extern "C" int spiffe_gpu_counts_async(spiffe_gpu_instance *in, int64_t *out)
{
  if (!in || !out)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  static_assert(offsetof(DevCounts, npActive) == offsetof(DevCounts, np) + sizeof(long long), "np, npActive adjacent");
  CUDA_TRY(cudaMemcpyAsync(out, &in->cnt->np, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, in->stream));
  return 0;
}

// ------------------------------------------------------------ measurement

extern "C" int spiffe_gpu_select_device(int32_t device)
{
  CUDA_TRY(cudaSetDevice(device));
  return 0;
}

extern "C" int spiffe_gpu_stream(spiffe_gpu_instance *in, void **stream)
{
  if (!in || !stream)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  *stream = (void *)in->stream;
  return 0;
}

extern "C" int spiffe_gpu_set_profiling(spiffe_gpu_instance *in, int32_t on)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  in->timer.on = on != 0;
  for (int p = 0; p < PH_COUNT; p++)
    in->timer.used[p] = 0;
  return 0;
}

// Per-phase device time since profiling was (re)started: emission, deposit,
// Poisson correction, FDTD, push.  Synchronises the stream and restarts.
extern "C" int spiffe_gpu_phase_times(spiffe_gpu_instance *in, double *ms, int64_t *count)
{
  if (!in || !ms || !count)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  CUDA_TRY(cudaStreamSynchronize(in->stream));
  for (int p = 0; p < PH_COUNT; p++) {
    double total = 0;
    for (size_t k = 0; k < in->timer.used[p]; k++) {
      float e = 0;
      CUDA_TRY(cudaEventElapsedTime(&e, in->timer.pool[p][k].first, in->timer.pool[p][k].second));
      total += e;
    }
    ms[p] = total;
    count[p] = (int64_t)in->timer.used[p];
    in->timer.used[p] = 0;
  }
  return 0;
}

// Split-precision form: reorder the particles by cell every n steps of the
// integration loop (0: never).
extern "C" int spiffe_gpu_set_sort_interval(spiffe_gpu_instance *in, int64_t n)
{
  if (!in || n < 0)
    return fail(SPIFFE_ERR_INVALID, "bad argument");
  if (in->s32) {
    in->s32->sort_interval = n;
    in->s32->since_sort = n; // the next step sorts
  }
  return 0;
}

extern "C" int spiffe_gpu_set_poisson_solver(spiffe_gpu_instance *in, int32_t solver)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (solver != SPIFFE_POISSON_SOR && solver != SPIFFE_POISSON_MULTIGRID)
    return fail(SPIFFE_ERR_INVALID, "unknown Poisson solver %d", (int)solver);
  if (!in->s32)
    return solver == SPIFFE_POISSON_SOR ? 0
                                        : fail(SPIFFE_ERR_UNSUPPORTED, "the FP64 form solves with the reference's SOR");
  in->s32->pcw.solver = solver;
  return 0;
}

extern "C" int spiffe_gpu_set_fdtd_kernel(spiffe_gpu_instance *in, int32_t kernel)
{
  if (!in)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  if (kernel != SPIFFE_FDTD_AUTO && kernel != SPIFFE_FDTD_TWO_KERNELS && kernel != SPIFFE_FDTD_FUSED)
    return fail(SPIFFE_ERR_INVALID, "unknown FDTD kernel choice %d", (int)kernel);
  if (!in->s32)
    return kernel == SPIFFE_FDTD_AUTO ? 0 : fail(SPIFFE_ERR_UNSUPPORTED, "the FP64 form has one FDTD path");
  in->s32->fdtd_mode = kernel;
  in->s32->fdtd.fused = -1; // planned again at the next step
  return 0;
}

// Work done so far: [0] particle-steps (active particles summed over pushes),
// [1] SOR half-sweeps, [2] Poisson solves, [3] FDTD steps, [4] V-cycles.
extern "C" int spiffe_gpu_work_counters(spiffe_gpu_instance *in, int64_t *out)
{
  if (!in || !out)
    return fail(SPIFFE_ERR_INVALID, "null argument");
  RC_TRY(read_counts(in));
  out[0] = in->h_cnt->pushed;
  out[1] = in->h_cnt->sor_halfsweeps;
  out[2] = in->h_cnt->sor_solves;
  out[3] = in->fdtd_steps;
  out[4] = in->h_cnt->mg_cycles;
  return 0;
}
