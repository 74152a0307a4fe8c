// spiffe_b200/csrc/common.cuh -- device-side data model shared by all kernels.
//
// One problem ("instance") lives on the device as contiguous (nz+1)x(nr+1)
// arrays, ir fastest, at row pitch `pitch` elements.  The plain FP64 form uses
// pitch = nr+1 (the reference's zarray_2d rows, spiffe.h:60-71); the
// single-precision form pads rows to a multiple of 32 elements so every row
// starts on a 128-byte boundary.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/spiffe_b200_constants.h"
#include "../../include/spiffe_b200_types.h"

// Per-instance scalars every kernel needs (the FIELDS scalars of spiffe.h).
#define SPIFFE_MAX_ON_AXIS 8

// One on-axis RF field (ON_AXIS_FIELD, spiffe.h): Ez(z) on increasing z and
// its first three z-derivatives, n points; k = omega / c.
struct OnAxisField {
  const double *z, *Ez, *D1, *D2, *D3;
  int n, order;
  double k;
};

struct DevMesh {
  int nz, nr, pitch;
  double zmin, zmax, rmax, dz, dr, dt;
  int lower_bc, upper_bc, right_bc, left_bc;
  unsigned modes;
  double constE[3], constB[3];
  short turn_off[6];
  int has_solenoid;
  // on-axis fields (add_on_axis_fields) and, for the push being launched,
  // sin(omega t + phase) and omega/c^2 cos(omega t + phase) of each
  int n_onaxis;
  const OnAxisField *onaxis;
  double oa_sin[SPIFFE_MAX_ON_AXIS], oa_bf[SPIFFE_MAX_ON_AXIS];
  double *oa_ext; // DevCounts' (oa_min, oa_max): the push's extremes of the summed on-axis Ez
};

// addOffAxisExpansionFields (onAxisFields.c:208-268) at (z, r): each of
// the n fields expanded off axis to its order and added into Ez, Er, Bphi;
// sin_wt[i] = sin(omega t + phase) and bf[i] = omega / c^2 cos(omega t +
// phase) of field i.  The position search follows binaryArraySearch in
// bracket mode (-1 below the first point, n-1 at or past the last, else the
// last point at or below z).  As in the reference, each field that covers z
// sets Er to zero before adding its own terms.
__host__ __device__ inline void onaxis_expand(const OnAxisField *fields, int n_fields, const double *sin_wt,
                                              const double *bf, double z, double r, double &Ez, double &Er, double &Bphi,
                                              double *lo = nullptr, double *hi = nullptr)
{
  for (int ip = 0; ip < n_fields; ip++) {
    const OnAxisField &F = fields[ip];
    int iz;
    if (z < F.z[0])
      iz = -1;
    else if (z >= F.z[F.n - 1])
      iz = F.n - 1;
    else {
      int lo = 0, hi = F.n - 1;
      while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (z >= F.z[mid])
          lo = mid;
        else
          hi = mid;
      }
      iz = lo;
    }
    if (iz < 0 || iz >= F.n - 1)
      continue;
    if (!(F.z[iz] <= z && F.z[iz + 1] > z))
      continue;
    const double s = sin_wt[ip], BF = bf[ip], k = F.k;
    const double dz = z - F.z[iz];
    const double Ez0 = F.Ez[iz] + F.D1[iz] * dz;
    Ez += Ez0 * s;
    Er = 0;
    if (F.order >= 1) {
      const double DzEz = F.D1[iz] + F.D2[iz] * dz;
      Er += -r / 2 * DzEz * s;
      Bphi += r / 2 * Ez0 * BF;
      if (F.order >= 2) {
        const double Dz2Ez = F.D2[iz] + F.D3[iz] * dz;
        Ez += -(r * r) / 4. * (Dz2Ez + k * k * Ez0) * s;
        if (F.order >= 3) {
          Er += (r * r * r) / 16. * (F.D3[iz] + k * k * DzEz) * s;
          Bphi += (r * r * r) / 16. * (Dz2Ez + k * k * Ez0) * BF;
        }
      }
    }
    if (lo) { // EzMin, EzMax (onAxisFields.c:262-265)
      if (*lo > Ez)
        *lo = Ez;
      if (*hi < Ez)
        *hi = Ez;
    }
  }
}

__device__ inline void atomic_min_f64(double *a, double v)
{
  unsigned long long *p = (unsigned long long *)a, old = *p;
  while (__longlong_as_double((long long)old) > v) {
    const unsigned long long seen = atomicCAS(p, old, (unsigned long long)__double_as_longlong(v));
    if (seen == old)
      break;
    old = seen;
  }
}

__device__ inline void atomic_max_f64(double *a, double v)
{
  unsigned long long *p = (unsigned long long *)a, old = *p;
  while (__longlong_as_double((long long)old) < v) {
    const unsigned long long seen = atomicCAS(p, old, (unsigned long long)__double_as_longlong(v));
    if (seen == old)
      break;
    old = seen;
  }
}

// The on-axis fields' contribution at a particle, summed apart and then added
// (advance_particles.c:836-844).
__device__ __forceinline__ void onaxis_add(const DevMesh &m, double z, double r, double &Ez, double &Er, double &Bphi)
{
  double EzO = 0, ErO = 0, BphiO = 0, lo = INFINITY, hi = -INFINITY;
  onaxis_expand(m.onaxis, m.n_onaxis, m.oa_sin, m.oa_bf, z, r, EzO, ErO, BphiO, &lo, &hi);
  if (lo <= hi) {
    atomic_min_f64(m.oa_ext, lo);
    atomic_max_f64(m.oa_ext + 1, hi);
  }
  Ez += EzO;
  Er += ErO;
  Bphi += BphiO;
}

template <typename T>
struct DevFields {
  const int16_t *flags;
  T *Ez, *Er, *Bphi, *Bphi2, *Jz, *Jr;
  T *Ephi, *Jphi, *Br, *Br2, *Bz, *Bz2;
  T *EzImposed, *ErImposed, *PsiImposed, *BzImposed, *BrImposed;
  T *Psi, *Q;
};

// FP64 structure-of-arrays beam (BEAM, spiffe.h:201-221).
struct DevBeam64 {
  double *z, *r, *pz, *pr, *r_pphi, *vz, *vr, *vphi, *Q;
  double *r0, *z0, *t0, *rmin, *rmax, *zmin, *zmax;
  int32_t *particleID;
  int16_t *generation;
  uint64_t *status;
  int64_t capacity;
};

// Screen record buffers, one set per screen (SCREEN, spiffe.h:341-352).
struct DevScreen {
  double z_position;
  int direction;
  int cell; // floor((z_position - zmin)/dz): a crossing starts or ends in a cell range containing it
  int64_t capacity;
  double *col[SPIFFE_SCREEN_QUANS];
  double *rmin, *rmax, *zmin, *zmax;
  int16_t *generation;
  int32_t *particleID;
  long long *order; // (time step << 32) | particle index: the reference's record order (advance_particles.c:362-434)
};

struct DevScreens {
  int n;
  long long step; // the push's time step
  DevScreen s[SPIFFE_MAX_SCREENS];
};

// Counters kept on the device so a step needs no host round trip.
struct DevCounts {
  long long np, npActive;
  long long nextParticleID;
  long long first_lost; // smallest lost index this step (reference compaction)
  long long n_lost;     // particles lost this step
  long long new_active; // activations this step
  long long screen_nb[SPIFFE_MAX_SCREENS];
  long long screen_overflow;
  double last_pz0, last_pr0, last_rpphi0; // pre-kick momenta of particle np-1
  long long pushed;                       // sum over pushes of the active count (particle-steps)
  double oa_min, oa_max;                  // EzOOEMin, EzOOEMax of the last push (advance_particles.c:113-114)
  long long sor_halfsweeps, sor_solves;   // red-black half-sweeps and Poisson solves run (either solver)
  long long mg_cycles;                    // multigrid V-cycles run
  unsigned int error;                     // SPIFFE_DEV_ERR_* bits
  unsigned int pad;
};

// One particle lost in a push, with what the loss epilogue of
// advance_particles (advance_particles.c:437-487) computes from it: the
// point and direction where its path left the mesh's open region
// (findLossCoordinates, below), its momentum magnitude, the pushed momenta,
// the birth position, the charge, id and generation, and the particle's
// index and the step, which order the records as the reference writes them.
struct LostRecord {
  double t, zLost, rLost, p, pz, pr, r0, z0, q;
  long long ip, step;
  int32_t id;
  int16_t gen, code; // code -1: a split-form row whose values are still to be formed (cell0, fz0, fr0, neg)
  int32_t cell0, neg;
  float fz0, fr0;
};

// Where a push appends its lost particles (rec null: not recorded).
struct LostLog {
  LostRecord *rec;
  unsigned long long *n;
  long long cap, step;
};

#ifdef __CUDACC__
__device__ __forceinline__ void lost_append(const LostLog &L, const LostRecord &r)
{
  const unsigned long long k = atomicAdd(L.n, 1ull);
  if ((long long)k < L.cap)
    L.rec[k] = r;
}
#endif

// findLossCoordinates (secondaryEmission.c:239-352): the point where the
// straight path from (z0, r0) to (z1, r1) leaves its cell through the face
// it crossed, and that face's direction code (1 left, 2 right, 3 up, 4
// down; 1 also when the particle did not move).  flags at pitch fpitch.
#define SPIFFE_GOING_LEFT 1
#define SPIFFE_GOING_RIGHT 2
#define SPIFFE_GOING_UP 3
#define SPIFFE_GOING_DOWN 4
__host__ __device__ inline int find_loss_coordinates(double zmin, double zmax, double dz, double dr, long nr,
                                                     const int16_t *flags, long fpitch, double z0, double r0,
                                                     double z1, double r1, double *zr, double *rr)
{
  const long iz0 = (long)((z0 - zmin) / dz), ir0 = (long)(r0 / dr);
  const long iz1 = z1 < zmin ? -1 : (long)((z1 - zmin) / dz);
  const long ir1 = r1 < 0 ? -1 : (long)(r1 / dr);
  auto metal = [&](long iz, long ir) { return (flags[iz * fpitch + ir] & SPIFFE_FL_IS_METAL) != 0; };
  int code = 0;
  if (r0 == r1 && z0 == z1) {
    *zr = z0;
    *rr = r0;
    return 1;
  }
  if (ir0 == ir1)
    code = iz0 > iz1 ? SPIFFE_GOING_LEFT : SPIFFE_GOING_RIGHT;
  else if (iz0 == iz1)
    code = ir0 > ir1 ? SPIFFE_GOING_DOWN : SPIFFE_GOING_UP;
  else if (z1 < z0) {
    if (z1 < 0)
      code = SPIFFE_GOING_LEFT;
    else if (ir0 != ir1) {
      if (ir1 >= 0 && ir1 < nr && metal(iz0, ir1))
        code = SPIFFE_GOING_LEFT;
      else if (ir1 < 0 && metal(iz0, -ir1))
        code = SPIFFE_GOING_LEFT;
    } else if (ir0 == ir1 && (ir0 < nr - 1 && metal(iz0, ir0 + 1)))
      code = SPIFFE_GOING_LEFT;
    else
      code = r1 < r0 ? SPIFFE_GOING_DOWN : SPIFFE_GOING_UP;
  } else if (z1 > z0) {
    if (z1 > zmax)
      code = SPIFFE_GOING_RIGHT;
    else if (ir0 != ir1) {
      if (ir1 >= 0 && ir1 < nr && metal(iz1, ir1))
        code = SPIFFE_GOING_RIGHT;
      else if (ir1 < 0 && metal(iz1, -ir1))
        code = SPIFFE_GOING_RIGHT;
    } else if (ir0 == ir1 && (ir0 < nr - 1 && metal(iz1, ir0 + 1)))
      code = SPIFFE_GOING_RIGHT;
    else
      code = r1 < r0 ? SPIFFE_GOING_DOWN : SPIFFE_GOING_UP;
  } else
    code = r1 < r0 ? SPIFFE_GOING_DOWN : SPIFFE_GOING_UP;
  double zm, rm;
  if (code == SPIFFE_GOING_LEFT) {
    zm = ((long)((z0 - zmin) / dz)) * dz + zmin + dz * 1e-12;
    rm = (r1 - r0) / (z1 - z0) * (zm - z0) + r0;
  } else if (code == SPIFFE_GOING_RIGHT) {
    zm = ((long)((z0 - zmin) / dz)) * dz + zmin + dz * (1 - 1e-12);
    rm = (r1 - r0) / (z1 - z0) * (zm - z0) + r0;
  } else if (code == SPIFFE_GOING_DOWN) {
    rm = ((long)(r0 / dr)) * dr + dr * 1e-12;
    zm = (z1 - z0) / (r1 - r0) * (rm - r0) + z0;
  } else {
    rm = ((long)(r0 / dr)) * dr + dr * (1 - 1e-12);
    zm = (z1 - z0) / (r1 - r0) * (rm - r0) + z0;
  }
  *zr = zm;
  *rr = fabs(rm);
  return code;
}

#define SPIFFE_DEV_ERR_CAPACITY 1u
#define SPIFFE_DEV_ERR_SCREEN 2u
#define SPIFFE_DEV_ERR_BARRIER 4u
#define SPIFFE_DEV_ERR_INDEX 8u
#define SPIFFE_DEV_ERR_WAIT 16u // a bounded wait inside a persistent kernel ran out

__host__ __device__ inline size_t node(int iz, int ir, int pitch) { return (size_t)iz * (size_t)pitch + (size_t)ir; }

#ifdef __CUDACC__
// signed 64-bit atomic add through the unsigned overload (two's complement)
__device__ __forceinline__ long long atomic_add_ll(long long *p, long long v)
{
  return (long long)atomicAdd((unsigned long long *)p, (unsigned long long)v);
}
#endif

// Host-side launch helpers.
inline unsigned blocks_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// Every host wrapper reports the kernels it queued (a process-wide count the
// benchmark reads around its timed region).
extern "C" void spiffe_note_launches(int n);
