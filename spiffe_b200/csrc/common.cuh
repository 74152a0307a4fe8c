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
};

struct DevScreens {
  int n;
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

#define SPIFFE_DEV_ERR_CAPACITY 1u
#define SPIFFE_DEV_ERR_SCREEN 2u
#define SPIFFE_DEV_ERR_BARRIER 4u
#define SPIFFE_DEV_ERR_INDEX 8u

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
