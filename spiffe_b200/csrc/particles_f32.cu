// spiffe_b200/csrc/particles_f32.cu -- particle kernels of the split-precision form.
//
// The push restates advance_particles' per-particle loop (advance_particles.c:
// 131-339) and screen loop (:362-434), the gather restates interpolateFields
// (:622-890) and the deposition restates add_particle_currents
// (space_charge.c:34-295), on the split representation of split32.cuh:
// a position is an integer cell plus an FP32 offset in [0,1), so the
// reference's (z-zmin)/dz and r/dr are iz+fz and ir+fr exactly and every
// stencil index is an integer shift of the cell.  Arithmetic is FP32 except
// for screen records, activation bookkeeping and the time, which are FP64.
//
// Inside the integration loop the push also deposits the pushed particles'
// current for the next step (the reference deposits at the start of the
// next step from exactly these positions and velocities).  Contributions are
// fixed-point integers; lanes of a warp that hit the same node are grouped
// with __match_any_sync and summed with __reduce_add_sync before one 64-bit
// atomic per node, so a warp of cell-sorted particles issues one atomic
// where it would issue 32, and the total is exact whatever the order.
#include "split32.cuh"
#include "modules.cuh"

#include "../../include/spiffe_b200_rng.h"

#include <cfloat>

#include <cub/block/block_radix_sort.cuh>

namespace {

constexpr int T = 256;
constexpr float C_F = (float)SPIFFE_C_MKS;

// (ξ + off) for ξ = i + f, f in [0,1), off in {0, 0.5, 1}: the reference's
// (long) truncation toward zero and the remainder, which is negative when
// ξ + off is negative (positions outside the mesh)
__device__ __forceinline__ void shift(int i, float f, float off, int &idx, float &frac)
{
  if (off == 0.f) {
    idx = i;
    frac = f;
  } else if (off == 1.f) {
    idx = i + 1;
    frac = f;
  } else {
    const float t = f + 0.5f;
    const int k = t >= 1.f ? 1 : 0;
    idx = i + k;
    frac = t - (float)k;
  }
  if (idx < 0 && frac > 0.f) {
    idx += 1;
    frac -= 1.f;
  }
}

// checkLossCode, advance_particles.c:31-65
__device__ int loss_code32(const DevMesh &m, const int16_t *__restrict__ fl, int iz, int ir)
{
  const int P = m.pitch;
  const int16_t f0 = __ldg(fl + iz * P + ir);
  if (f0 & SPIFFE_FL_IS_INSIDE)
    return 3;
  if (f0 & SPIFFE_FL_IS_SURFACE) {
    if (iz + 1 > m.nz)
      return 4;
    if (ir + 1 > m.nr)
      return 5;
    if (__ldg(fl + (iz + 1) * P + ir + 1) & SPIFFE_FL_IS_METAL && __ldg(fl + iz * P + ir + 1) & SPIFFE_FL_IS_METAL &&
        __ldg(fl + (iz + 1) * P + ir) & SPIFFE_FL_IS_METAL)
      return 6;
  }
  return 0;
}

// interpolateFields (advance_particles.c:622-890) at ξz = iz+fz, ξr = ir+fr.
// E = Ez, Er, Ephi, Bz, Br, Bphi.
// DEF: the default field modes (TM fields, longitudinal and radial
// interpolation, no TE, no switches), chosen on the host, so the mode tests
// fold away.
template <bool DEF>
__device__ void gather32(const DevMesh &m, const DevFields32 &f, int iz0, float fz, int ir0, float fr, float *E)
{
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  const bool longit = DEF || (m.modes & SPIFFE_FL_LONGIT_INTERP), radial = DEF || (m.modes & SPIFFE_FL_RADIAL_INTERP);
  const bool tm = DEF || (m.modes & SPIFFE_FL_TM_FIELDS), te = !DEF && (m.modes & SPIFFE_FL_TE_FIELDS);
  const uint8_t *__restrict__ um = f.umask;
  const bool r_nonzero = ir0 != 0 || fr != 0.f;
  const int16_t *__restrict__ fl = f.flags;
  int iz, ir, iz1, ir1;
  float wr, wl, wa, wb;
  float Ez = 0, Er = 0, Ephi = 0, Bz = 0, Br = 0, Bphi = 0;
  // 32-bit node offsets (a mesh holds fewer than 2^31 nodes) and read-only loads
#define N(a, b) ((a) * P + (b))
#define LD(arr, i) __ldg((arr) + (i))
  // Ez and Br (:649-710)
  if (longit) {
    shift(iz0, fz, 0.5f, iz, wr);
    wl = 1 - wr;
  } else {
    iz = iz0 + 1;
    wl = 1;
    wr = 0;
  }
  if (radial) {
    shift(ir0, fr, 0.f, ir, wa);
    wb = 1 - wa;
  } else {
    float t;
    shift(ir0, fr, 0.5f, ir, t);
    wa = 0;
    wb = 1;
  }
  if (iz >= 0 && iz < nz && ir >= 0 && ir < nr) {
    if ((iz1 = iz + 1) >= nz)
      iz1 = iz;
    if ((ir1 = ir + 1) >= nr)
      ir1 = ir;
    if (LD(um, N(iz, ir)) & S32_U_CLEAN) {
      // no metal near this cell
    } else if (LD(fl, N(iz, ir + 1)) & SPIFFE_FL_ER_ZERO && LD(fl, N(iz, ir)) & SPIFFE_FL_ER_ZERO) {
      if (iz > 0 && (LD(fl, N(iz - 1, ir)) || LD(fl, N(iz - 1, ir + 1))))
        iz = iz1;
      else
        iz1 = iz;
    } else if (LD(fl, N(iz1, ir + 1)) & SPIFFE_FL_ER_ZERO && LD(fl, N(iz1, ir)) & SPIFFE_FL_ER_ZERO) {
      iz1 = iz;
    }
    if (tm)
      Ez = wb * (wl * (LD(f.Ez, N(iz, ir)) + LD(f.EzImposed, N(iz, ir))) + wr * (LD(f.Ez, N(iz1, ir)) + LD(f.EzImposed, N(iz1, ir)))) +
           wa * (wl * (LD(f.Ez, N(iz, ir1)) + LD(f.EzImposed, N(iz, ir1))) + wr * (LD(f.Ez, N(iz1, ir1)) + LD(f.EzImposed, N(iz1, ir1))));
    if (r_nonzero && te)
      Br = wb * (wl * LD(f.Br2, N(iz, ir)) + wr * LD(f.Br2, N(iz1, ir))) + wa * (wl * LD(f.Br2, N(iz, ir1)) + wr * LD(f.Br2, N(iz1, ir1)));
  }
  // Er and Bz (:713-752)
  if (longit) {
    shift(iz0, fz, 0.f, iz, wr);
    wl = 1 - wr;
  } else {
    float t;
    shift(iz0, fz, 0.5f, iz, t);
    wr = 0;
    wl = 1;
  }
  if (radial) {
    shift(ir0, fr, 0.5f, ir, wa);
    wb = 1 - wa;
  } else {
    ir = ir0 + 1;
    wa = 0;
    wb = 1;
  }
  if (iz >= 0 && iz < nz && ir >= 0) {
    if (ir >= nr)
      ir = nr - 1;
    iz1 = iz + 1;
    ir1 = ir + 1;
    if (LD(um, N(iz, ir)) & S32_U_CLEAN) {
      // no metal near this cell
    } else if (LD(fl, N(iz + 1, ir)) & SPIFFE_FL_EZ_ZERO && LD(fl, N(iz, ir)) & SPIFFE_FL_EZ_ZERO)
      ir = ir1;
    else if (LD(fl, N(iz + 1, ir + 1)) & SPIFFE_FL_EZ_ZERO && LD(fl, N(iz, ir + 1)) & SPIFFE_FL_EZ_ZERO)
      ir1 = ir;
    if (r_nonzero && tm)
      Er = wl * (wb * (LD(f.Er, N(iz, ir)) + LD(f.ErImposed, N(iz, ir))) + wa * (LD(f.Er, N(iz, ir1)) + LD(f.ErImposed, N(iz, ir1)))) +
           wr * (wb * (LD(f.Er, N(iz1, ir)) + LD(f.ErImposed, N(iz1, ir))) + wa * (LD(f.Er, N(iz1, ir1)) + LD(f.ErImposed, N(iz1, ir1))));
    if (te)
      Bz = wl * (wb * LD(f.Bz2, N(iz, ir)) + wa * LD(f.Bz2, N(iz, ir1))) + wr * (wb * LD(f.Bz2, N(iz1, ir)) + wa * LD(f.Bz2, N(iz1, ir1)));
  }
  // Ephi (:754-786)
  if (te && r_nonzero) {
    if (longit) {
      shift(iz0, fz, 0.f, iz, wr);
      wl = 1 - wr;
    } else {
      float t;
      shift(iz0, fz, 0.5f, iz, t);
      wr = 0;
      wl = 1;
    }
    if (radial) {
      shift(ir0, fr, 0.f, ir, wa);
      wb = 1 - wa;
    } else {
      float t;
      shift(ir0, fr, 0.5f, ir, t);
      wa = 0;
      wb = 1;
    }
    if (iz >= 0 && iz < nz && ir >= 0 && ir < nr) {
      if ((iz1 = iz + 1) >= nz)
        iz1 = iz;
      if ((ir1 = ir + 1) >= nr)
        ir1 = ir;
      Ephi = wl * wb * LD(f.Ephi, N(iz, ir)) + wr * wb * LD(f.Ephi, N(iz1, ir)) + wl * wa * LD(f.Ephi, N(iz, ir1)) +
             wr * wa * LD(f.Ephi, N(iz1, ir1));
    }
  }
  // Bphi at the E time level (:788-825)
  if (tm) {
    if (longit) {
      shift(iz0, fz, 0.5f, iz, wr);
      wl = 1 - wr;
    } else {
      iz = iz0 + 1;
      wr = 0;
      wl = 1;
    }
    if (radial) {
      shift(ir0, fr, 0.5f, ir, wa);
      wb = 1 - wa;
    } else {
      ir = ir0 + 1;
      wa = 0;
      wb = 1;
    }
    if (r_nonzero && iz >= 0 && iz < nz) {
      if ((iz1 = iz + 1) >= nz)
        iz1 = iz;
      if (ir >= nr)
        ir = nr - 1;
      if ((ir1 = ir + 1) >= nr)
        ir1 = ir;
      Bphi = wl * wb * LD(f.Bphi2, N(iz, ir)) + wr * wb * LD(f.Bphi2, N(iz1, ir)) + wa * wl * LD(f.Bphi2, N(iz, ir1)) +
             wr * wa * LD(f.Bphi2, N(iz1, ir1));
    }
  }
  // uniform fields, the on-axis expansion and switches (:828-857)
  Ez += (float)m.constE[0];
  Er += (float)m.constE[1];
  Ephi += (float)m.constE[2];
  Bz += (float)m.constB[0];
  Br += (float)m.constB[1];
  Bphi += (float)m.constB[2];
  if (!DEF && m.n_onaxis) {
    double ez = 0, er = 0, bp = 0;
    onaxis_add(m, m.zmin + ((double)iz0 + fz) * m.dz, ((double)ir0 + fr) * m.dr, ez, er, bp);
    Ez += (float)ez;
    Er += (float)er;
    Bphi += (float)bp;
  }
  if (!DEF) {
    if (m.turn_off[0]) Ez = 0;
    if (m.turn_off[1]) Er = 0;
    if (m.turn_off[2]) Ephi = 0;
    if (m.turn_off[3]) Bz = 0;
    if (m.turn_off[4]) Br = 0;
    if (m.turn_off[5]) Bphi = 0;
  }
  // solenoid fields on nodes (:859-875)
  if (m.has_solenoid) {
    shift(iz0, fz, 0.f, iz, wr);
    shift(ir0, fr, 0.f, ir, wa);
    if (ir >= 0 && iz >= 0 && ir < nr && iz < nz) {
      wb = 1 - wa;
      wl = 1 - wr;
      Bz += wl * (wb * LD(f.BzImposed, N(iz, ir)) + wa * LD(f.BzImposed, N(iz, ir + 1))) +
            wr * (wb * LD(f.BzImposed, N(iz + 1, ir)) + wa * LD(f.BzImposed, N(iz + 1, ir + 1)));
      Br += wl * (wb * LD(f.BrImposed, N(iz, ir)) + wa * LD(f.BrImposed, N(iz, ir + 1))) +
            wr * (wb * LD(f.BrImposed, N(iz + 1, ir)) + wa * LD(f.BrImposed, N(iz + 1, ir + 1)));
    }
  }
#undef N
#undef LD
  E[0] = Ez;
  E[1] = Er;
  E[2] = Ephi;
  E[3] = Bz;
  E[4] = Br;
  E[5] = Bphi;
}

// ---- current contributions (space_charge.c:34-295) in fixed-point quanta.
// qvg = (v/c) Q 2^38/q_ref.  Four fixed slots: (iz,ir), (iz+1,ir) with
// longitudinal smearing, (iz,ir+1) with radial smearing, (iz+1,ir+1) with
// both; node -1 = nothing (fixed slots keep the arrays in registers).
struct Contrib32 {
  int node[4];
  long long q[4];
};

__device__ __forceinline__ void put(Contrib32 &c, int k, int nd, float v)
{
  c.node[k] = nd;
  c.q[k] = __float2ll_rn(v);
}

// component 0 Jz, 1 Jr, 2 Jphi
template <bool DEF>
__device__ void contrib32(const DevMesh &m, int comp, int iz0, float fz, int ir0, float fr, float qvg, Contrib32 &c)
{
  c.node[0] = c.node[1] = c.node[2] = c.node[3] = -1;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  const bool rsm = !DEF && (m.modes & SPIFFE_FL_RADIAL_SMEAR), lsm = !DEF && (m.modes & SPIFFE_FL_LONGIT_SMEAR);
  int iz, ir;
  float rfrac, zfrac;
  // radial index and fraction
  if (comp == 1)
    shift(ir0, fr, rsm ? 0.5f : 1.f, ir, rfrac);
  else
    shift(ir0, fr, rsm ? 0.f : 0.5f, ir, rfrac);
  // longitudinal index and fraction
  if (comp == 0)
    shift(iz0, fz, lsm ? 0.5f : 1.f, iz, zfrac);
  else
    shift(iz0, fz, lsm ? 0.f : 0.5f, iz, zfrac);
  if (iz < 0 || iz > nz || ir < 0 || ir > nr || (comp == 1 && ir >= nr))
    return;
  float fm, fp, Jm, Jp;
  if (rsm) {
    fp = rfrac;
    fm = 1 - fp;
  } else {
    fm = 1;
    fp = 0;
  }
  if (comp == 1) {
    if (ir == 0) {
      Jm = 0;
      Jp = qvg;
    } else if (ir < nr - 1) {
      Jm = __fdividef(fm * qvg, (float)(2 * ir - 1));
      Jp = __fdividef(fp * qvg, (float)(2 * ir + 1));
    } else {
      Jm = 0;
      ir--;
      Jp = __fdividef(qvg, (float)(2 * ir + 1));
    }
  } else {
    if (ir == 0) {
      Jm = 4 * fm * qvg;
      Jp = fp * qvg * 0.5f;
    } else if (ir < nr - 1) {
      Jm = __fdividef(fm * qvg, (float)(2 * ir));
      Jp = __fdividef(fp * qvg, (float)(2 * ir + 2));
    } else {
      Jm = 0;
      Jp = __fdividef(fp * qvg, (float)(2 * ir));
      ir--;
    }
  }
  if (lsm) {
    if (comp == 0 && iz == 0) {
      fp = 1;
      fm = 0;
    } else if ((comp != 2 && iz == nz) || (comp == 2 && iz == nz - 1)) {
      fm = 1;
      fp = 0;
    } else {
      fp = zfrac;
      fm = 1 - fp;
    }
  } else {
    fm = 1;
    fp = 0;
  }
  // row iz+1 exists only for iz < nz; at iz == nz its weight is zero
  const bool next_row = lsm && iz < nz;
  put(c, 0, (int)node(iz, ir, P), fm * Jm);
  if (next_row)
    put(c, 1, (int)node(iz + 1, ir, P), fp * Jm);
  if (rsm) {
    put(c, 2, (int)node(iz, ir + 1, P), fm * Jp);
    if (next_row)
      put(c, 3, (int)node(iz + 1, ir + 1, P), fp * Jp);
  }
}

// Warp-aggregated fixed-point add: lanes with the same node sum their values
// (biased to 43 non-negative bits and split 22/21 so __reduce_add_sync's
// 32-bit sums cannot overflow) and the group's lowest lane adds the total.
// Every lane of the warp must call this (node -1 = nothing to add).
__device__ __forceinline__ void warp_add(long long *J, int nd, long long v)
{
  // cell-sorted particles: a warp's lanes usually share the node, and one
  // vote settles that without the node-matching step
  const int nd0 = __shfl_sync(0xffffffffu, nd, 0);
  const unsigned grp = __all_sync(0xffffffffu, nd == nd0) ? 0xffffffffu : __match_any_sync(0xffffffffu, nd);
  const unsigned long long biased = (unsigned long long)(v + (1LL << 42));
  const unsigned lo = (unsigned)(biased & ((1u << 22) - 1)), hi = (unsigned)(biased >> 22);
  const unsigned slo = __reduce_add_sync(grp, lo), shi = __reduce_add_sync(grp, hi);
  const int lane = threadIdx.x & 31;
  if (nd >= 0 && lane == __ffs(grp) - 1) {
    const long long tot = ((long long)shi << 22) + (long long)slo - (long long)__popc(grp) * (1LL << 42);
    if (tot)
      atomic_add_ll(J + nd, tot);
  }
}

// Deposits the three components of one particle (or nothing, when !on);
// called by every lane of the warp.
template <bool DEF>
__device__ void deposit_particle(const DevMesh &m, const DevFields32 &f, bool on, int iz, float fz, int ir, float fr,
                                 float bz, float br, float bphi, float qs)
{
  const bool lsm = !DEF && (m.modes & SPIFFE_FL_LONGIT_SMEAR), rsm = !DEF && (m.modes & SPIFFE_FL_RADIAL_SMEAR);
  const bool tm = DEF || (m.modes & SPIFFE_FL_TM_FIELDS), te = !DEF && (m.modes & SPIFFE_FL_TE_FIELDS);
  Contrib32 c;
  unsigned lo = 0xffffffffu, hi = 0u; // node indices this lane adds to
  for (int comp = 0; comp < 3; comp++) {
    if ((comp < 2 && !tm) || (comp == 2 && !te))
      continue;
    if (on)
      contrib32<DEF>(m, comp, iz, fz, ir, fr, (comp == 0 ? bz : comp == 1 ? br : bphi) * qs, c);
    else
      c.node[0] = c.node[1] = c.node[2] = c.node[3] = -1;
    long long *J = comp == 0 ? f.Jz : comp == 1 ? f.Jr : f.Jphi;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      // the same slots are live in every lane (the smearing flags are per mesh)
      if ((k == 1 && !lsm) || (k == 2 && !rsm) || (k == 3 && !(lsm && rsm)))
        continue;
      warp_add(J, c.node[k], c.node[k] >= 0 ? c.q[k] : 0);
      if (c.node[k] >= 0) {
        lo = min(lo, (unsigned)c.node[k]);
        hi = max(hi, (unsigned)c.node[k]);
      }
    }
  }
  // widen the box of rows holding current (the FDTD reads and clears only
  // those rows); a warp skips the atomics when the box already covers it
  lo = __reduce_min_sync(0xffffffffu, lo);
  hi = __reduce_max_sync(0xffffffffu, hi);
  if ((threadIdx.x & 31) == 0 && lo <= hi) {
    const int rlo = (int)(lo / (unsigned)m.pitch), rhi = (int)(hi / (unsigned)m.pitch);
    if (rlo < f.jbox[0])
      atomicMin(f.jbox, rlo);
    if (rhi > f.jbox[1])
      atomicMax(f.jbox + 1, rhi);
  }
}

// v/c of a particle from its momenta at radius r (setParticleVelocities, :605-620)
__device__ __forceinline__ void betas(float pz, float pr, float rpp, float r, float &bz, float &br, float &bphi)
{
  const float pphi = r != 0.f ? rpp * __frcp_rn(r) : 0.f;
  const float ig = rsqrtf(pz * pz + pr * pr + pphi * pphi + 1.f); // 1/gamma
  bphi = pphi * ig;
  bz = pz * ig;
  br = pr * ig;
}

__global__ void __launch_bounds__(T) k_deposit32(DevMesh m, DevFields32 f, DevBeam32 b, const DevCounts *cnt,
                                                  S32Scales sc)
{
  const long ip = (long)blockIdx.x * T + threadIdx.x;
  const bool on = ip < (long)cnt->np && (b.status[ip] & S32_ACTIVE);
  int iz = 0, ir = 0;
  float fz = 0, fr = 0, bz = 0, br = 0, bphi = 0, qs = 0;
  if (on) {
    const int32_t cl = b.cell[ip];
    iz = s32_iz(cl);
    ir = s32_ir(cl);
    fz = b.fz[ip];
    fr = b.fr[ip];
    betas(b.pz[ip], b.pr[ip], b.rpphi[ip], ((float)ir + fr) * (float)m.dr, bz, br, bphi);
    qs = b.Q[ip] * sc.s_charge;
  }
  deposit_particle<false>(m, f, on, iz, fz, ir, fr, bz, br, bphi, qs);
}

struct ScreenCtx {
  int momentum_policy;
};

__device__ void record32(const DevScreen &s, long long step, long long *nb, long long *overflow, const DevBeam32 &b,
                         long ip, const double *q, float zmn, float zmx, float rmn, float rmx)
{
  const long long k = atomic_add_ll(nb, 1LL);
  if (k >= s.capacity) {
    atomic_add_ll(overflow, 1LL);
    return;
  }
  s.order[k] = (step << 32) | (long long)ip;
  for (int c = 0; c < SPIFFE_SCREEN_QUANS; c++)
    s.col[c][k] = q[c];
  s.rmin[k] = rmn == FLT_MAX ? DBL_MAX : (double)rmn;
  s.rmax[k] = rmx == -FLT_MAX ? -DBL_MAX : (double)rmx;
  s.zmin[k] = zmn == FLT_MAX ? DBL_MAX : (double)zmn;
  s.zmax[k] = zmx == -FLT_MAX ? -DBL_MAX : (double)zmx;
  s.generation[k] = b.generation[ip];
  s.particleID[k] = b.particleID[ip];
}

__global__ void k_snapshot_last32(DevBeam32 b, DevCounts *cnt)
{
  const long long np = cnt->np;
  if (np > 0) {
    cnt->last_pz0 = b.pz[np - 1];
    cnt->last_pr0 = b.pr[np - 1];
    cnt->last_rpphi0 = b.rpphi[np - 1];
  }
}

// advance_particles (:131-339) and its screen loop (:362-434); with DEP the
// pushed particle's current for the next step.
template <bool DEP, bool DEF>
__global__ void __launch_bounds__(T, 5) k_push32(DevMesh m, DevFields32 f, DevBeam32 b, Push32Params p, DevScreens scr,
                                               DevCounts *cnt, int32_t *lost_list, S32Scales sc)
{
  const long ip = (long)blockIdx.x * T + threadIdx.x;
  const long np = (long)cnt->np;
  const bool valid = ip < np;
  const int nz = m.nz, nr = m.nr;
  const float dr = (float)m.dr, dz = (float)m.dz;
  bool dep_on = false;
  int d_iz = 0, d_ir = 0;
  float d_fz = 0, d_fr = 0, d_bz = 0, d_br = 0, d_bphi = 0, d_qs = 0;
  if (valid) {
    const int16_t *fl = f.flags;
    const int32_t cl = b.cell[ip];
    const int iz0 = s32_iz(cl), ir0 = s32_ir(cl);
    const float fz0 = b.fz[ip], fr0 = b.fr[ip];
    uint8_t status = b.status[ip];
    float pz = b.pz[ip], pr = b.pr[ip], rpp = b.rpphi[ip];
    const float pz0 = pz, pr0 = pr, rpp0 = rpp;
    float zmx = b.zmax[ip], zmn = b.zmin[ip], rmx = b.rmax[ip], rmn = b.rmin[ip];
    unsigned moved = 0; // extrema that changed: bit 0 zmax, 1 zmin, 2 rmax, 3 rmin
    const float zmin = (float)m.zmin;
    // position before the drift and the stored (old) velocities
    const float zo = zmin + ((float)iz0 + fz0) * dz, ro = ((float)ir0 + fr0) * dr;
    if (zo > zmx) { zmx = zo; moved |= 1u; }
    if (zo < zmn) { zmn = zo; moved |= 2u; }
    if (ro > rmx) { rmx = ro; moved |= 4u; }
    if (ro < rmn) { rmn = ro; moved |= 8u; }
    float bz, br, bphi;
    betas(pz, pr, rpp, ro, bz, br, bphi);
    // drift with the old velocities (:157-158)
    float t = fz0 + bz * (C_F * p.dt_dz);
    int k = (int)floorf(t);
    int iz = iz0 + k;
    float fz = t - (float)k;
    if (fz >= 1.f) {
      fz -= 1.f;
      iz++;
    }
    t = fr0 + br * (C_F * p.dt_dr);
    k = (int)floorf(t);
    int irs = ir0 + k; // signed radial cell: r < 0 when irs < 0
    float frs = t - (float)k;
    if (frs >= 1.f) {
      frs -= 1.f;
      irs++;
    }
    // |r| / dr split (the loss tests index with fabs(r), :219-220)
    int ir = irs;
    float fr = frs;
    const bool r_negative = irs < 0;
    if (r_negative) {
      if (frs > 0.f) {
        ir = -irs - 1;
        fr = 1.f - frs;
      } else {
        ir = -irs;
        fr = 0.f;
      }
    }
    float adjust = 1.f;
    // FP64 positions, formed only where a rare branch needs them
    auto zd_of = [&]() { return m.zmin + ((double)iz + fz) * m.dz; };
    auto z0d_of = [&]() { return m.zmin + ((double)iz0 + fz0) * m.dz; };
    // zmax = zmin + (nz-1) dz and rmax = (nr-1) dr (geometry.c:75-76)
    const bool above_zmin = iz >= 0, below_zmax = iz < nz - 1 || (iz == nz - 1 && fz == 0.f);
    const bool r_le_rmax = r_negative || irs < nr - 1 || (irs == nr - 1 && frs == 0.f);
    if (!(status & S32_ACTIVE)) {
      // activation on entering the mesh (:167-189)
      if (above_zmin && below_zmax && r_le_rmax && ir <= nr && !loss_code32(m, fl, iz, ir)) {
        status |= S32_ACTIVE;
        atomic_add_ll(&cnt->new_active, 1LL);
        b.t0[ip] = p.time;
        b.r0[ip] = ((double)ir0 + fr0) * m.dr;
        b.z0[ip] = z0d_of();
        const float dxi = ((float)(iz - iz0) + (fz - fz0));
        if (iz > 0 && loss_code32(m, fl, iz - 1, ir))
          adjust = fz / dxi;
        else
          adjust = ((float)iz + fz) / dxi;
        if (adjust > 1.f)
          adjust = 1.f;
      }
    }
    if (p.zfs_on) {
      const double zd = zd_of(), z0d = z0d_of();
      if (z0d < p.z_forces_start) {
        if (zd < p.z_forces_start)
          adjust = 0.f;
        else
          adjust = (float)((zd - p.z_forces_start) / (zd - z0d));
      }
    }
    const bool active = status & S32_ACTIVE;
    bool lost = false;
    // loss tests (:211-236)
    if (active && (!above_zmin || !below_zmax || !r_le_rmax))
      lost = true;
    if (!lost && active) {
      if (iz > nz || ir > nr || iz < 0 || ir < 0)
        lost = true;
      else if (loss_code32(m, fl, iz, ir))
        lost = true;
    }
    if (r_negative)
      pr = -pr;
    const float r = ((float)ir + fr) * dr;
    if (!lost && active) {
      const float zn = zmin + ((float)iz + fz) * dz;
      if (zn > zmx) { zmx = zn; moved |= 1u; }
      if (zn < zmn) { zmn = zn; moved |= 2u; }
      if (r > rmx) { rmx = r; moved |= 4u; }
      if (r < rmn) { rmn = r; moved |= 8u; }
    }
    if (DEF || !p.forced) {
      // momentum kick with the old velocities (:270-287)
      float E[6];
      if (active)
        gather32<DEF>(m, f, iz, fz, ir, fr, E);
      else
        E[0] = E[1] = E[2] = E[3] = E[4] = E[5] = 0.f;
      const float ir_ = r != 0.f ? __frcp_rn(r) : 0.f;
      const float pphi = rpp * ir_;
      const float ig = rsqrtf(pr * pr + pz * pz + pphi * pphi + 1.f); // 1/gamma
      const float vz = C_F * bz, vr = C_F * br, vphi = C_F * bphi;
      const float a = adjust * p.stiff_inv;
      pr += a * (p.dt * (pphi * pphi * C_F * ig * ir_) + p.QoMC_dt * (E[1] + vphi * E[3] - vz * E[5]));
      pz += a * p.QoMC_dt * (E[0] + vr * E[5] - vphi * E[4]);
      rpp += a * p.QoMC_dt * r * (E[2] + vz * E[4] - vr * E[3]);
    } else {
      // forced test-beam acceleration (:289-311)
      const float ir_ = r != 0.f ? __frcp_rn(r) : 0.f;
      const float pphi = rpp * ir_;
      const float ig = rsqrtf(pr * pr + pz * pz + pphi * pphi + 1.f);
      pr += p.dt * (pphi * pphi * C_F * ig * ir_);
      if (zd_of() <= p.tb_z_decel)
        pz += p.tb_z_force_dt;
      else {
        pz -= p.tb_z_force_dt;
        if (pz < 0.f)
          pz = 0.f;
      }
      if (r_negative)
        pr = 0.f;
      else if ((double)r <= p.tb_r_decel)
        pr += p.tb_r_force_dt;
      else
        pr -= p.tb_r_force_dt;
    }
    b.cell[ip] = s32_cell(iz, ir);
    b.fz[ip] = fz;
    b.fr[ip] = fr;
    b.pz[ip] = pz;
    b.pr[ip] = pr;
    b.rpphi[ip] = rpp;
    // extrema change rarely except the leading one: store only what moved
    if (moved & 1u)
      b.zmax[ip] = zmx;
    if (moved & 2u)
      b.zmin[ip] = zmn;
    if (moved & 4u)
      b.rmax[ip] = rmx;
    if (moved & 8u)
      b.rmin[ip] = rmn;
    if (lost) {
      status &= ~S32_ACTIVE;
      status |= S32_LOST;
      const long long slot = atomic_add_ll(&cnt->n_lost, 1LL);
      atomicMin(&cnt->first_lost, (long long)ip);
      if (lost_list)
        lost_list[slot] = (int32_t)ip;
      if (p.lost.rec) { // the cell before the drift; k_lost32 forms the row after the push
        LostRecord rec{};
        rec.t = p.time;
        rec.ip = ip;
        rec.step = p.lost.step;
        rec.code = -1;
        rec.cell0 = s32_cell(iz0, ir0);
        rec.fz0 = fz0;
        rec.fr0 = fr0;
        rec.neg = r_negative;
        lost_append(p.lost, rec);
      }
    }
    b.status[ip] = status;
    if (iz < -32767 || iz > 32767)
      atomicOr(&cnt->error, SPIFFE_DEV_ERR_INDEX);

    // screen crossings (:362-434), in FP64
    // a crossing needs the screen's cell between the old and new cells
    bool near_screen = false;
    for (int is = 0; is < scr.n; is++)
      near_screen |= min(iz0, iz) <= scr.s[is].cell && scr.s[is].cell <= max(iz0, iz);
    if (near_screen) {
      const double zd = zd_of(), z0d = z0d_of();
      const bool ref = p.screen_momentum == SPIFFE_SCREEN_REFERENCE;
      const double pz0s = ref ? cnt->last_pz0 : pz0, pr0s = ref ? cnt->last_pr0 : pr0;
      const double rpp0s = ref ? cnt->last_rpphi0 : rpp0;
      const double dt = m.dt, vzd = SPIFFE_C_MKS * (double)bz, vrd = SPIFFE_C_MKS * (double)br;
      const double rd = ((double)ir + fr) * m.dr;
      double r0 = ((double)ir0 + fr0) * m.dr, q[SPIFFE_SCREEN_QUANS];
      for (int is = 0; is < scr.n; is++) {
        const DevScreen &s = scr.s[is];
        if (s.z_position <= zd && s.z_position > z0d && s.direction == 1) {
          const double dtp = (s.z_position - z0d) / vzd;
          const double pphi_new = rd ? rpp / rd : 0;
          const double pphi0 = r0 ? rpp0s / r0 : 0;
          q[0] = r0 + vrd * dtp;
          q[1] = pz0s + ((double)pz - pz0s) / dt * dtp;
          q[2] = pr0s + ((double)pr - pr0s) / dt * dtp;
          q[3] = pphi0 + (pphi_new - pphi0) / dt * dtp;
          q[4] = (p.time - dt + dtp);
          q[5] = b.Q[ip];
          q[6] = b.r0[ip];
          q[7] = b.t0[ip];
          record32(s, scr.step, &cnt->screen_nb[is], &cnt->screen_overflow, b, ip, q, zmn, zmx, rmn, rmx);
        } else if (s.z_position >= zd && s.z_position < z0d && s.direction == -1) {
          const double dtp = (s.z_position - z0d) / vzd;
          r0 += vrd * dtp;
          q[0] = r0;
          q[1] = pz;
          q[2] = pr;
          q[3] = r0 ? rpp / r0 : 0;
          q[4] = (p.time - dt + dtp);
          q[5] = b.Q[ip];
          q[6] = b.r0[ip];
          q[7] = b.t0[ip];
          record32(s, scr.step, &cnt->screen_nb[is], &cnt->screen_overflow, b, ip, q, zmn, zmx, rmn, rmx);
        }
      }
    }
    if (DEP && (status & S32_ACTIVE)) {
      dep_on = true;
      d_iz = iz;
      d_ir = ir;
      d_fz = fz;
      d_fr = fr;
      betas(pz, pr, rpp, r, d_bz, d_br, d_bphi);
      d_qs = b.Q[ip] * sc.s_charge;
    }
  }
  if (DEP)
    deposit_particle<DEF>(m, f, dep_on, d_iz, d_fz, d_ir, d_fr, d_bz, d_br, d_bphi, d_qs);
}

// The loss epilogue of advance_particles (:437-487) for the rows this push
// recorded, before the compaction moves the lost particles: the momentum,
// the loss point (findLossCoordinates) from the positions before and after
// the drift, in FP64.
__global__ void k_lost32(DevMesh m, const int16_t *fl, DevBeam32 b, LostLog L)
{
  const unsigned long long n = *L.n;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L.cap || (unsigned long long)k >= n)
    return;
  LostRecord &r = L.rec[k];
  if (r.code != -1)
    return;
  const long ip = (long)r.ip;
  const int32_t c = b.cell[ip];
  const double rd = ((double)s32_ir(c) + (double)b.fr[ip]) * m.dr, pz = b.pz[ip], pr = b.pr[ip];
  const double rpp = b.rpphi[ip];
  double pm = pz * pz + pr * pr;
  if (rd)
    pm += (rpp / rd) * (rpp / rd);
  r.p = sqrt(pm);
  r.pz = pz;
  r.pr = pr;
  r.r0 = b.r0[ip];
  r.z0 = b.z0[ip];
  r.q = b.Q[ip];
  r.id = b.particleID[ip];
  r.gen = b.generation[ip];
  const double z0 = m.zmin + ((double)s32_iz(r.cell0) + (double)r.fz0) * m.dz;
  const double r0 = ((double)s32_ir(r.cell0) + (double)r.fr0) * m.dr;
  const double z1 = m.zmin + ((double)s32_iz(c) + (double)b.fz[ip]) * m.dz;
  r.code = (int16_t)find_loss_coordinates(m.zmin, m.zmax, m.dz, m.dr, m.nr, fl, m.pitch, z0, r0, z1,
                                          r.neg ? -rd : rd, &r.zLost, &r.rLost);
}

// ---- compaction

__global__ void k_reset_step_counts32(DevCounts *cnt)
{
  cnt->first_lost = 0x7fffffffffffffffLL;
  cnt->n_lost = 0;
  cnt->new_active = 0;
  cnt->pushed += cnt->npActive;
  cnt->oa_min = INFINITY; // HUGE, advance_particles.c:113-114
  cnt->oa_max = -INFINITY;
}

// The reference's removal: the first lost index ends the beam (:490-518 as released).
__global__ void k_compact_reference32(DevCounts *cnt)
{
  const long long np = cnt->np;
  cnt->npActive += cnt->new_active;
  if (cnt->n_lost && cnt->first_lost < np) {
    cnt->npActive -= np - cnt->first_lost;
    cnt->np = cnt->first_lost;
  }
}

__device__ __forceinline__ void move32(const DevBeam32 &b, long dst, long src)
{
  b.cell[dst] = b.cell[src];
  b.fz[dst] = b.fz[src];
  b.fr[dst] = b.fr[src];
  b.pz[dst] = b.pz[src];
  b.pr[dst] = b.pr[src];
  b.rpphi[dst] = b.rpphi[src];
  b.Q[dst] = b.Q[src];
  b.status[dst] = b.status[src];
  b.zmin[dst] = b.zmin[src];
  b.zmax[dst] = b.zmax[src];
  b.rmin[dst] = b.rmin[src];
  b.rmax[dst] = b.rmax[src];
  b.r0[dst] = b.r0[src];
  b.z0[dst] = b.z0[src];
  b.t0[dst] = b.t0[src];
  b.particleID[dst] = b.particleID[src];
  b.generation[dst] = b.generation[src];
}

// Removes exactly the lost particles (order not kept): the lost slots below
// the new count are refilled from the survivors above it, the k-th hole in
// ascending index order from the k-th survivor in ascending order, so the
// result does not depend on the order the push appended the losses (which
// follows the timing of its blocks).  One block; the lists are built with
// block-wide prefix counts in chunks; the holes, collected from the push's
// list, are put in order by a block radix sort when there are at most
// CT * CT_ITEMS of them, else collected again by a scan of the statuses.
constexpr int CT = 1024, CT_ITEMS = 4;
__global__ void __launch_bounds__(CT) k_compact_any32(DevBeam32 b, const int32_t *lost_list, DevCounts *cnt,
                                                       int32_t *holes, int32_t *donors)
{
  __shared__ int warp_tot[CT / 32];
  __shared__ int base_sh, n_holes_sh;
  typedef cub::BlockRadixSort<int, CT, CT_ITEMS> HoleSort;
  __shared__ typename HoleSort::TempStorage sort_tmp;
  const long long n_lost = cnt->n_lost, np = cnt->np, new_np = np - n_lost;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (n_lost > 0) {
    // list 0: holes (lost slots < new_np) from the push's list; list 1:
    // donors (survivors >= new_np) in index order; list 2: holes again, in
    // index order, from the statuses (only when too many to sort)
    for (int list = 0; list < 3; list++) {
      if (list == 2 && n_holes_sh <= CT * CT_ITEMS)
        break;
      if (tid == 0)
        base_sh = 0;
      __syncthreads();
      const long long span = list == 2 ? new_np : n_lost;
      for (long long c0 = 0; c0 < span; c0 += CT) {
        const long long i = c0 + tid;
        bool take = false;
        int val = 0;
        if (i < span) {
          if (list == 0) {
            val = lost_list[i];
            take = val < new_np;
          } else if (list == 1) {
            val = (int)(new_np + i);
            take = !(b.status[val] & S32_LOST);
          } else {
            val = (int)i;
            take = b.status[val] & S32_LOST;
          }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, take);
        if (lane == 0)
          warp_tot[wid] = __popc(bal);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < CT / 32; w++) {
          before += w < wid ? warp_tot[w] : 0;
          total += warp_tot[w];
        }
        const int base = base_sh;
        if (take)
          (list == 1 ? donors : holes)[base + before + __popc(bal & ((1u << lane) - 1))] = val;
        __syncthreads();
        if (tid == 0)
          base_sh = base + total;
        __syncthreads();
      }
      if (list == 0) {
        if (tid == 0)
          n_holes_sh = base_sh;
        __syncthreads();
        const int nh = n_holes_sh;
        if (nh <= CT * CT_ITEMS) {
          // the holes in ascending order (INT_MAX pads sort last)
          int k[CT_ITEMS];
#pragma unroll
          for (int q = 0; q < CT_ITEMS; q++) {
            const int at = tid * CT_ITEMS + q;
            k[q] = at < nh ? holes[at] : 0x7fffffff;
          }
          HoleSort(sort_tmp).Sort(k);
#pragma unroll
          for (int q = 0; q < CT_ITEMS; q++) {
            const int at = tid * CT_ITEMS + q;
            if (at < nh)
              holes[at] = k[q];
          }
          __syncthreads();
        }
      }
    }
    const int n_move = base_sh; // equal counts: every hole has a donor
    for (int k = tid; k < n_move; k += CT)
      move32(b, holes[k], donors[k]);
  }
  __syncthreads();
  if (tid == 0) {
    cnt->npActive += cnt->new_active - n_lost;
    cnt->np = new_np;
  }
}

// ---- cell sort

__global__ void k_sort_keys(DevBeam32 b, const DevCounts *cnt, uint32_t *keys, int32_t *idx, long long n)
{
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i >= n)
    return;
  if (i < cnt->np) {
    keys[i] = (uint32_t)b.cell[i] ^ 0x80000000u;
    idx[i] = (int32_t)i;
  } else {
    keys[i] = 0xffffffffu;
    idx[i] = (int32_t)i;
  }
}

__global__ void k_permute(DevBeam32 dst, DevBeam32 src, const int32_t *idx, const DevCounts *cnt)
{
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i >= cnt->np)
    return;
  const long s = idx[i];
  dst.cell[i] = src.cell[s];
  dst.fz[i] = src.fz[s];
  dst.fr[i] = src.fr[s];
  dst.pz[i] = src.pz[s];
  dst.pr[i] = src.pr[s];
  dst.rpphi[i] = src.rpphi[s];
  dst.Q[i] = src.Q[s];
  dst.status[i] = src.status[s];
  dst.zmin[i] = src.zmin[s];
  dst.zmax[i] = src.zmax[s];
  dst.rmin[i] = src.rmin[s];
  dst.rmax[i] = src.rmax[s];
  dst.r0[i] = src.r0[s];
  dst.z0[i] = src.z0[s];
  dst.t0[i] = src.t0[s];
  dst.particleID[i] = src.particleID[s];
  dst.generation[i] = src.generation[s];
}

// ---- births (cathode.c:464-659) into the split beam

__global__ void __launch_bounds__(T) k_births32(DevMesh m, DevFields32 f, DevBeam32 b, BirthParams p, DevCounts *cnt,
                                                 S32Scales sc, int deposit)
{
  const long long k = (long long)blockIdx.x * T + threadIdx.x;
  const long long np = cnt->np;
  const bool fits = np + p.total <= b.capacity;
  const bool on = k < p.total && fits;
  if (k == 0 && !fits)
    atomicOr(&cnt->error, SPIFFE_DEV_ERR_CAPACITY);
  int iz = 0, ir = 0;
  float fz = 0, fr = 0, bz = 0, br = 0, bphi = 0, qs = 0;
  const bool test = p.mode == SPIFFE_BIRTH_TEST;
  if (on && p.mode == SPIFFE_BIRTH_LIST) {
    // emitSecondaryElectrons (secondaryEmission.c:471-497) from the host's list
    const long long ip = np + k, n = p.total;
    const double *L = p.list;
    const double xz = (L[k] - m.zmin) / m.dz, xr = L[n + k] / m.dr;
    iz = (int)floor(xz);
    fz = (float)(xz - iz);
    if (fz >= 1.f) {
      fz = 0.f;
      iz++;
    }
    ir = (int)floor(xr);
    fr = (float)(xr - ir);
    if (fr >= 1.f) {
      fr = 0.f;
      ir++;
    }
    b.cell[ip] = s32_cell(iz, ir);
    b.fz[ip] = fz;
    b.fr[ip] = fr;
    b.pz[ip] = (float)L[2 * n + k];
    b.pr[ip] = (float)L[3 * n + k];
    b.rpphi[ip] = 0.f;
    b.Q[ip] = (float)L[6 * n + k];
    b.status[ip] = S32_ACTIVE;
    b.rmin[ip] = b.zmin[ip] = FLT_MAX;
    b.rmax[ip] = b.zmax[ip] = -FLT_MAX;
    b.z0[ip] = L[k];
    b.r0[ip] = L[n + k];
    b.t0[ip] = L[7 * n + k];
    b.particleID[ip] = (int32_t)L[9 * n + k];
    b.generation[ip] = (int16_t)L[8 * n + k];
    betas(b.pz[ip], b.pr[ip], 0.f, ((float)ir + fr) * (float)m.dr, bz, br, bphi);
    qs = b.Q[ip] * sc.s_charge;
  } else if (on && test) {
    // test_beam.c:91-103: position, momenta and charge; the rest as a fresh
    // slot holds it, inactive until the push activates it (no deposit)
    const long long ip = np + k;
    const double xz = (p.z_position - m.zmin) / m.dz, xr = p.inner_radius / m.dr;
    iz = (int)floor(xz);
    fz = (float)(xz - iz);
    if (fz >= 1.f) {
      fz = 0.f;
      iz++;
    }
    ir = (int)floor(xr);
    fr = (float)(xr - ir);
    if (fr >= 1.f) {
      fr = 0.f;
      ir++;
    }
    b.cell[ip] = s32_cell(iz, ir);
    b.fz[ip] = fz;
    b.fr[ip] = fr;
    b.pz[ip] = (float)p.pz0;
    b.pr[ip] = (float)p.pr0;
    b.rpphi[ip] = (float)p.rpphi0;
    b.Q[ip] = (float)p.Q;
    b.status[ip] = 0;
    b.rmin[ip] = b.zmin[ip] = b.rmax[ip] = b.zmax[ip] = 0;
    b.z0[ip] = b.r0[ip] = b.t0[ip] = 0;
    b.particleID[ip] = 0;
    b.generation[ip] = 0;
  } else if (on) {
    const long long ip = np + k;
    const double c = SPIFFE_C_MKS;
    double r, dte = 0;
    if (p.mode == 1) {
      int bin = 0;
      while (bin + 1 < p.n_bins && k >= p.bins[bin + 1].start)
        bin++;
      const BirthBin B = p.bins[bin];
      r = sqrt(spiffe_rng_uniform(p.key, p.counter_base + (uint64_t)k + 1) * B.area / SPIFFE_PI + B.rmin * B.rmin);
      dte = m.dt * (double)(k - B.start) / (1.0 * B.count);
    } else if (p.mode == 0) {
      const double rn = spiffe_rng_uniform(p.key, p.counter_base + (uint64_t)k + 1);
      r = sqrt(rn * (p.outer_radius * p.outer_radius - p.inner_radius * p.inner_radius) +
               p.inner_radius * p.inner_radius);
      dte = m.dt * (double)k / (1.0 * p.total);
    } else {
      r = sqrt(p.inner_r2 + (double)(k + 1) * p.dr2);
      dte = m.dt * (double)k / (1.0 * p.total);
    }
    double vz = p.initial_vz, vr = 0, vphi = p.initial_omega * r;
    double gamma = 1 / sqrt(1 - (vz / c) * (vz / c) - (vr / c) * (vr / c) - (vphi / c) * (vphi / c));
    double pz = vz / c * gamma, pr = vr / c * gamma, r_pphi = r * vphi / c * gamma;
    double z = p.z_position, t0 = p.time;
    if (p.spread) {
      const int P = m.pitch;
      long izc = (long)((p.z_position - m.zmin) / m.dz);
      if (izc <= 0)
        izc = 1;
      if (izc > m.nz)
        izc = m.nz;
      long irc = (long)(r / m.dr);
      double Ez = m.constE[0], Er = m.constE[1];
      if (m.modes & SPIFFE_FL_TM_FIELDS)
        Ez = (double)f.Ez[node((int)izc, (int)irc, P)] + (double)f.EzImposed[node((int)izc, (int)irc, P)];
      irc += 1;
      izc -= 1;
      if (m.modes & SPIFFE_FL_TM_FIELDS)
        Er = (double)f.Er[node((int)izc, (int)irc, P)] + (double)f.ErImposed[node((int)izc, (int)irc, P)];
      t0 -= dte;
      const double pphi = (r ? r_pphi / r : 0);
      z += vz * dte;
      r += vr * dte;
      pr += dte * p.QoMC * Er / p.stiffness;
      pz += dte * p.QoMC * Ez / p.stiffness;
      gamma = sqrt(pz * pz + pr * pr + pphi * pphi + 1);
    }
    const double xz = (z - m.zmin) / m.dz, xr = r / m.dr;
    iz = (int)floor(xz);
    fz = (float)(xz - iz);
    if (fz >= 1.f) {
      fz = 0.f;
      iz++;
    }
    ir = (int)floor(xr);
    fr = (float)(xr - ir);
    if (fr >= 1.f) {
      fr = 0.f;
      ir++;
    }
    b.cell[ip] = s32_cell(iz, ir);
    b.fz[ip] = fz;
    b.fr[ip] = fr;
    b.pz[ip] = (float)pz;
    b.pr[ip] = (float)pr;
    b.rpphi[ip] = (float)r_pphi;
    b.Q[ip] = (float)p.Q;
    b.status[ip] = S32_ACTIVE;
    b.rmin[ip] = b.zmin[ip] = FLT_MAX;
    b.rmax[ip] = b.zmax[ip] = -FLT_MAX;
    b.z0[ip] = z;
    b.r0[ip] = r;
    b.t0[ip] = t0;
    b.particleID[ip] = (int32_t)(cnt->nextParticleID + k);
    b.generation[ip] = 0;
    betas(b.pz[ip], b.pr[ip], b.rpphi[ip], ((float)ir + fr) * (float)m.dr, bz, br, bphi);
    qs = b.Q[ip] * sc.s_charge;
  }
  if (deposit)
    deposit_particle<false>(m, f, on && !test, iz, fz, ir, fr, bz, br, bphi, qs);
}

__global__ void k_births_commit32(long long total, long long capacity, int mode, DevCounts *cnt)
{
  if (cnt->np + total > capacity)
    return;
  cnt->np += total;
  if (mode == SPIFFE_BIRTH_TEST) // inactive and without an ID, test_beam.c:104
    return;
  cnt->npActive += total;
  if (mode != SPIFFE_BIRTH_LIST) // listed particles carry the IDs given at their queueing
    cnt->nextParticleID += total;
}

// interpolateFields at n points (zr[2i], zr[2i+1]) of the split form's
// fields: Ez, Er into E[2i], E[2i+1]
__global__ void k_gather_points32(DevMesh m, DevFields32 f, const double *zr, int n, int ncomp, double *E)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const double xz = (zr[2 * i] - m.zmin) / m.dz, xr = zr[2 * i + 1] / m.dr;
  const int iz = (int)floor(xz), ir = (int)floor(xr);
  float e[6];
  gather32<false>(m, f, iz, (float)(xz - iz), ir, (float)(xr - ir), e);
  for (int c = 0; c < ncomp; c++)
    E[(size_t)ncomp * i + c] = e[c];
}

// ---- conversions between the FP64 SoA and the split beam

__global__ void k_pack_pos(DevMesh m, const double *z, const double *r, DevBeam32 b, long long n, DevCounts *cnt)
{
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i >= n)
    return;
  const double xz = (z[i] - m.zmin) / m.dz, xr = r[i] / m.dr;
  double fiz = floor(xz), fir = floor(xr);
  if (fiz < -32767 || fiz > 32767 || fir < -32767 || fir > 32767) {
    atomicOr(&cnt->error, SPIFFE_DEV_ERR_INDEX);
    fiz = fiz < -32767 ? -32767 : (fiz > 32767 ? 32767 : fiz);
    fir = fir < -32767 ? -32767 : (fir > 32767 ? 32767 : fir);
  }
  int iz = (int)fiz, ir = (int)fir;
  float fz = (float)(xz - fiz), fr = (float)(xr - fir);
  if (fz >= 1.f) {
    fz = 0.f;
    iz++;
  }
  if (fr >= 1.f) {
    fr = 0.f;
    ir++;
  }
  b.cell[i] = s32_cell(iz, ir);
  b.fz[i] = fz;
  b.fr[i] = fr;
}

__global__ void k_unpack_pos(DevMesh m, DevBeam32 b, double *z, double *r, long long n)
{
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i >= n)
    return;
  const int32_t c = b.cell[i];
  z[i] = m.zmin + ((double)s32_iz(c) + (double)b.fz[i]) * m.dz;
  r[i] = ((double)s32_ir(c) + (double)b.fr[i]) * m.dr;
}

__global__ void k_unpack_vel(DevMesh m, DevBeam32 b, double *vz, double *vr, double *vphi, long long n)
{
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i >= n)
    return;
  const double r = ((double)s32_ir(b.cell[i]) + (double)b.fr[i]) * m.dr;
  const double pz = b.pz[i], pr = b.pr[i], rpp = b.rpphi[i], c = SPIFFE_C_MKS;
  double g, w = 0;
  if (r != 0) {
    g = sqrt(pz * pz + pr * pr + (rpp / r) * (rpp / r) + 1);
    w = c * rpp / r / g;
  } else {
    g = sqrt(pz * pz + pr * pr + 1);
  }
  if (vz) vz[i] = c * pz / g;
  if (vr) vr[i] = c * pr / g;
  if (vphi) vphi[i] = w;
}

__global__ void k_d2f(const double *s, float *d, long long n)
{
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i < n) {
    const double v = s[i];
    d[i] = v >= 1.7976931348623157e308 ? FLT_MAX : (v <= -1.7976931348623157e308 ? -FLT_MAX : (float)v);
  }
}

__global__ void k_f2d(const float *s, double *d, long long n)
{
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i < n) {
    const float v = s[i];
    d[i] = v == FLT_MAX ? DBL_MAX : (v == -FLT_MAX ? -DBL_MAX : (double)v);
  }
}

__global__ void k_status_pack(const uint64_t *s, uint8_t *d, long long n)
{
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i < n)
    d[i] = (uint8_t)((s[i] & SPIFFE_PART_ACTIVE ? S32_ACTIVE : 0u) | (s[i] & SPIFFE_PART_LOST ? S32_LOST : 0u));
}

__global__ void k_status_unpack(const uint8_t *s, uint64_t *d, long long n)
{
  const long long i = (long long)blockIdx.x * T + threadIdx.x;
  if (i < n)
    d[i] = (s[i] & S32_ACTIVE ? SPIFFE_PART_ACTIVE : 0ull) | (s[i] & S32_LOST ? SPIFFE_PART_LOST : 0ull);
}

} // namespace

// ------------------------------------------------------------ host entry

#include <cub/device/device_radix_sort.cuh>

extern "C" int s32_beam_alloc(DevBeam32 *b, long long n)
{
  *b = DevBeam32();
  b->capacity = n;
  cudaError_t e = cudaSuccess;
#define AL(x) \
  if (e == cudaSuccess) e = cudaMalloc(&b->x, sizeof(*b->x) * (size_t)n);
  AL(cell) AL(fz) AL(fr) AL(pz) AL(pr) AL(rpphi) AL(Q) AL(status) AL(zmin) AL(zmax) AL(rmin) AL(rmax) AL(r0) AL(z0)
  AL(t0) AL(particleID) AL(generation)
#undef AL
  return (int)e;
}

extern "C" void s32_beam_free(DevBeam32 *b)
{
  void *p[] = {b->cell, b->fz, b->fr, b->pz, b->pr, b->rpphi, b->Q, b->status, b->zmin, b->zmax,
               b->rmin, b->rmax, b->r0, b->z0, b->t0, b->particleID, b->generation};
  for (void *q : p)
    cudaFree(q);
  *b = DevBeam32();
}

extern "C" int s32_beam_copy(DevBeam32 *dst, const DevBeam32 *src, long long n, cudaStream_t s)
{
  cudaError_t e = cudaSuccess;
#define CP(x) \
  if (e == cudaSuccess && n) e = cudaMemcpyAsync(dst->x, src->x, sizeof(*src->x) * (size_t)n, cudaMemcpyDeviceToDevice, s);
  CP(cell) CP(fz) CP(fr) CP(pz) CP(pr) CP(rpphi) CP(Q) CP(status) CP(zmin) CP(zmax) CP(rmin) CP(rmax) CP(r0) CP(z0)
  CP(t0) CP(particleID) CP(generation)
#undef CP
  return (int)e;
}

extern "C" int s32_particles_work(Particles32Work *w, long long capacity)
{
  if (w->capacity >= capacity)
    return 0;
  s32_particles_work_free(w);
  cudaError_t e = cudaMalloc(&w->lost_list, sizeof(int32_t) * (size_t)(capacity + 16));
  if (e == cudaSuccess) e = cudaMalloc(&w->keys, sizeof(int32_t) * (size_t)(capacity + 16));
  if (e == cudaSuccess) e = cudaMalloc(&w->keys_alt, sizeof(int32_t) * (size_t)(capacity + 16));
  if (e == cudaSuccess) e = cudaMalloc(&w->idx, sizeof(int32_t) * (size_t)(capacity + 16));
  if (e == cudaSuccess) e = cudaMalloc(&w->idx_alt, sizeof(int32_t) * (size_t)(capacity + 16));
  size_t sort_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint32_t *)nullptr, (uint32_t *)nullptr, (int32_t *)nullptr,
                                  (int32_t *)nullptr, (int)capacity);
  w->cub_bytes = sort_bytes;
  if (e == cudaSuccess) e = cudaMalloc(&w->cub_tmp, w->cub_bytes);
  if (e == cudaSuccess) e = (cudaError_t)s32_beam_alloc(&w->alt, capacity);
  w->capacity = capacity;
  return (int)e;
}

extern "C" void s32_particles_work_free(Particles32Work *w)
{
  cudaFree(w->lost_list);
  cudaFree(w->keys);
  cudaFree(w->keys_alt);
  cudaFree(w->idx);
  cudaFree(w->idx_alt);
  cudaFree(w->cub_tmp);
  s32_beam_free(&w->alt);
  *w = Particles32Work();
}

extern "C" int s32_deposit(const DevMesh *m, const DevFields32 *f, const DevBeam32 *b, const DevCounts *cnt,
                           long long np_bound, const S32Scales *sc, cudaStream_t s)
{
  if (np_bound <= 0)
    return 0;
  k_deposit32<<<blocks_for(np_bound, T), T, 0, s>>>(*m, *f, *b, cnt, *sc);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_push(const DevMesh *m, const DevFields32 *f, const DevBeam32 *b, const Push32Params *p,
                        const DevScreens *scr, DevCounts *cnt, long long np_bound, int compaction,
                        const S32Scales *sc, Particles32Work *w, cudaStream_t s)
{
  k_reset_step_counts32<<<1, 1, 0, s>>>(cnt);
  spiffe_note_launches(1);
  const bool any = compaction != SPIFFE_COMPACT_REFERENCE;
  if (np_bound > 0) {
    if (scr->n && p->screen_momentum == SPIFFE_SCREEN_REFERENCE) {
      k_snapshot_last32<<<1, 1, 0, s>>>(*b, cnt);
      spiffe_note_launches(1);
    }
    // the default field modes get a variant with the mode tests folded away
    const unsigned def_modes = SPIFFE_FL_TM_FIELDS | SPIFFE_FL_LONGIT_INTERP | SPIFFE_FL_RADIAL_INTERP;
    const unsigned mode_bits = SPIFFE_FL_TM_FIELDS | SPIFFE_FL_TE_FIELDS | SPIFFE_FL_LONGIT_INTERP |
                               SPIFFE_FL_RADIAL_INTERP | SPIFFE_FL_LONGIT_SMEAR | SPIFFE_FL_RADIAL_SMEAR;
    bool def = (m->modes & mode_bits) == def_modes && !p->forced && !m->n_onaxis;
    for (int k = 0; k < 6; k++)
      def = def && !m->turn_off[k];
    int32_t *ll = any ? w->lost_list : nullptr;
    const unsigned nb = blocks_for(np_bound, T);
    if (p->deposit && def)
      k_push32<true, true><<<nb, T, 0, s>>>(*m, *f, *b, *p, *scr, cnt, ll, *sc);
    else if (p->deposit)
      k_push32<true, false><<<nb, T, 0, s>>>(*m, *f, *b, *p, *scr, cnt, ll, *sc);
    else if (def)
      k_push32<false, true><<<nb, T, 0, s>>>(*m, *f, *b, *p, *scr, cnt, ll, *sc);
    else
      k_push32<false, false><<<nb, T, 0, s>>>(*m, *f, *b, *p, *scr, cnt, ll, *sc);
    spiffe_note_launches(1);
    if (p->lost.rec) {
      k_lost32<<<blocks_for(p->lost.cap, T), T, 0, s>>>(*m, f->flags, *b, p->lost);
      spiffe_note_launches(1);
    }
  }
  if (!any) {
    k_compact_reference32<<<1, 1, 0, s>>>(cnt);
  } else {
    k_compact_any32<<<1, CT, 0, s>>>(*b, w->lost_list, cnt, w->keys, w->idx);
  }
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

// Reorders the beam by cell (stable radix sort of the cell keys), leaving the
// result in *b (the buffers of b and w->alt are exchanged).
extern "C" int s32_sort(const DevMesh *m, DevBeam32 *b, DevCounts *cnt, long long np_bound, Particles32Work *w,
                        cudaStream_t s)
{
  (void)m;
  if (np_bound <= 1)
    return 0;
  const int n = (int)np_bound;
  k_sort_keys<<<blocks_for(n, T), T, 0, s>>>(*b, cnt, (uint32_t *)w->keys, w->idx, n);
  spiffe_note_launches(1);
  size_t bytes = w->cub_bytes;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(w->cub_tmp, bytes, (uint32_t *)w->keys, (uint32_t *)w->keys_alt,
                                                  w->idx, w->idx_alt, n, 0, 32, s);
  if (e != cudaSuccess)
    return (int)e;
  k_permute<<<blocks_for(n, T), T, 0, s>>>(w->alt, *b, w->idx_alt, cnt);
  spiffe_note_launches(1);
  const DevBeam32 t = *b;
  *b = w->alt;
  w->alt = t;
  return (int)cudaGetLastError();
}

extern "C" int s32_births(const DevMesh *m, const DevFields32 *f, const DevBeam32 *b, const BirthParams *p,
                          DevCounts *cnt, const S32Scales *sc, int deposit, cudaStream_t s)
{
  if (p->total <= 0)
    return 0;
  k_births32<<<blocks_for(p->total, T), T, 0, s>>>(*m, *f, *b, *p, cnt, *sc, deposit);
  k_births_commit32<<<1, 1, 0, s>>>(p->total, b->capacity, p->mode, cnt);
  spiffe_note_launches(2);
  return (int)cudaGetLastError();
}

extern "C" int s32_gather_points(const DevMesh *m, const DevFields32 *f, const double *zr, int n, int ncomp, double *E,
                                 cudaStream_t s)
{
  if (n <= 0)
    return 0;
  k_gather_points32<<<blocks_for(n, 128), 128, 0, s>>>(*m, *f, zr, n, ncomp < 6 ? ncomp : 6, E);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_beam_pack_pos(const DevMesh *m, const double *z, const double *r, DevBeam32 *b, long long n,
                                     DevCounts *cnt, cudaStream_t s)
{
  if (n <= 0)
    return 0;
  k_pack_pos<<<blocks_for(n, T), T, 0, s>>>(*m, z, r, *b, n, cnt);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_beam_unpack_pos(const DevMesh *m, const DevBeam32 *b, double *z, double *r, long long n,
                                   cudaStream_t s)
{
  if (n <= 0)
    return 0;
  k_unpack_pos<<<blocks_for(n, T), T, 0, s>>>(*m, *b, z, r, n);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_beam_unpack_vel(const DevMesh *m, const DevBeam32 *b, double *vz, double *vr, double *vphi,
                                   long long n, cudaStream_t s)
{
  if (n <= 0)
    return 0;
  k_unpack_vel<<<blocks_for(n, T), T, 0, s>>>(*m, *b, vz, vr, vphi, n);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_d2f(const double *src, float *dst, long long n, cudaStream_t s)
{
  if (n <= 0)
    return 0;
  k_d2f<<<blocks_for(n, T), T, 0, s>>>(src, dst, n);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_f2d(const float *src, double *dst, long long n, cudaStream_t s)
{
  if (n <= 0)
    return 0;
  k_f2d<<<blocks_for(n, T), T, 0, s>>>(src, dst, n);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_status_pack(const uint64_t *src, uint8_t *dst, long long n, cudaStream_t s)
{
  if (n <= 0)
    return 0;
  k_status_pack<<<blocks_for(n, T), T, 0, s>>>(src, dst, n);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_status_unpack(const uint8_t *src, uint64_t *dst, long long n, cudaStream_t s)
{
  if (n <= 0)
    return 0;
  k_status_unpack<<<blocks_for(n, T), T, 0, s>>>(src, dst, n);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}
