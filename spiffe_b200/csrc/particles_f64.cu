// spiffe_b200/csrc/particles_f64.cu -- plain FP64 particle kernels.
//
// Current deposition (space_charge.c:34-295), field gather (interpolateFields,
// advance_particles.c:622-890), the momentum kick and drift with loss tests
// (advance_particles.c:131-339), screen crossings (:362-434) and the removal
// of lost particles (:490-518), one thread per particle over the
// structure-of-arrays beam.  Arithmetic keeps the reference's expression
// order and the file is built with -fmad=false, so a particle's trajectory is
// bit-identical to the reference's given the same fields.  Deposition sums
// with FP64 atomics by default (order-dependent in the last bits) or, in the
// ordered mode, in particle order exactly as the serial reference does.
#include "modules.cuh"

namespace {

constexpr int T = 256;

__device__ __forceinline__ long trunc_l(double x) { return (long)x; }

// checkLossCode, advance_particles.c:31-65
__device__ int loss_code(const DevMesh &m, const int16_t *fl, long iz, long ir)
{
  const int P = m.pitch;
  const int16_t f0 = fl[node((int)iz, (int)ir, P)];
  if (f0 & SPIFFE_FL_IS_INSIDE)
    return 3;
  if (f0 & SPIFFE_FL_IS_SURFACE) {
    if (iz + 1 > m.nz)
      return 4;
    if (ir + 1 > m.nr)
      return 5;
    if (fl[node((int)iz + 1, (int)ir + 1, P)] & SPIFFE_FL_IS_METAL && fl[node((int)iz, (int)ir + 1, P)] & SPIFFE_FL_IS_METAL &&
        fl[node((int)iz + 1, (int)ir, P)] & SPIFFE_FL_IS_METAL)
      return 6;
  }
  return 0;
}

// interpolateFields, advance_particles.c:622-890.  E = Ez, Er, Ephi, Bz, Br, Bphi.
__device__ void gather(const DevMesh &m, const DevFields<double> &f, double z, double r, double *E)
{
  const long nz = m.nz, nr = m.nr;
  const int P = m.pitch;
  const double dz = m.dz, dr = m.dr, zmin = m.zmin;
  const bool longit = m.modes & SPIFFE_FL_LONGIT_INTERP, radial = m.modes & SPIFFE_FL_RADIAL_INTERP;
  const bool tm = m.modes & SPIFFE_FL_TM_FIELDS, te = m.modes & SPIFFE_FL_TE_FIELDS;
  const int16_t *fl = f.flags;
  long iz, ir, iz1, ir1;
  double fr, fl_, fa, fb;
  double Ez = 0, Er = 0, Ephi = 0, Bz = 0, Br = 0, Bphi = 0;
#define N(a, b) node((int)(a), (int)(b), P)
  // Ez and Br, :649-710
  if (longit) {
    fr = (z - zmin) / dz + 0.5;
    iz = trunc_l(fr);
    fr -= iz;
    fl_ = 1 - fr;
  } else {
    iz = trunc_l((z - zmin) / dz + 1);
    fl_ = 1;
    fr = 0;
  }
  if (radial) {
    fa = r / dr;
    ir = trunc_l(fa);
    fa -= ir;
    fb = 1 - fa;
  } else {
    ir = trunc_l(r / dr + 0.5);
    fa = 0;
    fb = 1;
  }
  if (iz >= 0 && iz < nz && ir >= 0 && ir < nr) {
    if ((iz1 = iz + 1) >= nz)
      iz1 = iz;
    if ((ir1 = ir + 1) >= nr)
      ir1 = ir;
    if (fl[N(iz, ir + 1)] & SPIFFE_FL_ER_ZERO && fl[N(iz, ir)] & SPIFFE_FL_ER_ZERO) {
      if (iz > 0 && (fl[N(iz - 1, ir)] || fl[N(iz - 1, ir + 1)]))
        iz = iz1;
      else
        iz1 = iz;
    } else if (fl[N(iz1, ir + 1)] & SPIFFE_FL_ER_ZERO && fl[N(iz1, ir)] & SPIFFE_FL_ER_ZERO) {
      iz1 = iz;
    }
    if (tm)
      Ez = fb * (fl_ * (f.Ez[N(iz, ir)] + f.EzImposed[N(iz, ir)]) + fr * (f.Ez[N(iz1, ir)] + f.EzImposed[N(iz1, ir)])) +
           fa * (fl_ * (f.Ez[N(iz, ir1)] + f.EzImposed[N(iz, ir1)]) + fr * (f.Ez[N(iz1, ir1)] + f.EzImposed[N(iz1, ir1)]));
    if (r != 0 && te)
      Br = fb * (fl_ * f.Br2[N(iz, ir)] + fr * f.Br2[N(iz1, ir)]) + fa * (fl_ * f.Br2[N(iz, ir1)] + fr * f.Br2[N(iz1, ir1)]);
  }
  // Er and Bz, :713-752
  if (longit) {
    fr = (z - zmin) / dz;
    iz = trunc_l(fr);
    fr -= iz;
    fl_ = 1 - fr;
  } else {
    iz = trunc_l((z - zmin) / dz + 0.5);
    fr = 0;
    fl_ = 1;
  }
  if (radial) {
    fa = r / dr + 0.5;
    ir = trunc_l(fa);
    fa -= ir;
    fb = 1 - fa;
  } else {
    ir = trunc_l(r / dr + 1);
    fa = 0;
    fb = 1;
  }
  if (iz >= 0 && iz < nz && ir >= 0) {
    if (ir >= nr)
      ir = nr - 1;
    iz1 = iz + 1;
    ir1 = ir + 1;
    if (fl[N(iz + 1, ir)] & SPIFFE_FL_EZ_ZERO && fl[N(iz, ir)] & SPIFFE_FL_EZ_ZERO)
      ir = ir1;
    else if (fl[N(iz + 1, ir + 1)] & SPIFFE_FL_EZ_ZERO && fl[N(iz, ir + 1)] & SPIFFE_FL_EZ_ZERO)
      ir1 = ir;
    if (r != 0 && tm)
      Er = fl_ * (fb * (f.Er[N(iz, ir)] + f.ErImposed[N(iz, ir)]) + fa * (f.Er[N(iz, ir1)] + f.ErImposed[N(iz, ir1)])) +
           fr * (fb * (f.Er[N(iz1, ir)] + f.ErImposed[N(iz1, ir)]) + fa * (f.Er[N(iz1, ir1)] + f.ErImposed[N(iz1, ir1)]));
    if (te)
      Bz = fl_ * (fb * f.Bz2[N(iz, ir)] + fa * f.Bz2[N(iz, ir1)]) + fr * (fb * f.Bz2[N(iz1, ir)] + fa * f.Bz2[N(iz1, ir1)]);
  }
  // Ephi, :754-786
  if (te && r != 0) {
    if (longit) {
      fr = (z - zmin) / dz;
      iz = trunc_l(fr);
      fr -= iz;
      fl_ = 1 - fr;
    } else {
      iz = trunc_l((z - zmin) / dz + 0.5);
      fr = 0;
      fl_ = 1;
    }
    if (radial) {
      fa = r / dr;
      ir = trunc_l(fa);
      fa -= ir;
      fb = 1 - fa;
    } else {
      ir = trunc_l(r / dr + 0.5);
      fa = 0;
      fb = 1;
    }
    if (iz >= 0 && iz < nz && ir >= 0 && ir < nr) {
      if ((iz1 = iz + 1) >= nz)
        iz1 = iz;
      if ((ir1 = ir + 1) >= nr)
        ir1 = ir;
      Ephi = fl_ * fb * f.Ephi[N(iz, ir)] + fr * fb * f.Ephi[N(iz1, ir)] + fl_ * fa * f.Ephi[N(iz, ir1)] +
             fr * fa * f.Ephi[N(iz1, ir1)];
    }
  }
  // Bphi at the E time level, :788-825
  if (tm) {
    if (longit) {
      fr = (z - zmin) / dz + 0.5;
      iz = trunc_l(fr);
      fr -= iz;
      fl_ = 1 - fr;
    } else {
      iz = trunc_l((z - zmin) / dz + 1);
      fr = 0;
      fl_ = 1;
    }
    if (radial) {
      fa = r / dr + 0.5;
      ir = trunc_l(fa);
      fa -= ir;
      fb = 1 - fa;
    } else {
      ir = trunc_l(r / dr + 1);
      fa = 0;
      fb = 1;
    }
    if (r != 0 && iz >= 0 && iz < nz) {
      if ((iz1 = iz + 1) >= nz)
        iz1 = iz;
      if (ir >= nr)
        ir = nr - 1;
      if ((ir1 = ir + 1) >= nr)
        ir1 = ir;
      Bphi = fl_ * fb * f.Bphi2[N(iz, ir)] + fr * fb * f.Bphi2[N(iz1, ir)] + fa * fl_ * f.Bphi2[N(iz, ir1)] +
             fr * fa * f.Bphi2[N(iz1, ir1)];
    }
  }
  // uniform fields, the on-axis expansion, switches, :828-857
  Ez += m.constE[0];
  Er += m.constE[1];
  Ephi += m.constE[2];
  Bz += m.constB[0];
  Br += m.constB[1];
  Bphi += m.constB[2];
  if (m.n_onaxis)
    onaxis_add(m, z, r, Ez, Er, Bphi);
  if (m.turn_off[0]) Ez = 0;
  if (m.turn_off[1]) Er = 0;
  if (m.turn_off[2]) Ephi = 0;
  if (m.turn_off[3]) Bz = 0;
  if (m.turn_off[4]) Br = 0;
  if (m.turn_off[5]) Bphi = 0;
  // solenoid fields on nodes, :859-875
  if (m.has_solenoid) {
    fr = (z - zmin) / dz;
    iz = trunc_l(fr);
    fa = r / dr;
    ir = trunc_l(fa);
    if (ir >= 0 && iz >= 0 && ir < nr && iz < nz) {
      fa -= ir;
      fb = 1 - fa;
      fr -= iz;
      fl_ = 1 - fr;
      Bz += fl_ * (fb * f.BzImposed[N(iz, ir)] + fa * f.BzImposed[N(iz, ir + 1)]) +
            fr * (fb * f.BzImposed[N(iz + 1, ir)] + fa * f.BzImposed[N(iz + 1, ir + 1)]);
      Br += fl_ * (fb * f.BrImposed[N(iz, ir)] + fa * f.BrImposed[N(iz, ir + 1)]) +
            fr * (fb * f.BrImposed[N(iz + 1, ir)] + fa * f.BrImposed[N(iz + 1, ir + 1)]);
    }
  }
#undef N
  E[0] = Ez;
  E[1] = Er;
  E[2] = Ephi;
  E[3] = Bz;
  E[4] = Br;
  E[5] = Bphi;
}


struct PushParams {
  double time, z_forces_start;
  double QoMC, stiffness;
  double tb_epm, tb_z_force, tb_r_force, tb_z_decel, tb_r_decel;
  int screen_momentum;
  LostLog lost;
};

__device__ void record(const DevScreen &s, long long step, long long *nb, long long *overflow, const DevBeam64 &b,
                       long ip, const double *q)
{
  const long long k = atomic_add_ll(nb, 1LL);
  if (k >= s.capacity) {
    atomic_add_ll(overflow, 1LL);
    return;
  }
  s.order[k] = (step << 32) | (long long)ip;
  for (int c = 0; c < SPIFFE_SCREEN_QUANS; c++)
    s.col[c][k] = q[c];
  s.rmin[k] = b.rmin[ip];
  s.rmax[k] = b.rmax[ip];
  s.zmin[k] = b.zmin[ip];
  s.zmax[k] = b.zmax[ip];
  s.generation[k] = b.generation[ip];
  s.particleID[k] = b.particleID[ip];
}

// Pre-kick momenta of the last particle, which the reference's screen loop
// reads through its function-scope pz0/pr0/r_pphi0 (advance_particles.c:79,
// :202-204, :383-385).
__global__ void k_snapshot_last(DevBeam64 b, DevCounts *cnt)
{
  const long long np = cnt->np;
  if (np > 0) {
    cnt->last_pz0 = b.pz[np - 1];
    cnt->last_pr0 = b.pr[np - 1];
    cnt->last_rpphi0 = b.r_pphi[np - 1];
  }
}

// advance_particles' per-particle loop (:131-339) and screen loop (:362-434).
__global__ void __launch_bounds__(T) k_push(DevMesh m, DevFields<double> f, DevBeam64 b, PushParams p,
                                             DevScreens scr, DevCounts *cnt, uint8_t *lost_flag)
{
  const long ip = (long)blockIdx.x * T + threadIdx.x;
  const long np = (long)cnt->np;
  if (ip >= np)
    return;
  const double dt = m.dt, dz = m.dz, dr = m.dr, zmin = m.zmin, zmax = m.zmax, rmax = m.rmax;
  const long nz = m.nz, nr = m.nr;
  const int16_t *fl = f.flags;
  const bool forced = p.tb_epm && (p.tb_z_force || p.tb_r_force);
  double z, r, z0, r0s, vz, vr, pz, pr, r_pphi, vphi, gamma, pphi, adjust = 1, E[6];
  long iz, ir;
  bool lost = false, r_was_negative = false;
  uint64_t status = b.status[ip];
  double zmx = b.zmax[ip], zmn = b.zmin[ip], rmx = b.rmax[ip], rmn = b.rmin[ip];

  z = z0 = b.z[ip];
  r = r0s = b.r[ip];
  if (z > zmx) zmx = z;
  if (z < zmn) zmn = z;
  if (r > rmx) rmx = r;
  if (r < rmn) rmn = r;
  vz = b.vz[ip];
  vr = b.vr[ip];
  z += vz * dt;
  r += vr * dt;
  if (!(status & SPIFFE_PART_ACTIVE)) {
    // activation on entering the mesh, :167-189 (|r|/dr is bounded by nr
    // here; the reference would index past the flag array beyond it)
    iz = trunc_l((z - zmin) / dz);
    ir = trunc_l(fabs(r) / dr);
    if ((z >= zmin && z <= zmax && r <= rmax) && ir <= nr && !loss_code(m, fl, iz, ir)) {
      status |= SPIFFE_PART_ACTIVE;
      atomic_add_ll(&cnt->new_active, 1LL);
      b.t0[ip] = p.time;
      b.r0[ip] = r0s;
      b.z0[ip] = z0;
      if (iz > 0 && loss_code(m, fl, iz - 1, ir))
        adjust = (z - (iz * dz + zmin)) / (z - z0);
      else
        adjust = (z - zmin) / (z - z0);
      if (adjust > 1)
        adjust = 1;
    }
  }
  if (p.z_forces_start > zmin && p.z_forces_start < zmax) {
    if (z0 < p.z_forces_start) {
      if (z < p.z_forces_start)
        adjust = 0;
      else
        adjust = (z - p.z_forces_start) / (z - z0);
    }
  }
  const double pz0 = b.pz[ip], pr0 = b.pr[ip], rpp0 = b.r_pphi[ip];
  pz = pz0;
  pr = pr0;
  r_pphi = rpp0;
  vphi = b.vphi[ip];
  const bool active = status & SPIFFE_PART_ACTIVE;
  // loss tests, :211-236
  if (active && (z < zmin || z > zmax || r > rmax))
    lost = true;
  if (!lost && active) {
    iz = trunc_l((z - zmin) / dz);
    ir = trunc_l(fabs(r) / dr);
    if (iz > nz || ir > nr || iz < 0 || ir < 0)
      lost = true;
    else if (loss_code(m, fl, iz, ir))
      lost = true;
  }
  if (r < 0) {
    r *= -1;
    pr *= -1;
    r_was_negative = true;
  }
  if (!lost && active) {
    if (z > zmx) zmx = z;
    if (z < zmn) zmn = z;
    if (r > rmx) rmx = r;
    if (r < rmn) rmn = r;
  }
  if (!forced) {
    // momentum kick with the stored (old) velocities, :270-287
    if (active)
      gather(m, f, z, r, E);
    else
      E[0] = E[1] = E[2] = E[3] = E[4] = E[5] = 0;
    const double QoMC = p.QoMC, stiff = p.stiffness;
    pphi = (r ? r_pphi / r : 0);
    gamma = sqrt(pr * pr + pz * pz + pphi * pphi + 1);
    pr += adjust * dt * ((r ? pphi * pphi * SPIFFE_C_MKS / gamma / r : 0) + QoMC * (E[1] + vphi * E[3] - vz * E[5])) / stiff;
    pz += adjust * dt * QoMC * (E[0] + vr * E[5] - vphi * E[4]) / stiff;
    r_pphi += adjust * dt * QoMC * r * (E[2] + vz * E[4] - vr * E[3]) / stiff;
  } else {
    // forced test-beam acceleration, :289-311
    pphi = (r ? r_pphi / r : 0);
    gamma = sqrt(pr * pr + pz * pz + pphi * pphi + 1);
    pr += dt * ((r ? pphi * pphi * SPIFFE_C_MKS / gamma / r : 0));
    if (z <= p.tb_z_decel)
      pz += dt * p.tb_z_force;
    else {
      pz -= dt * p.tb_z_force;
      if (pz < 0)
        pz = 0;
    }
    if (r_was_negative)
      pr = 0;
    else if (r <= p.tb_r_decel)
      pr += dt * p.tb_r_force;
    else
      pr -= dt * p.tb_r_force;
  }
  // new velocities, setParticleVelocities :605-620
  double nvz, nvr, nvphi;
  if (r) {
    gamma = sqrt(pz * pz + pr * pr + (r_pphi / r) * (r_pphi / r) + 1);
    nvphi = SPIFFE_C_MKS * r_pphi / r / gamma;
  } else {
    gamma = sqrt(pz * pz + pr * pr + 1);
    nvphi = 0;
  }
  nvz = SPIFFE_C_MKS * pz / gamma;
  nvr = SPIFFE_C_MKS * pr / gamma;
  b.z[ip] = z;
  b.r[ip] = r;
  b.pz[ip] = pz;
  b.pr[ip] = pr;
  b.r_pphi[ip] = r_pphi;
  b.vz[ip] = nvz;
  b.vr[ip] = nvr;
  b.vphi[ip] = nvphi;
  b.zmax[ip] = zmx;
  b.zmin[ip] = zmn;
  b.rmax[ip] = rmx;
  b.rmin[ip] = rmn;
  if (lost) {
    status &= ~SPIFFE_PART_ACTIVE;
    status |= SPIFFE_PART_LOST;
    atomic_add_ll(&cnt->n_lost, 1LL);
    atomicMin(&cnt->first_lost, (long long)ip);
  }
  b.status[ip] = status;
  lost_flag[ip] = lost ? 1 : 0;
  if (lost && p.lost.rec) { // the loss epilogue, :437-487
    double pm = pz * pz + pr * pr;
    if (r)
      pm += (r_pphi / r) * (r_pphi / r);
    LostRecord rec{p.time, 0, 0, sqrt(pm), pz, pr, b.r0[ip], b.z0[ip], b.Q[ip], (long long)ip, p.lost.step,
                   b.particleID[ip], b.generation[ip], 0, 0, 0, 0.f, 0.f};
    rec.code = (int16_t)find_loss_coordinates(zmin, zmax, dz, dr, nr, fl, m.pitch, z0, r0s, z,
                                              r_was_negative ? -r : r, &rec.zLost, &rec.rLost);
    lost_append(p.lost, rec);
  }

  // screen crossings, :362-434
  if (scr.n) {
    const bool ref = p.screen_momentum == SPIFFE_SCREEN_REFERENCE;
    const double pz0s = ref ? cnt->last_pz0 : pz0, pr0s = ref ? cnt->last_pr0 : pr0;
    const double rpp0s = ref ? cnt->last_rpphi0 : rpp0;
    double r0 = r0s, q[SPIFFE_SCREEN_QUANS];
    for (int is = 0; is < scr.n; is++) {
      const DevScreen &s = scr.s[is];
      if (s.z_position <= z && s.z_position > z0 && s.direction == 1) {
        const double dtp = (s.z_position - z0) / vz;
        const double pphi_new = r ? r_pphi / r : 0;
        const double pphi0 = r0 ? rpp0s / r0 : 0;
        q[0] = r0 + vr * dtp;
        q[1] = pz0s + (pz - pz0s) / dt * dtp;
        q[2] = pr0s + (pr - pr0s) / dt * dtp;
        q[3] = pphi0 + (pphi_new - pphi0) / dt * dtp;
        q[4] = (p.time - dt + dtp);
        q[5] = b.Q[ip];
        q[6] = b.r0[ip];
        q[7] = b.t0[ip];
        record(s, scr.step, &cnt->screen_nb[is], &cnt->screen_overflow, b, ip, q);
      } else if (s.z_position >= z && s.z_position < z0 && s.direction == -1) {
        const double dtp = (s.z_position - z0) / vz;
        r0 += vr * dtp;
        q[0] = r0;
        q[1] = pz;
        q[2] = pr;
        q[3] = r0 ? r_pphi / r0 : 0;
        q[4] = (p.time - dt + dtp);
        q[5] = b.Q[ip];
        q[6] = b.r0[ip];
        q[7] = b.t0[ip];
        record(s, scr.step, &cnt->screen_nb[is], &cnt->screen_overflow, b, ip, q);
      }
    }
  }
}

// ------------------------------------------------------------ deposition
// add_particle_currents, space_charge.c:34-295, one thread per particle.
// Each particle's (up to) four node contributions per component are formed
// exactly as the reference forms them; they are either added with FP64
// atomics or written to a contribution list for the ordered reduction.

struct Contrib {
  int node[4];
  double val[4];
  int n;
};

__device__ void contrib_jz(const DevMesh &m, double z, double r, double v, double Q, double one_over, Contrib &c)
{
  const long nz = m.nz, nr = m.nr;
  const bool rsm = m.modes & SPIFFE_FL_RADIAL_SMEAR, lsm = m.modes & SPIFFE_FL_LONGIT_SMEAR;
  const double dz = m.dz, dr = m.dr, zmin = m.zmin;
  long iz, ir;
  double fp, fm, Jm, Jp;
  c.n = 0;
  ir = rsm ? trunc_l(r / dr) : trunc_l(r / dr + 0.5);
  iz = lsm ? trunc_l((z - zmin) / dz + 0.5) : trunc_l((z - zmin) / dz + 1.0);
  if (iz < 0 || iz > nz || ir < 0 || ir > nr)
    return;
  const double QVG = v * (Q * one_over);
  if (rsm) {
    fp = r / dr - ir;
    fm = 1 - fp;
  } else {
    fm = 1;
    fp = 0;
  }
  if (ir == 0) {
    Jm = 4 * fm * QVG;
    Jp = fp * QVG / (1.5 * 1.5 - 0.5 * 0.5);
  } else if (ir < nr - 1) {
    Jm = fm * QVG / ((ir + 0.5) * (ir + 0.5) - (ir - 0.5) * (ir - 0.5));
    Jp = fp * QVG / ((ir + 1.5) * (ir + 1.5) - (ir + 0.5) * (ir + 0.5));
  } else {
    Jm = 0;
    Jp = fp * QVG / ((ir + 0.5) * (ir + 0.5) - (ir - 0.5) * (ir - 0.5));
    ir--;
  }
  if (lsm) {
    if (iz == 0) {
      fp = 1;
      fm = 0;
    } else if (iz == nz) {
      fm = 1;
      fp = 0;
    } else {
      fp = (z - zmin) / dz + 0.5 - iz;
      fm = 1 - fp;
    }
  } else {
    fm = 1;
    fp = 0;
  }
  const int P = m.pitch;
  c.node[c.n] = (int)node((int)iz, (int)ir, P);
  c.val[c.n++] = fm * Jm;
  // row iz+1 exists only for iz < nz; at iz == nz its weight is zero (the
  // reference would index past the last row)
  if (lsm && iz < nz) {
    c.node[c.n] = (int)node((int)iz + 1, (int)ir, P);
    c.val[c.n++] = fp * Jm;
  }
  if (rsm) {
    c.node[c.n] = (int)node((int)iz, (int)ir + 1, P);
    c.val[c.n++] = fm * Jp;
    if (lsm && iz < nz) {
      c.node[c.n] = (int)node((int)iz + 1, (int)ir + 1, P);
      c.val[c.n++] = fp * Jp;
    }
  }
}

__device__ void contrib_jr(const DevMesh &m, double z, double r, double v, double Q, double one_over, Contrib &c)
{
  const long nz = m.nz, nr = m.nr;
  const bool rsm = m.modes & SPIFFE_FL_RADIAL_SMEAR, lsm = m.modes & SPIFFE_FL_LONGIT_SMEAR;
  const double dz = m.dz, dr = m.dr, zmin = m.zmin;
  long iz, ir;
  double fp, fm, Jm, Jp;
  c.n = 0;
  ir = rsm ? trunc_l(r / dr + 0.5) : trunc_l(r / dr + 1.0);
  iz = lsm ? trunc_l((z - zmin) / dz) : trunc_l((z - zmin) / dz + 0.5);
  if (iz < 0 || iz > nz || ir < 0 || ir >= nr)
    return;
  if (rsm) {
    fp = r / dr + 0.5 - ir;
    fm = 1 - fp;
  } else {
    fm = 1;
    fp = 0;
  }
  const double QVG = v * (Q * one_over);
  if (ir == 0) {
    Jm = 0;
    Jp = QVG;
  } else if (ir < nr - 1) {
    Jm = fm * QVG / ((double)ir * ir - (double)(ir - 1) * (ir - 1));
    Jp = fp * QVG / ((double)(ir + 1) * (ir + 1) - (double)ir * ir);
  } else {
    Jm = 0;
    ir--;
    Jp = QVG / ((double)(ir + 1) * (ir + 1) - (double)ir * ir);
  }
  if (lsm) {
    if (iz == nz) {
      fm = 1;
      fp = 0;
    } else {
      fp = (z - zmin) / dz - iz;
      fm = 1 - fp;
    }
  } else {
    fm = 1;
    fp = 0;
  }
  const int P = m.pitch;
  c.node[c.n] = (int)node((int)iz, (int)ir, P);
  c.val[c.n++] = fm * Jm;
  // row iz+1 exists only for iz < nz; at iz == nz its weight is zero (the
  // reference would index past the last row)
  if (lsm && iz < nz) {
    c.node[c.n] = (int)node((int)iz + 1, (int)ir, P);
    c.val[c.n++] = fp * Jm;
  }
  if (rsm) {
    c.node[c.n] = (int)node((int)iz, (int)ir + 1, P);
    c.val[c.n++] = fm * Jp;
    if (lsm && iz < nz) {
      c.node[c.n] = (int)node((int)iz + 1, (int)ir + 1, P);
      c.val[c.n++] = fp * Jp;
    }
  }
}

__device__ void contrib_jphi(const DevMesh &m, double z, double r, double v, double Q, double one_over, Contrib &c)
{
  const long nz = m.nz, nr = m.nr;
  const bool rsm = m.modes & SPIFFE_FL_RADIAL_SMEAR, lsm = m.modes & SPIFFE_FL_LONGIT_SMEAR;
  const double dz = m.dz, dr = m.dr, zmin = m.zmin;
  long iz, ir;
  double fp, fm, Jm, Jp;
  c.n = 0;
  ir = rsm ? trunc_l(r / dr) : trunc_l(r / dr + 0.5);
  iz = lsm ? trunc_l((z - zmin) / dz) : trunc_l((z - zmin) / dz + 0.5);
  if (iz < 0 || iz > nz || ir < 0 || ir > nr)
    return;
  if (rsm) {
    fp = r / dr - ir;
    fm = 1 - fp;
  } else {
    fm = 1;
    fp = 0;
  }
  const double QVG = v * (Q * one_over);
  if (ir == 0) {
    Jm = 4 * fm * QVG;
    Jp = fp * QVG / (1.5 * 1.5 - 0.5 * 0.5);
  } else if (ir < nr - 1) {
    Jm = fm * QVG / ((ir + 0.5) * (ir + 0.5) - (ir - 0.5) * (ir - 0.5));
    Jp = fp * QVG / ((ir + 1.5) * (ir + 1.5) - (ir + 0.5) * (ir + 0.5));
  } else {
    Jm = 0;
    Jp = fp * QVG / ((ir + 0.5) * (ir + 0.5) - (ir - 0.5) * (ir - 0.5));
    ir--;
  }
  if (lsm) {
    if (iz == nz - 1) {
      fp = 0;
      fm = 1 - fp;
    } else {
      fp = (z - zmin) / dz - iz;
      fm = 1 - fp;
    }
  } else {
    fm = 1;
    fp = 0;
  }
  const int P = m.pitch;
  c.node[c.n] = (int)node((int)iz, (int)ir, P);
  c.val[c.n++] = fm * Jm;
  // row iz+1 exists only for iz < nz; at iz == nz its weight is zero (the
  // reference would index past the last row)
  if (lsm && iz < nz) {
    c.node[c.n] = (int)node((int)iz + 1, (int)ir, P);
    c.val[c.n++] = fp * Jm;
  }
  if (rsm) {
    c.node[c.n] = (int)node((int)iz, (int)ir + 1, P);
    c.val[c.n++] = fm * Jp;
    if (lsm && iz < nz) {
      c.node[c.n] = (int)node((int)iz + 1, (int)ir + 1, P);
      c.val[c.n++] = fp * Jp;
    }
  }
}

// component: 0 Jz, 1 Jr, 2 Jphi.  keys/vals != nullptr selects the ordered
// mode: slot 4*ip+k receives contribution k (key = node, or INT_MAX) for
// every ip below the host's bound n_slots, so slots past the live np (after
// losses) hold padding rather than an earlier step's contributions.
__global__ void __launch_bounds__(T) k_deposit(DevMesh m, DevFields<double> f, DevBeam64 b, const DevCounts *cnt,
                                                int component, int *keys, double *vals, long long n_slots)
{
  const long ip = (long)blockIdx.x * T + threadIdx.x;
  const long np = (long)cnt->np;
  if (ip >= np) {
    if (keys && ip < n_slots)
      for (int k = 0; k < 4; k++) {
        keys[4 * ip + k] = 0x7fffffff;
        vals[4 * ip + k] = 0.0;
      }
    return;
  }
  Contrib c;
  c.n = 0;
  if (b.status[ip] & SPIFFE_PART_ACTIVE) {
    const double one_over = 1 / (SPIFFE_PI * m.dz * (m.dr * m.dr));
    if (component == 0)
      contrib_jz(m, b.z[ip], b.r[ip], b.vz[ip], b.Q[ip], one_over, c);
    else if (component == 1)
      contrib_jr(m, b.z[ip], b.r[ip], b.vr[ip], b.Q[ip], one_over, c);
    else
      contrib_jphi(m, b.z[ip], b.r[ip], b.vphi[ip], b.Q[ip], one_over, c);
  }
  if (keys) {
    for (int k = 0; k < 4; k++) {
      keys[4 * ip + k] = k < c.n ? c.node[k] : 0x7fffffff;
      vals[4 * ip + k] = k < c.n ? c.val[k] : 0.0;
    }
    return;
  }
  double *J = component == 0 ? f.Jz : (component == 1 ? f.Jr : f.Jphi);
  for (int k = 0; k < c.n; k++)
    atomicAdd(J + c.node[k], c.val[k]);
}

// Ordered reduction: after a stable sort by node, each run of equal keys is
// summed in particle order starting from the array's current value, which is
// the reference's serial J[node] += ... sequence (space_charge.c:130-137).
__global__ void k_ordered_sum(const int *keys, const double *vals, long long n, double *J)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const int k = keys[i];
  if (k == 0x7fffffff || (i > 0 && keys[i - 1] == k))
    return;
  double acc = J[k];
  for (long long j = i; j < n && keys[j] == k; j++)
    acc += vals[j];
  J[k] = acc;
}

// ------------------------------------------------------------ compaction

#define MOVE_ALL(dst, src)                       \
  do {                                           \
    b.Q[dst] = b.Q[src];                         \
    b.z[dst] = b.z[src];                         \
    b.r[dst] = b.r[src];                         \
    b.pz[dst] = b.pz[src];                       \
    b.pr[dst] = b.pr[src];                       \
    b.vz[dst] = b.vz[src];                       \
    b.vr[dst] = b.vr[src];                       \
    b.r_pphi[dst] = b.r_pphi[src];               \
    b.vphi[dst] = b.vphi[src];                   \
    b.t0[dst] = b.t0[src];                       \
    b.r0[dst] = b.r0[src];                       \
    b.z0[dst] = b.z0[src];                       \
    b.rmin[dst] = b.rmin[src];                   \
    b.zmin[dst] = b.zmin[src];                   \
    b.rmax[dst] = b.rmax[src];                   \
    b.zmax[dst] = b.zmax[src];                   \
    b.generation[dst] = b.generation[src];       \
    b.particleID[dst] = b.particleID[src];       \
    b.status[dst] = b.status[src];               \
  } while (0)

// Reference compaction: the first lost index ends the beam.
__global__ void k_compact_reference(DevCounts *cnt)
{
  const long long np = cnt->np;
  cnt->npActive += cnt->new_active;
  if (cnt->n_lost && cnt->first_lost < np) {
    cnt->npActive -= np - cnt->first_lost;
    cnt->np = cnt->first_lost;
  }
}

// Swap compaction: survivors at the end refill lost slots at the front, the
// j-th lost slot (ascending) taking the j-th survivor counted from the end.
// surv_before[] is an exclusive prefix count of survivors over [0, np).
__global__ void k_compact_swap_map(const uint8_t *lost, const int *surv_before, const DevCounts *cnt, int *map)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long np = cnt->np, n_lost = cnt->n_lost, new_np = np - n_lost;
  if (i >= np || !n_lost)
    return;
  if (i >= new_np && !lost[i]) {
    const long long d = new_np - surv_before[i] - 1; // descending rank among tail survivors
    map[d] = (int)i;
  }
}

__global__ void k_compact_swap_move(DevBeam64 b, const uint8_t *lost, const int *surv_before, const DevCounts *cnt,
                                    const int *map)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long np = cnt->np, n_lost = cnt->n_lost, new_np = np - n_lost;
  if (i >= new_np || !n_lost || !lost[i])
    return;
  const long long a = i - surv_before[i]; // ascending rank among front lost slots
  const int src = map[a];
  MOVE_ALL(i, src);
}

__global__ void k_compact_swap_finish(DevCounts *cnt)
{
  cnt->npActive += cnt->new_active - cnt->n_lost;
  cnt->np -= cnt->n_lost;
}

__global__ void k_survivor_flags(const uint8_t *lost, const DevCounts *cnt, int *surv, long long n)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    surv[i] = (i < cnt->np && !lost[i]) ? 1 : 0;
}

__global__ void k_reset_step_counts(DevCounts *cnt)
{
  cnt->first_lost = 0x7fffffffffffffffLL;
  cnt->n_lost = 0;
  cnt->new_active = 0;
  cnt->pushed += cnt->npActive;
  cnt->oa_min = INFINITY; // HUGE, advance_particles.c:113-114
  cnt->oa_max = -INFINITY;
}

} // namespace

// ------------------------------------------------------------ host entry

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>


extern "C" int spiffe_particles64_work(Particles64Work *w, long long capacity, bool ordered)
{
  cudaError_t e = cudaSuccess;
  if (w->capacity < capacity) {
    cudaFree(w->lost);
    cudaFree(w->surv);
    cudaFree(w->surv_before);
    cudaFree(w->map);
    cudaFree(w->keys);
    cudaFree(w->keys_alt);
    cudaFree(w->vals);
    cudaFree(w->vals_alt);
    cudaFree(w->cub_tmp);
    *w = Particles64Work();
    e = cudaMalloc(&w->lost, capacity + 16);
    if (e == cudaSuccess) e = cudaMalloc(&w->surv, sizeof(int) * (capacity + 16));
    if (e == cudaSuccess) e = cudaMalloc(&w->surv_before, sizeof(int) * (capacity + 16));
    if (e == cudaSuccess) e = cudaMalloc(&w->map, sizeof(int) * (capacity + 16));
    size_t scan_bytes = 0, sort_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, w->surv, w->surv_before, (int)capacity);
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (int *)nullptr, (int *)nullptr, (double *)nullptr,
                                    (double *)nullptr, (int)(4 * capacity));
    w->cub_bytes = scan_bytes > sort_bytes ? scan_bytes : sort_bytes;
    if (e == cudaSuccess) e = cudaMalloc(&w->cub_tmp, w->cub_bytes);
    w->capacity = capacity;
  }
  if (e == cudaSuccess && ordered && !w->keys) {
    e = cudaMalloc(&w->keys, sizeof(int) * 4 * w->capacity);
    if (e == cudaSuccess) e = cudaMalloc(&w->keys_alt, sizeof(int) * 4 * w->capacity);
    if (e == cudaSuccess) e = cudaMalloc(&w->vals, sizeof(double) * 4 * w->capacity);
    if (e == cudaSuccess) e = cudaMalloc(&w->vals_alt, sizeof(double) * 4 * w->capacity);
  }
  return (int)e;
}

extern "C" void spiffe_particles64_work_free(Particles64Work *w)
{
  cudaFree(w->lost);
  cudaFree(w->surv);
  cudaFree(w->surv_before);
  cudaFree(w->map);
  cudaFree(w->keys);
  cudaFree(w->keys_alt);
  cudaFree(w->vals);
  cudaFree(w->vals_alt);
  cudaFree(w->cub_tmp);
  *w = Particles64Work();
}

// add_particle_currents.  np_bound is a host-side upper bound on np.
extern "C" int spiffe_deposit64(const DevMesh *m, const DevFields<double> *f, const DevBeam64 *b, const DevCounts *cnt,
                                long long np_bound, bool ordered, Particles64Work *w, cudaStream_t s)
{
  if (np_bound <= 0)
    return 0;
  const unsigned nb = blocks_for(np_bound, T);
  const size_t nodes = (size_t)(m->nz + 1) * m->pitch;
  int bits = 1;
  while ((1ull << bits) <= nodes)
    bits++;
  for (int comp = 0; comp < 3; comp++) {
    if (comp < 2 && !(m->modes & SPIFFE_FL_TM_FIELDS))
      continue;
    if (comp == 2 && !(m->modes & SPIFFE_FL_TE_FIELDS))
      continue;
    if (!ordered) {
      k_deposit<<<nb, T, 0, s>>>(*m, *f, *b, cnt, comp, nullptr, nullptr, 0);
      spiffe_note_launches(1);
      continue;
    }
    const int n = (int)(4 * np_bound);
    k_deposit<<<nb, T, 0, s>>>(*m, *f, *b, cnt, comp, w->keys, w->vals, np_bound);
    spiffe_note_launches(1);
    double *J = comp == 0 ? f->Jz : (comp == 1 ? f->Jr : f->Jphi);
    if (int rc = spiffe_ordered_add64(w, n, J, s))
      return rc;
    (void)bits;
  }
  return (int)cudaGetLastError();
}

extern "C" int spiffe_ordered_add64(Particles64Work *w, long long n, double *dst, cudaStream_t s)
{
  if (n <= 0)
    return 0;
  if (!w->keys || n > 4 * w->capacity)
    return (int)cudaErrorInvalidValue;
  // stable LSD radix sort keeps entry order inside each node's run; the
  // INT_MAX pad key sorts last within the 31-bit key space
  size_t bytes = w->cub_bytes;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(w->cub_tmp, bytes, w->keys, w->keys_alt, w->vals, w->vals_alt,
                                                  (int)n, 0, 31, s);
  if (e != cudaSuccess)
    return (int)e;
  k_ordered_sum<<<blocks_for(n, T), T, 0, s>>>(w->keys_alt, w->vals_alt, n, dst);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}


namespace {
// interpolateFields at n points (zr[2i], zr[2i+1]): the first ncomp of
// Ez, Er, Ephi, Bz, Br, Bphi into E[ncomp*i ...]
__global__ void k_gather_points64(DevMesh m, DevFields<double> f, const double *zr, int n, int ncomp, double *E)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double e[6];
  gather(m, f, zr[2 * i], zr[2 * i + 1], e);
  for (int c = 0; c < ncomp; c++)
    E[(size_t)ncomp * i + c] = e[c];
}
} // namespace

extern "C" int spiffe_gather_points64(const DevMesh *m, const DevFields<double> *f, const double *zr, int n, int ncomp,
                                      double *E, cudaStream_t s)
{
  if (n <= 0)
    return 0;
  k_gather_points64<<<blocks_for(n, 128), 128, 0, s>>>(*m, *f, zr, n, ncomp < 6 ? ncomp : 6, E);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

// advance_particles: snapshot, push with screens, then compaction.
extern "C" int spiffe_push64(const DevMesh *m, const DevFields<double> *f, const DevBeam64 *b, const PushHostParams *hp,
                             const DevScreens *scr, DevCounts *cnt, long long np_bound, Particles64Work *w, cudaStream_t s)
{
  k_reset_step_counts<<<1, 1, 0, s>>>(cnt);
  spiffe_note_launches(1);
  if (np_bound > 0) {
    PushParams p{hp->time, hp->z_forces_start, hp->QoMC, hp->stiffness, hp->tb_epm, hp->tb_z_force,
                 hp->tb_r_force, hp->tb_z_decel, hp->tb_r_decel, hp->screen_momentum, hp->lost};
    if (scr->n && hp->screen_momentum == SPIFFE_SCREEN_REFERENCE)
      { k_snapshot_last<<<1, 1, 0, s>>>(*b, cnt); spiffe_note_launches(1); }
    k_push<<<blocks_for(np_bound, T), T, 0, s>>>(*m, *f, *b, p, *scr, cnt, w->lost);
    spiffe_note_launches(1);
  }
  if (hp->compaction == SPIFFE_COMPACT_REFERENCE || np_bound <= 0) {
    k_compact_reference<<<1, 1, 0, s>>>(cnt);
    spiffe_note_launches(1);
  } else {
    const unsigned nb = blocks_for(np_bound, T);
    k_survivor_flags<<<nb, T, 0, s>>>(w->lost, cnt, w->surv, np_bound);
    spiffe_note_launches(1);
    size_t bytes = w->cub_bytes;
    cub::DeviceScan::ExclusiveSum(w->cub_tmp, bytes, w->surv, w->surv_before, (int)np_bound, s);
    k_compact_swap_map<<<nb, T, 0, s>>>(w->lost, w->surv_before, cnt, w->map);
    spiffe_note_launches(1);
    k_compact_swap_move<<<nb, T, 0, s>>>(*b, w->lost, w->surv_before, cnt, w->map);
    spiffe_note_launches(1);
    k_compact_swap_finish<<<1, 1, 0, s>>>(cnt);
    spiffe_note_launches(1);
  }
  return (int)cudaGetLastError();
}
