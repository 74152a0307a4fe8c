// spiffe_b200/csrc/emit.cu -- cathode births and antenna current on the device.
//
// The host decides how many macroparticles a cathode emits this step (the
// reference's count logic, cathode.c:349-422, runs in runtime.cu with the
// shared counter-based generator); this kernel writes the births straight
// into the device beam, one thread per birth, drawing radius k from the
// generator at counter base+k+1 so the stream is consumed exactly as the
// serial reference consumes it (cathode.c:464-659).  Built with -fmad=false.
#include "modules.cuh"

#include "../../include/spiffe_b200_rng.h"



namespace {

constexpr int T = 256;

__global__ void __launch_bounds__(T) k_births(DevMesh m, DevFields<double> f, DevBeam64 b, BirthParams p, DevCounts *cnt)
{
  const long long k = (long long)blockIdx.x * T + threadIdx.x;
  if (k >= p.total)
    return;
  const long long np = cnt->np;
  if (np + p.total > b.capacity) {
    if (k == 0)
      atomicOr(&cnt->error, SPIFFE_DEV_ERR_CAPACITY);
    return;
  }
  const long long ip = np + k;
  const double c = SPIFFE_C_MKS;
  if (p.mode == SPIFFE_BIRTH_LIST) {
    // emitSecondaryElectrons (secondaryEmission.c:471-497): the host drew the
    // momenta; position and birth position are the loss point
    const double *L = p.list;
    const long long n = p.total;
    b.z[ip] = b.z0[ip] = L[k];
    b.r[ip] = b.r0[ip] = L[n + k];
    b.pz[ip] = L[2 * n + k];
    b.pr[ip] = L[3 * n + k];
    b.vz[ip] = L[4 * n + k];
    b.vr[ip] = L[5 * n + k];
    b.Q[ip] = L[6 * n + k];
    b.t0[ip] = L[7 * n + k];
    b.generation[ip] = (int16_t)L[8 * n + k];
    b.particleID[ip] = (int32_t)L[9 * n + k];
    b.vphi[ip] = b.r_pphi[ip] = 0;
    b.rmin[ip] = b.zmin[ip] = 1.7976931348623157e308;
    b.rmax[ip] = b.zmax[ip] = -1.7976931348623157e308;
    b.status[ip] = SPIFFE_PART_ACTIVE;
    return;
  }
  if (p.mode == SPIFFE_BIRTH_TEST) {
    // test_beam.c:91-103 sets position, momenta, velocities and charge only;
    // every other per-particle value is what a fresh (zeroed) slot holds, and
    // the push activates the particle (advance_particles.c:165-187)
    const double r = p.inner_radius, pz = p.pz0, pr = p.pr0, r_pphi = p.rpphi0;
    double gamma, vphi;
    if (r) {
      gamma = sqrt(pz * pz + pr * pr + (r_pphi / r) * (r_pphi / r) + 1);
      vphi = c * r_pphi / r / gamma;
    } else {
      gamma = sqrt(pz * pz + pr * pr + 1);
      vphi = 0;
    }
    b.z[ip] = p.z_position;
    b.r[ip] = r;
    b.pz[ip] = pz;
    b.pr[ip] = pr;
    b.r_pphi[ip] = r_pphi;
    b.vz[ip] = c * pz / gamma;
    b.vr[ip] = c * pr / gamma;
    b.vphi[ip] = vphi;
    b.Q[ip] = p.Q;
    b.z0[ip] = b.r0[ip] = b.t0[ip] = 0;
    b.rmin[ip] = b.rmax[ip] = b.zmin[ip] = b.zmax[ip] = 0;
    b.particleID[ip] = 0;
    b.generation[ip] = 0;
    b.status[ip] = 0;
    return;
  }
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
    r = sqrt(rn * (p.outer_radius * p.outer_radius - p.inner_radius * p.inner_radius) + p.inner_radius * p.inner_radius);
    dte = m.dt * (double)k / (1.0 * p.total);
  } else {
    r = sqrt(p.inner_r2 + (double)(k + 1) * p.dr2);
    dte = m.dt * (double)k / (1.0 * p.total);
  }
  // cathode.c:466-488
  double vz = p.initial_vz, vr = 0, vphi = p.initial_omega * r;
  double gamma = 1 / sqrt(1 - (vz / c) * (vz / c) - (vr / c) * (vr / c) - (vphi / c) * (vphi / c));
  double pz = vz / c * gamma, pr = vr / c * gamma, r_pphi = r * vphi / c * gamma;
  double z = p.z_position, t0 = p.time;
  if (p.spread) {
    // cathode.c:490-518: partial kick by the local Ez, Er over dte
    const int P = m.pitch;
    long iz = (long)((p.z_position - m.zmin) / m.dz);
    if (iz <= 0)
      iz = 1;
    if (iz > m.nz)
      iz = m.nz;
    long ir = (long)(r / m.dr);
    double Ez = m.constE[0], Er = m.constE[1];
    if (m.modes & SPIFFE_FL_TM_FIELDS)
      Ez = f.Ez[node((int)iz, (int)ir, P)] + f.EzImposed[node((int)iz, (int)ir, P)];
    ir += 1;
    iz -= 1;
    if (m.modes & SPIFFE_FL_TM_FIELDS)
      Er = f.Er[node((int)iz, (int)ir, P)] + f.ErImposed[node((int)iz, (int)ir, P)];
    t0 -= dte;
    const double pphi = (r ? r_pphi / r : 0);
    z += vz * dte;
    r += vr * dte;
    pr += dte * p.QoMC * Er / p.stiffness;
    pz += dte * p.QoMC * Ez / p.stiffness;
    gamma = sqrt(pz * pz + pr * pr + pphi * pphi + 1);
    vz = c * pz / gamma;
    vr = c * pr / gamma;
  }
  b.particleID[ip] = (int32_t)(cnt->nextParticleID + k);
  b.rmin[ip] = b.zmin[ip] = 1.7976931348623157e308;
  b.rmax[ip] = b.zmax[ip] = -1.7976931348623157e308;
  b.z[ip] = z;
  b.z0[ip] = z;
  b.r[ip] = r;
  b.r0[ip] = r;
  b.t0[ip] = t0;
  b.generation[ip] = 0;
  b.Q[ip] = p.Q;
  b.vz[ip] = vz;
  b.vr[ip] = vr;
  b.vphi[ip] = vphi;
  b.pz[ip] = pz;
  b.pr[ip] = pr;
  b.r_pphi[ip] = r_pphi;
  b.status[ip] = SPIFFE_PART_ACTIVE;
}

__global__ void k_births_commit(long long total, long long capacity, int mode, DevCounts *cnt)
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

__global__ void k_antenna(double *J, int P, int direction, long istart, long iend, long iposition, double value)
{
  const long i = istart + (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > iend)
    return;
  // antenna.c:398-415
  if (direction == 1)
    J[node((int)iposition, (int)i, P)] += value;
  else
    J[node((int)i, (int)iposition, P)] += value;
}

} // namespace

extern "C" int spiffe_births64(const DevMesh *m, const DevFields<double> *f, const DevBeam64 *b, const BirthParams *p,
                               DevCounts *cnt, cudaStream_t s)
{
  if (p->total <= 0)
    return 0;
  k_births<<<blocks_for(p->total, T), T, 0, s>>>(*m, *f, *b, *p, cnt);
  spiffe_note_launches(1);
  k_births_commit<<<1, 1, 0, s>>>(p->total, b->capacity, p->mode, cnt);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int spiffe_antenna64(double *J, int pitch, int direction, long istart, long iend, long iposition, double value,
                                cudaStream_t s)
{
  if (iend < istart)
    return 0;
  const long n = iend - istart + 1;
  k_antenna<<<blocks_for(n, 128), 128, 0, s>>>(J, pitch, direction, istart, iend, iposition, value);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}
