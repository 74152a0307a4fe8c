// spiffe_b200/csrc/reduce.cu -- the status row's FP64 reductions on the device.
//
// do_status_printouts (status_pr.c:18-356), kinetic_energy and field_energy
// (:342-452): the beam's charge, kinetic energy, moments and extremes and the
// fields' energies and extreme values, computed where the state lives so a
// status row reads back a few doubles instead of every field and particle.
//
// The reference's sums are sequential loops, and the FP64 form must give its
// numbers bit for bit (compiled with -fmad=false), so every order-dependent
// sum keeps the reference's order:
//   * field energies: one thread per column sums that column over iz as the
//     reference's inner loop does, and one thread then adds the column sums
//     in the reference's order of columns and terms;
//   * beam sums (charge, the kinetic-energy sum, the moment sums of z, r, pz,
//     pr): each is one serial chain over the particles, and the chains run
//     side by side, one warp each;
// extremes are order-free and reduced in parallel.
#include <cfloat>

#include "split32.cuh"

namespace {

// one column's serial sums: [0] Ez^2, [1] Er^2, [2] Bphi2^2, [3] Ephi^2,
// [4] Br2^2, [5] Bz2^2 (each over the reference's rows, skipping the nodes
// whose flag holds that component at zero), and the column's extremes of
// Ez + EzImposed (rows 1..nz-1) and Er + ErImposed (rows 0..nz-1)
template <typename T>
struct FieldView {
  const T *Ez, *Er, *Bphi2, *EzI, *ErI, *Ephi, *Br2, *Bz2;
  const int16_t *flags;
  int P, fP; // pitch of the field arrays and of the flags
};

template <typename T>
__global__ void k_energy_columns(FieldView<T> v, int nz, int nr, int tm, int te, double *cols)
{
  const int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir >= nr)
    return;
  double s[6] = {0, 0, 0, 0, 0, 0};
  double ezlo = DBL_MAX, ezhi = -DBL_MAX, erlo = DBL_MAX, erhi = -DBL_MAX;
  for (int iz = 0; iz < nz; iz++) {
    const size_t i = (size_t)iz * v.P + ir;
    const int16_t fl = v.flags[(size_t)iz * v.fP + ir];
    if (tm) {
      const double ez = (double)v.Ez[i], er = (double)v.Er[i];
      if (iz >= 1) {
        const double e = ez + (double)v.EzI[i];
        ezlo = e < ezlo ? e : ezlo;
        ezhi = e > ezhi ? e : ezhi;
        if (!(fl & SPIFFE_FL_EZ_ZERO))
          s[0] += ez * ez;
      }
      const double e = er + (double)v.ErI[i];
      erlo = e < erlo ? e : erlo;
      erhi = e > erhi ? e : erhi;
      if (ir >= 1 && !(fl & SPIFFE_FL_ER_ZERO))
        s[1] += er * er;
      if (ir >= 1 && iz >= 1 && !(fl & SPIFFE_FL_BPHI_ZERO)) {
        const double b = (double)v.Bphi2[i];
        s[2] += b * b;
      }
    }
    if (te) {
      if (!(fl & SPIFFE_FL_EPHI_ZERO)) {
        const double e = (double)v.Ephi[i];
        s[3] += e * e;
      }
      if (iz >= 1 && !(fl & SPIFFE_FL_BR_ZERO)) {
        const double b = (double)v.Br2[i];
        s[4] += b * b;
      }
      if (ir >= 1 && !(fl & SPIFFE_FL_BZ_ZERO)) {
        const double b = (double)v.Bz2[i];
        s[5] += b * b;
      }
    }
  }
  for (int k = 0; k < 6; k++)
    cols[(size_t)k * nr + ir] = s[k];
  cols[(size_t)6 * nr + ir] = ezlo;
  cols[(size_t)7 * nr + ir] = ezhi;
  cols[(size_t)8 * nr + ir] = erlo;
  cols[(size_t)9 * nr + ir] = erhi;
}

// out: [0] electric energy, [1] magnetic energy, [2] EzAbsMax, [3] ErAbsMax
__global__ void k_energy_finish(const double *cols, int nr, double dz, double dr, int tm, int te, double *out)
{
  if (threadIdx.x != 0)
    return;
  const double dr2 = dr * dr;
  // calculate_areas (integrate.c:689-701)
  auto area_c = [&](int ir) { return ir ? SPIFFE_PIx2 * ir * dr2 : SPIFFE_PI * dr2 / 4; };
  auto area_o = [&](int ir) { return SPIFFE_PI * (2 * ir - 1) * dr2; };
  double E0 = 0, E1 = 0, ezAbs = 0, erAbs = 0;
  if (tm) {
    double lo = DBL_MAX, hi = -DBL_MAX;
    for (int ir = 0; ir < nr; ir++) {
      lo = fmin(lo, cols[(size_t)6 * nr + ir]);
      hi = fmax(hi, cols[(size_t)7 * nr + ir]);
    }
    ezAbs = fabs(lo) > fabs(hi) ? fabs(lo) : fabs(hi);
    lo = DBL_MAX;
    hi = -DBL_MAX;
    for (int ir = 0; ir < nr; ir++) {
      lo = fmin(lo, cols[(size_t)8 * nr + ir]);
      hi = fmax(hi, cols[(size_t)9 * nr + ir]);
    }
    erAbs = fabs(lo) > fabs(hi) ? fabs(lo) : fabs(hi);
    // field_energy (status_pr.c:380-410), the reference's order of terms
    for (int ir = 0; ir < nr; ir++)
      E0 += cols[ir] * area_c(ir) * dz * SPIFFE_EPSILON_O / 2;
    for (int ir = 1; ir < nr; ir++)
      E0 += cols[(size_t)nr + ir] * area_o(ir) * dz * SPIFFE_EPSILON_O / 2;
    for (int ir = 1; ir < nr; ir++)
      E1 += cols[(size_t)2 * nr + ir] * area_o(ir) * dz / (2 * SPIFFE_MU_O);
  }
  if (te) {
    for (int ir = 0; ir < nr; ir++)
      E0 += cols[(size_t)3 * nr + ir] * area_c(ir) * dz * SPIFFE_EPSILON_O / 2;
    for (int ir = 0; ir < nr; ir++)
      E1 += cols[(size_t)4 * nr + ir] * area_c(ir) * dz / (2 * SPIFFE_MU_O);
    for (int ir = 1; ir < nr; ir++)
      E1 += cols[(size_t)5 * nr + ir] * area_o(ir) * dz / (2 * SPIFFE_MU_O);
  }
  out[0] = E0;
  out[1] = E1;
  out[2] = ezAbs;
  out[3] = erAbs;
}

// the beam as FP64 values, from either form's layout
struct Beam64View {
  DevBeam64 b;
  __device__ double z(long i) const { return b.z[i]; }
  __device__ double r(long i) const { return b.r[i]; }
  __device__ double pz(long i) const { return b.pz[i]; }
  __device__ double pr(long i) const { return b.pr[i]; }
  __device__ double rpp(long i) const { return b.r_pphi[i]; }
  __device__ double Q(long i) const { return b.Q[i]; }
  __device__ bool active(long i) const { return b.status[i] & SPIFFE_PART_ACTIVE; }
  __device__ int gen(long i) const { return b.generation[i]; }
};

struct Beam32View {
  DevBeam32 b;
  double zmin, dz, dr;
  __device__ double z(long i) const { return zmin + ((double)s32_iz(b.cell[i]) + (double)b.fz[i]) * dz; }
  __device__ double r(long i) const { return ((double)s32_ir(b.cell[i]) + (double)b.fr[i]) * dr; }
  __device__ double pz(long i) const { return b.pz[i]; }
  __device__ double pr(long i) const { return b.pr[i]; }
  __device__ double rpp(long i) const { return b.rpphi[i]; }
  __device__ double Q(long i) const { return b.Q[i]; }
  __device__ bool active(long i) const { return b.status[i] & S32_ACTIVE; }
  __device__ int gen(long i) const { return b.generation[i]; }
};

enum { BQ, BSEC, BKE, BZ_AVE, BZ_RMS, BZ_SD, BR_AVE, BR_RMS, BR_SD, BPZ_AVE, BPZ_RMS, BPZ_SD, BPR_AVE, BPR_RMS,
       BPR_SD, BZ_MIN, BZ_MAX, BR_MIN, BR_MAX, BPZ_MIN, BPZ_MAX, BPR_MIN, BPR_MAX, BEAM_OUT };

// computeMoments' sums in its order (the moment restatement the status file uses)
template <typename V, typename Get>
__device__ void moments_chain(const V &v, long n, Get get, double *ave, double *rms, double *sd)
{
  double s = 0, s2 = 0, d = 0;
  for (long i = 0; i < n; i++) {
    const double x = get(v, i);
    s += x;
    s2 += x * x;
  }
  const double m = s / n;
  for (long i = 0; i < n; i++) {
    const double x = get(v, i);
    d += (x - m) * (x - m);
  }
  *ave = m;
  *rms = sqrt(s2 / n);
  *sd = n > 1 ? sqrt(d / (n - 1)) : 0;
}

// six warps: warp w's first lane runs serial chain w; the extremes are
// reduced by every thread
template <typename V>
__global__ void __launch_bounds__(192) k_beam_status(V v, const DevCounts *cnt, double stiffness, double *out)
{
  const long n = (long)cnt->np;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0 && n > 0) {
    if (w == 0) {
      double Q = 0;
      long long sec = 0;
      for (long i = 0; i < n; i++)
        if (v.active(i)) {
          Q += v.Q(i);
          if (v.gen(i) > 0)
            sec++;
        }
      out[BQ] = Q;
      out[BSEC] = (double)sec;
    } else if (w == 1) {
      // kinetic_energy (status_pr.c:342-359)
      double sum = 0;
      for (long i = 0; i < n; i++) {
        const double r = v.r(i), pz = v.pz(i), pr = v.pr(i);
        const double a = r ? v.rpp(i) / r : 0;
        sum += sqrt(1 + pz * pz + pr * pr + a * a);
      }
      out[BKE] = stiffness * SPIFFE_ME_MKS * (SPIFFE_C_MKS * SPIFFE_C_MKS) * (sum - n);
    } else if (w == 2) {
      moments_chain(v, n, [](const V &u, long i) { return u.z(i); }, out + BZ_AVE, out + BZ_RMS, out + BZ_SD);
    } else if (w == 3) {
      moments_chain(v, n, [](const V &u, long i) { return u.r(i); }, out + BR_AVE, out + BR_RMS, out + BR_SD);
    } else if (w == 4) {
      moments_chain(v, n, [](const V &u, long i) { return u.pz(i); }, out + BPZ_AVE, out + BPZ_RMS, out + BPZ_SD);
    } else if (w == 5) {
      moments_chain(v, n, [](const V &u, long i) { return u.pr(i); }, out + BPR_AVE, out + BPR_RMS, out + BPR_SD);
    }
  }
  // extremes of z, r, pz, pr over all np particles (find_min_max)
  __shared__ double lo[4][192], hi[4][192];
  double l[4] = {DBL_MAX, DBL_MAX, DBL_MAX, DBL_MAX}, h[4] = {-DBL_MAX, -DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    const double x[4] = {v.z(i), v.r(i), v.pz(i), v.pr(i)};
    for (int k = 0; k < 4; k++) {
      l[k] = x[k] < l[k] ? x[k] : l[k];
      h[k] = x[k] > h[k] ? x[k] : h[k];
    }
  }
  for (int k = 0; k < 4; k++) {
    lo[k][threadIdx.x] = l[k];
    hi[k][threadIdx.x] = h[k];
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int k = threadIdx.x;
    double a = DBL_MAX, b = -DBL_MAX;
    for (int t = 0; t < (int)blockDim.x; t++) {
      a = lo[k][t] < a ? lo[k][t] : a;
      b = hi[k][t] > b ? hi[k][t] : b;
    }
    out[BZ_MIN + 2 * k] = a;
    out[BZ_MIN + 2 * k + 1] = b;
  }
}

} // namespace

// Fills the status row's field and beam values (do_status_printouts'
// numbers) from device state; `scratch` holds 10 nr + 32 doubles.
extern "C" int spiffe_status_device(const DevMesh *m, bool split, const void *fields, const int16_t *flags, int fpitch,
                                    const void *beam, const DevCounts *cnt, double stiffness, double *scratch,
                                    double *host_out, cudaStream_t s)
{
  const int nz = m->nz, nr = m->nr;
  const int tm = (m->modes & SPIFFE_FL_TM_FIELDS) != 0, te = (m->modes & SPIFFE_FL_TE_FIELDS) != 0;
  double *cols = scratch, *out = scratch + (size_t)10 * nr;
  const int nb = (nr + 127) / 128;
  if (split) {
    const DevFields32 &f = *(const DevFields32 *)fields;
    FieldView<float> v{f.Ez, f.Er, f.Bphi2, f.EzImposed, f.ErImposed, f.Ephi, f.Br2, f.Bz2, flags, m->pitch, fpitch};
    k_energy_columns<float><<<nb, 128, 0, s>>>(v, nz, nr, tm, te, cols);
    Beam32View bv{*(const DevBeam32 *)beam, m->zmin, m->dz, m->dr};
    k_beam_status<Beam32View><<<1, 192, 0, s>>>(bv, cnt, stiffness, out + 4);
  } else {
    const DevFields<double> &f = *(const DevFields<double> *)fields;
    FieldView<double> v{f.Ez, f.Er, f.Bphi2, f.EzImposed, f.ErImposed, f.Ephi, f.Br2, f.Bz2, flags, m->pitch, fpitch};
    k_energy_columns<double><<<nb, 128, 0, s>>>(v, nz, nr, tm, te, cols);
    Beam64View bv{*(const DevBeam64 *)beam};
    k_beam_status<Beam64View><<<1, 192, 0, s>>>(bv, cnt, stiffness, out + 4);
  }
  k_energy_finish<<<1, 32, 0, s>>>(cols, nr, m->dz, m->dr, tm, te, out);
  spiffe_note_launches(3);
  cudaError_t e = cudaMemcpyAsync(host_out, out, sizeof(double) * (4 + BEAM_OUT), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  return (int)e;
}

// ---- exit-plane moments of a screen's records (no counterpart in the
// reference, which leaves moments to external tools): with weights |q|,
//   charge = sum q, mean kinetic energy m c^2 <gamma - 1> and its rms spread,
//   rms bunch length sigma_t <beta_z> c, and the normalized rms emittance of
//   the x projection of the axisymmetric beam, <x^2> = <r^2>/2,
//   <px^2> = (<pr^2> + <pphi^2>)/2, <x px> = <r pr>/2 (momenta in m c).
// Two passes of per-block partial sums, each finished in a fixed order, so
// the result does not depend on timing.
namespace {

constexpr int MOM_NT = 256, MOM_BLOCKS = 148;
constexpr double MC2_EV = 0.51099895000e6; // electron rest energy, eV
constexpr int MOM_S1 = 9, MOM_S2 = 2;

__device__ __forceinline__ double gamma_of(const DevScreen &s, long i)
{
  const double pz = s.col[1][i], pr = s.col[2][i], pp = s.col[3][i];
  return sqrt(1 + pz * pz + pr * pr + pp * pp);
}

// pass 1: sum|q|, sum q, sum|q| ke, sum|q| t, sum|q| pz/gamma, sum|q| r^2,
// sum|q| pr^2, sum|q| pphi^2, sum|q| r pr
__global__ void __launch_bounds__(MOM_NT) k_moments1(DevScreen s, const long long *nb, double *part)
{
  __shared__ double sh[MOM_S1][MOM_NT];
  const long n = (long)min(*nb, (long long)s.capacity);
  double a[MOM_S1] = {0};
  for (long i = (long)blockIdx.x * MOM_NT + threadIdx.x; i < n; i += (long)gridDim.x * MOM_NT) {
    const double q = s.col[5][i], w = fabs(q), g = gamma_of(s, i), r = s.col[0][i];
    const double pz = s.col[1][i], pr = s.col[2][i], pp = s.col[3][i];
    a[0] += w;
    a[1] += q;
    a[2] += w * (MC2_EV * (g - 1));
    a[3] += w * s.col[4][i];
    a[4] += w * (pz / g);
    a[5] += w * (r * r);
    a[6] += w * (pr * pr);
    a[7] += w * (pp * pp);
    a[8] += w * (r * pr);
  }
  for (int k = 0; k < MOM_S1; k++)
    sh[k][threadIdx.x] = a[k];
  __syncthreads();
  if (threadIdx.x < MOM_S1) {
    double t = 0;
    for (int j = 0; j < MOM_NT; j++)
      t += sh[threadIdx.x][j];
    part[(size_t)blockIdx.x * MOM_S1 + threadIdx.x] = t;
  }
}

__global__ void k_moments_sum(const double *part, int blocks, int nsum, double *tot)
{
  if (threadIdx.x < nsum) {
    double t = 0;
    for (int b = 0; b < blocks; b++)
      t += part[(size_t)b * nsum + threadIdx.x];
    tot[threadIdx.x] = t;
  }
}

// pass 2: sum|q| (ke - <ke>)^2, sum|q| (t - <t>)^2
__global__ void __launch_bounds__(MOM_NT) k_moments2(DevScreen s, const long long *nb, const double *tot1,
                                                      double *part)
{
  __shared__ double sh[MOM_S2][MOM_NT];
  const long n = (long)min(*nb, (long long)s.capacity);
  const double W = tot1[0], ke_m = W ? tot1[2] / W : 0, t_m = W ? tot1[3] / W : 0;
  double a[MOM_S2] = {0};
  for (long i = (long)blockIdx.x * MOM_NT + threadIdx.x; i < n; i += (long)gridDim.x * MOM_NT) {
    const double w = fabs(s.col[5][i]);
    const double dk = MC2_EV * (gamma_of(s, i) - 1) - ke_m, dt = s.col[4][i] - t_m;
    a[0] += w * (dk * dk);
    a[1] += w * (dt * dt);
  }
  for (int k = 0; k < MOM_S2; k++)
    sh[k][threadIdx.x] = a[k];
  __syncthreads();
  if (threadIdx.x < MOM_S2) {
    double t = 0;
    for (int j = 0; j < MOM_NT; j++)
      t += sh[threadIdx.x][j];
    part[(size_t)blockIdx.x * MOM_S2 + threadIdx.x] = t;
  }
}

// out: count, charge, mean kinetic energy (eV), rms energy spread (eV), rms
// bunch length (m), normalized emittance (m)
__global__ void k_moments_finish(const long long *nb, long long capacity, const double *t1, const double *t2,
                                 double *out)
{
  const long long n = *nb < capacity ? *nb : capacity;
  const double W = t1[0];
  out[0] = (double)n;
  out[1] = t1[1];
  if (n == 0 || W == 0) {
    out[1] = out[2] = out[3] = out[4] = out[5] = 0;
    return;
  }
  out[2] = t1[2] / W;
  out[3] = sqrt(t2[0] / W);
  out[4] = sqrt(t2[1] / W) * (t1[4] / W) * SPIFFE_C_MKS;
  const double x2 = t1[5] / W / 2, px2 = (t1[6] / W + t1[7] / W) / 2, xpx = t1[8] / W / 2;
  out[5] = sqrt(fmax(x2 * px2 - xpx * xpx, 0.0));
}

} // namespace

// scratch: MOM_BLOCKS * 9 + 32 doubles
extern "C" int spiffe_screen_moments_device(const DevScreen *scr, const long long *nb, double *scratch,
                                            double *host_out, cudaStream_t s)
{
  double *part = scratch, *t1 = scratch + (size_t)MOM_BLOCKS * MOM_S1, *t2 = t1 + 16, *out = t2 + 8;
  k_moments1<<<MOM_BLOCKS, MOM_NT, 0, s>>>(*scr, nb, part);
  k_moments_sum<<<1, 32, 0, s>>>(part, MOM_BLOCKS, MOM_S1, t1);
  k_moments2<<<MOM_BLOCKS, MOM_NT, 0, s>>>(*scr, nb, t1, part);
  k_moments_sum<<<1, 32, 0, s>>>(part, MOM_BLOCKS, MOM_S2, t2);
  k_moments_finish<<<1, 1, 0, s>>>(nb, scr->capacity, t1, t2, out);
  spiffe_note_launches(5);
  cudaError_t e = cudaMemcpyAsync(host_out, out, sizeof(double) * 6, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  return (int)e;
}
