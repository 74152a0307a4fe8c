// spiffe_b200/csrc/poisson_f64.cu -- plain FP64 Poisson correction.
//
// add_poisson_correction (poisson_correction.c:73-454), solve_poisson_cyl
// (poisson.c:17-130) and compute_imposed_Efield (poisson_correction.c:
// 456-562) as device kernels.  The decision whether to solve (the error-
// charge threshold, :258-265) is taken on the device, so a correction needs
// no host round trip.  The red-black SOR runs as one persistent cooperative
// kernel: each half-sweep updates one colour (the reference's colour test,
// poisson.c:70), every block reduces its |residual| sum, and after a grid
// barrier all blocks add the per-block sums in the same fixed order and take
// the same stop decision (poisson.c:120-121).  Node updates are bit-identical
// to the reference (a colour's nodes read only the other colour); the stop
// sum is reduced in a fixed tree order rather than the reference's serial
// order, which changes the half-sweep count only if the sum lands within
// rounding distance of the threshold.  Built with -fmad=false.
#include "modules.cuh"

#include <cooperative_groups.h>

namespace {

constexpr int BX = 32, BY = 8, RT = 256;

// Fixed-order block reduction of one double per thread (blockDim.x*y <= 1024).
__device__ double block_sum(double v, double *sh)
{
  const int t = threadIdx.y * blockDim.x + threadIdx.x, n = blockDim.x * blockDim.y;
  sh[t] = v;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if (t < s && t + s < n)
      sh[t] += sh[t + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

__device__ bool surface_cell(const DevMesh &m, int16_t fl, int iz, int ir)
{
  return (fl & SPIFFE_FL_IS_METAL) || (iz == 0 && m.left_bc == SPIFFE_NEUMANN) ||
         (iz == m.nz - 1 && m.right_bc == SPIFFE_NEUMANN) || (ir == m.nr - 1 && m.upper_bc == SPIFFE_NEUMANN);
}

// Apparent charge from the flux of E through each cell (:141-182, second pass
// :335-375, where the top-row surface term changes sign).  Per-block partial
// sums of Qsurface and the centroid numerator go to part[2*block+{0,1}].
__global__ void __launch_bounds__(BX *BY) k_apparent_charge(DevMesh m, DevFields<double> f, const double *Az_,
                                                             const double *Ari, const double *Aro, int second,
                                                             double *part)
{
  __shared__ double sh[BX * BY];
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  const double eps = SPIFFE_EPSILON_O;
  double qs = 0, cen = 0;
  if (ir < nr && iz < nz) {
    const size_t i = node(iz, ir, P);
    const double Az = Az_[ir], Ar_inner = Ari[ir], Ar_outer = Aro[ir];
    double dQ;
    if (ir == 0)
      dQ = (f.Er[i + 1] * Ar_outer + (f.Ez[i + P] - f.Ez[i]) * Az) * eps;
    else
      dQ = (f.Er[i + 1] * Ar_outer - f.Er[i] * Ar_inner + (f.Ez[i + P] - f.Ez[i]) * Az) * eps;
    if (surface_cell(m, f.flags[i], iz, ir)) {
      if (iz == 0)
        dQ += f.Ez[i] * Az * eps;
      if (iz == nz - 1)
        dQ -= f.Ez[i + P] * Az * eps;
      if (ir == nr - 1) {
        if (second)
          dQ -= f.Ez[i + 1] * Ar_outer * eps;
        else
          dQ += f.Ez[i + 1] * Ar_outer * eps;
      }
      qs = dQ;
      f.Q[i] = 0;
    } else {
      f.Q[i] = dQ;
      cen = dQ * (iz * m.dz + m.zmin);
    }
  }
  const double s0 = block_sum(qs, sh), s1 = block_sum(cen, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int b = blockIdx.y * gridDim.x + blockIdx.x;
    part[2 * b] = s0;
    part[2 * b + 1] = s1;
  }
}

// Removal of the particles' own charge (:190-242); Qreal partial sums per
// block.  With keys null each share is subtracted by an FP64 atomic, whose
// order varies between runs once three or more particles share a node; with
// keys set, particle ip writes its four (node, -share) pairs to entries
// 4 ip .. 4 ip + 3 (unused ones keyed INT_MAX) for an ordered reduction that
// applies them in particle order, the reference's serial Q[iz][ir] -= ...
// sequence.
__global__ void __launch_bounds__(RT) k_remove_charge(DevMesh m, DevFields<double> f, DevBeam64 b,
                                                       const DevCounts *cnt, double *part, int *keys, double *vals,
                                                       long np_bound)
{
  __shared__ double sh[RT];
  const long ip = (long)blockIdx.x * RT + threadIdx.x;
  double qreal = 0;
  int at[4] = {0x7fffffff, 0x7fffffff, 0x7fffffff, 0x7fffffff};
  double share[4] = {0, 0, 0, 0};
  if (ip < (long)cnt->np && (b.status[ip] & SPIFFE_PART_ACTIVE)) {
    const long nz = m.nz, nr = m.nr;
    const int P = m.pitch;
    const double dz = m.dz, dr = m.dr;
    const bool lsm = m.modes & SPIFFE_FL_LONGIT_SMEAR, rsm = m.modes & SPIFFE_FL_RADIAL_SMEAR;
    const bool ln = m.left_bc == SPIFFE_NEUMANN, rn = m.right_bc == SPIFFE_NEUMANN, un = m.upper_bc == SPIFFE_NEUMANN;
    const double z = b.z[ip], r = b.r[ip], Q = b.Q[ip];
    const long iz = lsm ? (long)((z - m.zmin) / dz) : (long)((z - m.zmin) / dz + 0.5);
    const long ir = rsm ? (long)(r / dr) : (long)(r / dr + 0.5);
    if (iz >= 0 && iz < nz && ir >= 0 && ir < nr) {
      double fa, fb, fr, fl;
      if (rsm && ir != nr - 1) {
        fa = r / dr - ir;
        fb = 1 - fa;
      } else {
        fb = 1;
        fa = 0;
      }
      if (lsm && iz != nz - 1) {
        fr = (z - m.zmin) / dz - iz;
        fl = 1 - fr;
      } else {
        fl = 1;
        fr = 0;
      }
      const int16_t *F = f.flags;
      const int n0 = node(iz, ir, P), n1 = node(iz + 1, ir, P), n2 = node(iz, ir + 1, P), n3 = node(iz + 1, ir + 1, P);
      if (!((F[n0] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz - 1 && rn) || (ir >= nr - 1 && un))) {
        at[0] = n0;
        share[0] = Q * fb * fl;
        qreal += share[0];
      }
      if (!((F[n1] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz && rn) || (ir >= nr - 1 && un))) {
        at[1] = n1;
        share[1] = Q * fb * fr;
        qreal += share[1];
      }
      if (!((F[n2] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz - 1 && rn) || (ir >= nr && un))) {
        at[2] = n2;
        share[2] = Q * fa * fl;
        qreal += share[2];
      }
      if (!((F[n3] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz && rn) || (ir >= nr && un))) {
        at[3] = n3;
        share[3] = Q * fa * fr;
        qreal += share[3];
      }
    }
  }
  if (keys) {
    if (ip < np_bound)
      for (int k = 0; k < 4; k++) {
        keys[4 * ip + k] = at[k];
        vals[4 * ip + k] = at[k] == 0x7fffffff ? 0.0 : -share[k];
      }
  } else {
    for (int k = 0; k < 4; k++)
      if (at[k] != 0x7fffffff)
        atomicAdd(f.Q + at[k], -share[k]);
  }
  const double s = block_sum(qreal, sh);
  if (threadIdx.x == 0)
    part[blockIdx.x] = s;
}

// Sum over a (rows x cols) window of a pitched array, |x| when absval.
__global__ void __launch_bounds__(BX *BY) k_region_sum(const double *a, int rows, int cols, int P, int absval,
                                                        double *part)
{
  __shared__ double sh[BX * BY];
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  double v = 0;
  if (ir < cols && iz < rows) {
    v = a[node(iz, ir, P)];
    if (absval)
      v = fabs(v);
  }
  const double s = block_sum(v, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    part[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// Serial fixed-order sum of n partials (strided by `stride`) into *out.
__global__ void k_finish_sum(const double *part, int n, int stride, double *out)
{
  __shared__ double sh[1024];
  double v = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    v += part[(size_t)i * stride];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    *out = sh[0];
}

// error-charge threshold test (:258-265).  The reference sums Qerror
// serially, iz outer and ir inner (:245-248); the device's tree sum of the
// same values differs from it by at most 2 gamma_(n-1) sum|Q| (n terms,
// gamma_k = k u / (1 - k u), u = 2^-53).  When |Qerror| is farther than that
// from a positive threshold the decision is the reference's; otherwise (an
// error charge at the level of rounding noise, as with no particles left)
// this thread redoes the sum in the reference's order.
__global__ void k_pc_decide(PcState *st, double threshold, const double *Q, int nz, int nr, int P,
                            const double *abs_sum)
{
  if (threshold > 0 && abs_sum) {
    const double n = (double)nz * (double)nr, u = 1.1102230246251565e-16;
    const double margin = 2.0 * (n * u / (1.0 - n * u)) * *abs_sum * 1.0001 + 1e-300;
    if (fabs(fabs(st->Qerror) - threshold) <= margin) {
      double q = 0;
      for (int iz = 0; iz < nz; iz++)
        for (int ir = 0; ir < nr; ir++)
          q += Q[node(iz, ir, P)];
      st->Qerror = q;
    }
  }
  const double Qerror = st->Qerror, Qreal = st->Qreal;
  int skip = (threshold > 0 && fabs(Qerror) < threshold) ||
             (threshold < 0 && (Qreal == 0 || fabs(Qerror / Qreal) < fabs(threshold)));
  st->do_solve = !skip;
}

// Q -> -Q/(V eps0) over iz < nz, ir < nr (:268-274)
__global__ void __launch_bounds__(BX *BY) k_scale_rhs(DevMesh m, DevFields<double> f, const double *volume,
                                                       const PcState *st)
{
  if (!st->do_solve)
    return;
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  if (ir < m.nr && iz < m.nz) {
    const size_t i = node(iz, ir, m.pitch);
    f.Q[i] = -f.Q[i] / (volume[ir] * SPIFFE_EPSILON_O);
  }
}

// poisson_guess (:564-615)
__global__ void __launch_bounds__(BX *BY) k_guess(DevMesh m, DevFields<double> f, int code, const PcState *st)
{
  if (!st->do_solve)
    return;
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  if (ir >= m.nr || iz >= m.nz)
    return;
  const size_t i = node(iz, ir, m.pitch);
  const double charge = st->Qerror;
  if (code == 1)
    f.Psi[i] = charge / (SPIFFE_PIx2 * SPIFFE_EPSILON_O) * log((ir ? ir : 0.5) * m.dr);
  else if (code == 2) {
    const double zz = (iz * m.dz + m.zmin) - st->centroid, rr = m.dr * (ir + 0.5);
    const double dist = sqrt(zz * zz + rr * rr);
    f.Psi[i] = charge / (4 * SPIFFE_PI * SPIFFE_EPSILON_O * dist);
  } else if (code == 3)
    f.Psi[i] = 0;
}

// Bounded grid barrier for a cooperative launch: returns false (and raises
// the device error bit) if the other blocks do not arrive within `limit` polls.
__device__ bool grid_barrier(unsigned *count, unsigned *gen, unsigned nblocks, DevCounts *cnt)
{
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    ok = 1;
    volatile unsigned *vgen = gen;
    const unsigned g = *vgen;
    __threadfence();
    if (atomicAdd(count, 1u) == nblocks - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      unsigned long long polls = 0;
      while (*vgen == g) {
        if (++polls > (1ull << 26)) {
          ok = 0;
          atomicOr(&cnt->error, SPIFFE_DEV_ERR_BARRIER);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok;
}

struct SorArgs {
  double *Psi;
  const double *rhs; // null for the Laplace solve of the imposed potential
  const int16_t *flags;
  const double *omega;       // omega[n] for half-sweep n
  const double *crow, *drow; // c and d of each row ir >= 1 (poisson.c:357-358)
  double a, e, c4_axis, e2c_axis, accuracy; // 4c and e-2c of the axis row (poisson.c:361, :386-387)
  const double *driving;     // sum |rhs|
  long long limit;
  double *partials; // 2*gridDim.x doubles
  unsigned *bar_count, *bar_gen;
  PcState *st; // iterations and final residual; do_solve gate (may be null)
  long long *iterations_out;
};

// solve_poisson_cyl (poisson.c:17-130): rows ir = 0..nr-2 of the iz the
// boundary conditions leave free; half-sweep n updates the nodes with
// (ir+iz)%2 == n%2.  Each block owns whole iz rows (block-strided) and its
// threads visit only that row's nodes of the current colour, so a warp reads
// every other Psi of a row.  Psi of neighbouring rows was written by other
// blocks in the previous half-sweep, so it is read through L2 (ld.cg).
__global__ void __launch_bounds__(RT) k_sor(DevMesh m, SorArgs s, DevCounts *cnt)
{
  __shared__ double sh[RT];
  if (s.st && !s.st->do_solve)
    return;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  const int lo = m.left_bc == SPIFFE_DIRICHLET ? 0 : 1, hi = m.right_bc == SPIFFE_DIRICHLET ? nz - 1 : nz - 2;
  const int cols = nr - 1, rows = hi - lo + 1;
  const double a = s.a, e = s.e;
  const double thr = s.accuracy * *s.driving;
  long long result = -1;
  double total = 0;
  for (long long n = 0; n < s.limit; n++) {
    const double omega = s.omega[n];
    const int colour = (int)(n & 1);
    double acc = 0;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
      const int iz = lo + row;
      const int parity = (colour + iz) & 1; // ir with (ir+iz)%2 == colour
      const size_t base = node(iz, 0, P);
      // the left and right Dirichlet rows mirror their only neighbour (poisson.c:369-375, :404-410)
      const long up = (iz == 0 && lo == 0) ? P : (iz == nz - 1 && hi == nz - 1 ? -P : P);
      const long dn = (iz == 0 && lo == 0) ? P : -P;
      for (int ir = 2 * threadIdx.x + parity; ir < cols; ir += 2 * RT) {
        const size_t i = base + ir;
        if (s.flags[i] & SPIFFE_FL_IS_METAL)
          continue;
        const double left = __ldcg(s.Psi + i + up), right = __ldcg(s.Psi + i + dn);
        const double drive = s.rhs ? s.rhs[i] : 0;
        const double self = __ldcg(s.Psi + i);
        double residual;
        if (ir == 0) {
          residual = a * (left + right) + s.c4_axis * __ldcg(s.Psi + i + 1) + s.e2c_axis * self - drive;
          __stcg(s.Psi + i, self - omega * residual / s.e2c_axis);
        } else {
          residual = a * (left + right) + s.crow[ir] * __ldcg(s.Psi + i + 1) + s.drow[ir] * __ldcg(s.Psi + i - 1) +
                     e * self - drive;
          __stcg(s.Psi + i, self - omega * residual / e);
        }
        acc += fabs(residual);
      }
    }
    // partial sums alternate between two halves of the buffer, so a block
    // that runs ahead cannot overwrite sums another block is still reading
    double *part = s.partials + (size_t)(n & 1) * gridDim.x;
    const double bs = block_sum(acc, sh);
    if (threadIdx.x == 0)
      __stcg(part + blockIdx.x, bs);
    __threadfence();
    if (!grid_barrier(s.bar_count, s.bar_gen, gridDim.x, cnt))
      return;
    // every block forms the same fixed-order sum of the partials
    double v = 0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += RT)
      v += __ldcg(part + b);
    total = block_sum(v, sh);
    if (n > 0 && (total < thr || total == 0)) {
      result = n;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (s.iterations_out)
      *s.iterations_out = result;
    if (s.st) {
      s.st->iterations = result;
      s.st->residual = total;
    }
    cnt->sor_halfsweeps += result >= 0 ? result + 1 : s.limit;
    cnt->sor_solves += 1;
  }
}

// Ez, Er -= grad Psi (:288-326) with the FDTD boundary copies; one writer per node.
__global__ void __launch_bounds__(BX *BY) k_subtract_gradient(DevMesh m, DevFields<double> f, const PcState *st)
{
  if (!st->do_solve)
    return;
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (ir > nr || iz > nz)
    return;
  const size_t i = node(iz, ir, P);
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;
  if (ir < nr && iz >= 1 && iz <= nz - 1) {
    double v = f.Ez[i];
    if (!(f.flags[i] & SPIFFE_FL_EZ_ZERO))
      v -= -(f.Psi[i] - f.Psi[i - P]) / m.dz;
    if (ir == nr - 1)
      v = 0.0;
    f.Ez[i] = v;
    if (iz == 1)
      f.Ez[node(0, ir, P)] = ir == nr - 1 ? 0.0 : (leftN ? v : -v);
    if (iz == nz - 1)
      f.Ez[node(nz, ir, P)] = ir == nr - 1 ? 0.0 : (rightN ? v : -v);
  }
  if (iz <= nz - 1) {
    const bool zero_row = (leftN && iz == 0) || (rightN && iz == nz - 1);
    if (ir >= 1) {
      double v = f.Er[i];
      if (!(f.flags[i] & SPIFFE_FL_ER_ZERO))
        v -= -(f.Psi[i] - f.Psi[i - 1]) / m.dr;
      f.Er[i] = zero_row ? 0.0 : v;
      if (ir == 1)
        f.Er[node(iz, 0, P)] = zero_row ? 0.0 : -v;
    }
  }
}

// EzImposed, ErImposed = -factor grad PsiImposed (:523-561).
__global__ void __launch_bounds__(BX *BY) k_imposed_field(DevMesh m, DevFields<double> f, double ff)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (ir > nr || iz > nz)
    return;
  const size_t i = node(iz, ir, P);
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;
  if (ir < nr && iz >= 1 && iz <= nz - 1) {
    double v = f.EzImposed[i];
    if (!(f.flags[i] & SPIFFE_FL_EZ_ZERO))
      v = -ff * (f.PsiImposed[i] - f.PsiImposed[i - P]) / m.dz;
    if (ir == nr - 1)
      v = 0.0;
    f.EzImposed[i] = v;
    if (iz == 1)
      f.EzImposed[node(0, ir, P)] = ir == nr - 1 ? 0.0 : (leftN ? v : -v);
    if (iz == nz - 1)
      f.EzImposed[node(nz, ir, P)] = ir == nr - 1 ? 0.0 : (rightN ? v : -v);
  }
  if (iz <= nz - 1) {
    const bool zero_row = (leftN && iz == 0) || (rightN && iz == nz - 1);
    if (ir >= 1) {
      double v = f.ErImposed[i];
      if (!(f.flags[i] & SPIFFE_FL_ER_ZERO))
        v = -ff * (f.PsiImposed[i] - f.PsiImposed[i - 1]) / m.dr;
      f.ErImposed[i] = zero_row ? 0.0 : v;
      if (ir == 1)
        f.ErImposed[node(iz, 0, P)] = zero_row ? 0.0 : -v;
    }
  }
}

__global__ void k_set_state(PcState *st, double *qs_cen, double *qreal, double *qerr, int space_charge)
{
  st->Qsurface = qs_cen[0];
  st->centroid = qs_cen[1];
  st->Qreal = space_charge ? *qreal : 0.0;
  st->Qerror = *qerr;
}

} // namespace

// ---------------------------------------------------------------- host side


extern "C" int spiffe_poisson64_setup(const DevMesh *m, Poisson64Work *w, long long np_capacity, cudaStream_t s)
{
  const int nr = m->nr, nz = m->nz;
  const double dr = m->dr, dz = m->dz, dr2 = dr * dr, drdz = dr * dz;
  double *Az = new double[nr + 1], *Ari = new double[nr + 1], *Aro = new double[nr + 1], *vol = new double[nr + 1];
  for (int ir = 0; ir <= nr; ir++) {
    if (ir == 0) {
      Ari[ir] = Aro[ir] = SPIFFE_PI * drdz;
      Az[ir] = dr2 / 4 * SPIFFE_PI;
    } else {
      Ari[ir] = SPIFFE_PI * (2 * ir - 1) * drdz;
      Aro[ir] = SPIFFE_PI * (2 * ir + 1) * drdz;
      Az[ir] = SPIFFE_PI * dr2 / 4 * (double)((long)(2 * ir + 1) * (2 * ir + 1) - (long)(2 * ir - 1) * (2 * ir - 1));
    }
    vol[ir] = Az[ir] * dz;
  }
  cudaError_t e = cudaSuccess;
  const size_t gx = (nr + 1 + BX - 1) / BX, gy = (nz + 1 + BY - 1) / BY;
  size_t parts = 2 * gx * gy;
  const size_t pblocks = (size_t)blocks_for(np_capacity > 0 ? np_capacity : 1, RT);
  if (pblocks > parts)
    parts = pblocks;
  if (parts < 4096)
    parts = 4096;
  if (!w->Az) {
    e = cudaMalloc(&w->Az, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->Ari, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->Aro, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->volume, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->scalars, sizeof(double) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&w->bar, sizeof(unsigned) * 2);
    if (e == cudaSuccess) e = cudaMemsetAsync(w->bar, 0, sizeof(unsigned) * 2, s);
    if (e == cudaSuccess) e = cudaMalloc(&w->st, sizeof(PcState));
    if (e == cudaSuccess) e = cudaMemsetAsync(w->st, 0, sizeof(PcState), s);
    if (e == cudaSuccess) e = cudaMalloc(&w->iters, sizeof(long long));
  }
  if (e == cudaSuccess && w->part_n < parts) {
    cudaFree(w->part);
    e = cudaMalloc(&w->part, sizeof(double) * parts);
    w->part_n = parts;
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->Az, Az, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->Ari, Ari, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->Aro, Aro, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->volume, vol, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  // SOR row coefficients with the reference's expressions (poisson.c:355-361)
  double *crow = new double[nr + 1], *drow = new double[nr + 1];
  for (int ir = 0; ir <= nr; ir++) {
    if (ir != 0) {
      crow[ir] = 1 / (dr * dr) * (1 + 1. / (2 * ir));
      drow[ir] = 1 / (dr * dr) * (1 - 1. / (2 * ir));
    } else
      crow[ir] = drow[ir] = 1 / (dr * dr);
  }
  if (e == cudaSuccess && !w->crow) e = cudaMalloc(&w->crow, sizeof(double) * (nr + 1));
  if (e == cudaSuccess && !w->drow) e = cudaMalloc(&w->drow, sizeof(double) * (nr + 1));
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->crow, crow, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->drow, drow, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  delete[] crow;
  delete[] drow;
  delete[] Az;
  delete[] Ari;
  delete[] Aro;
  delete[] vol;
  if (e == cudaSuccess && !w->sor_grid) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sor, RT, 0);
    if (per > 4)
      per = 4;
    w->sor_grid = sms * (per > 0 ? per : 1);
    if ((size_t)(2 * w->sor_grid) > w->part_n)
      w->sor_grid = (int)(w->part_n / 2);
  }
  return (int)e;
}

extern "C" void spiffe_poisson64_free(Poisson64Work *w)
{
  cudaFree(w->Az);
  cudaFree(w->Ari);
  cudaFree(w->Aro);
  cudaFree(w->volume);
  cudaFree(w->part);
  cudaFree(w->scalars);
  cudaFree(w->omega);
  cudaFree(w->bar);
  cudaFree(w->st);
  cudaFree(w->iters);
  cudaFree(w->crow);
  cudaFree(w->drow);
  *w = Poisson64Work();
}

// Chebyshev over-relaxation sequence, poisson.c:342-344, :416-419.
static int ensure_omega(const DevMesh *m, Poisson64Work *w, long long limit, cudaStream_t s)
{
  if (w->omega && w->omega_n >= limit)
    return 0;
  cudaFree(w->omega);
  const double rz = m->dz / m->dr;
  const double rj = (cos(SPIFFE_PI / m->nz) + rz * rz * cos(SPIFFE_PI / m->nr)) / (1 + rz * rz);
  double *om = new double[limit];
  double omega = 1.0;
  for (long long n = 0; n < limit; n++) {
    om[n] = omega;
    if (n == 0)
      omega = 1.0 / (1 - rj * rj / 2);
    else
      omega = 1.0 / (1 - rj * rj * omega / 4);
  }
  cudaError_t e = cudaMalloc(&w->omega, sizeof(double) * limit);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->omega, om, sizeof(double) * limit, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  delete[] om;
  w->omega_n = limit;
  return (int)e;
}

static int sum_region(const double *a, int rows, int cols, int P, int absval, Poisson64Work *w, double *out,
                      cudaStream_t s)
{
  dim3 block(BX, BY), grid((cols + BX - 1) / BX, (rows + BY - 1) / BY);
  if (grid.x * grid.y == 0) {
    cudaMemsetAsync(out, 0, sizeof(double), s);
    return 0;
  }
  k_region_sum<<<grid, block, 0, s>>>(a, rows, cols, P, absval, w->part);
  spiffe_note_launches(1);
  k_finish_sum<<<1, 1024, 0, s>>>(w->part, grid.x * grid.y, 1, out);
  spiffe_note_launches(1);
  return 0;
}

static int launch_sor(const DevMesh *m, Poisson64Work *w, double *Psi, const double *rhs, const int16_t *flags,
                      double accuracy, long long limit, PcState *st, long long *iters, DevCounts *cnt, cudaStream_t s)
{
  int rc = ensure_omega(m, w, limit, s);
  if (rc)
    return rc;
  // sum |rhs| over iz < nz, ir < nr-1 (poisson.c:333-336)
  if (rhs)
    sum_region(rhs, m->nz, m->nr - 1, m->pitch, 1, w, w->scalars + 4, s);
  else
    cudaMemsetAsync(w->scalars + 4, 0, sizeof(double), s);
  SorArgs a;
  a.Psi = Psi;
  a.rhs = rhs;
  a.flags = flags;
  a.omega = w->omega;
  a.a = 1 / (m->dz * m->dz);
  a.e = -2 * (1 / (m->dz * m->dz) + 1 / (m->dr * m->dr));
  a.crow = w->crow;
  a.drow = w->drow;
  const double c_axis = 1 / (m->dr * m->dr);
  a.c4_axis = 4 * c_axis;
  a.e2c_axis = a.e - 2 * c_axis;
  a.accuracy = accuracy;
  a.driving = w->scalars + 4;
  a.limit = limit;
  a.partials = w->part;
  a.bar_count = w->bar;
  a.bar_gen = w->bar + 1;
  a.st = st;
  a.iterations_out = iters;
  DevMesh mm = *m;
  void *args[] = {&mm, &a, &cnt};
  cudaError_t e = cudaLaunchCooperativeKernel((void *)k_sor, dim3(w->sor_grid), dim3(RT), args, 0, s);
  spiffe_note_launches(1);
  return (int)e;
}

// solve_poisson_cyl on device arrays; *iterations receives the reference's
// return value (n, or -1 when the limit was reached) after the stream syncs.
extern "C" int spiffe_sor64(const DevMesh *m, Poisson64Work *w, double *Psi, const double *rhs, const int16_t *flags,
                            double accuracy, long long limit, DevCounts *cnt, long long *iterations, cudaStream_t s)
{
  int rc = launch_sor(m, w, Psi, rhs, flags, accuracy, limit, nullptr, w->iters, cnt, s);
  if (rc)
    return rc;
  if (iterations) {
    cudaMemcpyAsync(iterations, w->iters, sizeof(long long), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
  }
  return (int)cudaGetLastError();
}


// One add_poisson_correction pass (the interval test is the caller's).
extern "C" int spiffe_poisson_correction64(const DevMesh *m, const DevFields<double> *f, const DevBeam64 *b,
                                           DevCounts *cnt, long long np_bound, const PoissonHostOptions *o,
                                           Poisson64Work *w, Particles64Work *pw, bool ordered, cudaStream_t s)
{
  if (ordered && (!pw || !pw->keys || pw->capacity < np_bound))
    return (int)cudaErrorInvalidValue;
  // the particles' own charge leaves Q (:190-242)
  auto remove_charge = [&]() -> int {
    k_remove_charge<<<blocks_for(np_bound, RT), RT, 0, s>>>(*m, *f, *b, cnt, w->part, ordered ? pw->keys : nullptr,
                                                            ordered ? pw->vals : nullptr, (long)np_bound);
    spiffe_note_launches(1);
    return ordered ? spiffe_ordered_add64(pw, 4 * np_bound, f->Q, s) : 0;
  };
  dim3 block(BX, BY), grid((m->nr + 1 + BX - 1) / BX, (m->nz + 1 + BY - 1) / BY);
  const int nblk = grid.x * grid.y;
  // apparent charge, then the particles' own charge
  k_apparent_charge<<<grid, block, 0, s>>>(*m, *f, w->Az, w->Ari, w->Aro, 0, w->part);
  spiffe_note_launches(1);
  k_finish_sum<<<1, 1024, 0, s>>>(w->part, nblk, 2, w->scalars + 0);
  spiffe_note_launches(1);
  k_finish_sum<<<1, 1024, 0, s>>>(w->part + 1, nblk, 2, w->scalars + 1);
  spiffe_note_launches(1);
  if (o->space_charge && np_bound > 0) {
    const unsigned pb = blocks_for(np_bound, RT);
    if (int rc = remove_charge())
      return rc;
    k_finish_sum<<<1, 1024, 0, s>>>(w->part, (int)pb, 1, w->scalars + 2);
    spiffe_note_launches(1);
  } else {
    cudaMemsetAsync(w->scalars + 2, 0, sizeof(double), s);
  }
  sum_region(f->Q, m->nz, m->nr, m->pitch, 0, w, w->scalars + 3, s);
  const bool bound = o->error_charge_threshold > 0;
  if (bound)
    sum_region(f->Q, m->nz, m->nr, m->pitch, 1, w, w->scalars + 5, s);
  k_set_state<<<1, 1, 0, s>>>(w->st, w->scalars, w->scalars + 2, w->scalars + 3, o->space_charge);
  spiffe_note_launches(1);
  k_pc_decide<<<1, 1, 0, s>>>(w->st, o->error_charge_threshold, f->Q, m->nz, m->nr, m->pitch,
                              bound ? w->scalars + 5 : nullptr);
  spiffe_note_launches(1);
  k_scale_rhs<<<grid, block, 0, s>>>(*m, *f, w->volume, w->st);
  spiffe_note_launches(1);
  if (o->guess_code)
    { k_guess<<<grid, block, 0, s>>>(*m, *f, o->guess_code, w->st); spiffe_note_launches(1); }
  int rc = launch_sor(m, w, f->Psi, f->Q, f->flags, o->accuracy, o->maximum_iterations, w->st, w->iters, cnt, s);
  if (rc)
    return rc;
  k_subtract_gradient<<<grid, block, 0, s>>>(*m, *f, w->st);
  spiffe_note_launches(1);
  // the reference recomputes the apparent charge afterwards (:333-439)
  k_apparent_charge<<<grid, block, 0, s>>>(*m, *f, w->Az, w->Ari, w->Aro, 1, w->part);
  spiffe_note_launches(1);
  if (o->space_charge && np_bound > 0)
    if (int rc = remove_charge())
      return rc;
  return (int)cudaGetLastError();
}

// Downloads the last correction's report (synchronises the stream).
extern "C" int spiffe_poisson64_report(Poisson64Work *w, spiffe_poisson_report *rep, cudaStream_t s)
{
  PcState st;
  cudaMemcpyAsync(&st, w->st, sizeof(st), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  rep->ran = st.do_solve;
  rep->iterations = st.iterations;
  rep->Qreal = st.Qreal;
  rep->Qerror = st.Qerror;
  rep->Qsurface = st.Qsurface;
  rep->residual = st.residual;
  double drv = 0;
  cudaMemcpy(&drv, w->scalars + 4, sizeof(double), cudaMemcpyDeviceToHost);
  rep->driving = drv;
  return (int)e;
}

extern "C" int spiffe_imposed_field64(const DevMesh *m, const DevFields<double> *f, double factor, cudaStream_t s)
{
  dim3 block(BX, BY), grid((m->nr + 1 + BX - 1) / BX, (m->nz + 1 + BY - 1) / BY);
  k_imposed_field<<<grid, block, 0, s>>>(*m, *f, factor);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

// ----------------------------------------------- allocation-free SOR solve
//
// spiffe_gpu_solve_poisson_cyl_noalloc runs the same red-black SOR as
// spiffe_gpu_solve_poisson_cyl on device arrays the caller owns, for callers
// that must not allocate device memory: a host application whose device
// memory is owned by another framework's pool, which has reserved it and
// whose budget a cudaMalloc would break; or a control or real-time loop that
// forbids allocation after start-up so a solve can never fail for lack of
// memory or stall in the allocator.  Every piece of scratch the solve needs
// (the Chebyshev factors, the row coefficients, the block partial sums, the
// grid-barrier words and a counter block) lives in the fixed array below,
// which every GPU that loads this library holds until the process exits.

#define SPIFFE_NOALLOC_MAX_HALFSWEEPS 16384 // iteration_limit
#define SPIFFE_NOALLOC_MAX_NR 4096          // nr
#define SPIFFE_NOALLOC_MAX_PARTS 16384      // blocks of the |rhs| sum: ceil((nr-1)/32) * ceil(nz/8)
#define SPIFFE_NOALLOC_MAX_GRID 1024        // SOR blocks

struct NoallocScratch {
  double omega[SPIFFE_NOALLOC_MAX_HALFSWEEPS];
  double crow[SPIFFE_NOALLOC_MAX_NR + 1], drow[SPIFFE_NOALLOC_MAX_NR + 1];
  double part[SPIFFE_NOALLOC_MAX_PARTS];
  double sor_part[2 * SPIFFE_NOALLOC_MAX_GRID];
  double driving;
  long long iterations;
  unsigned bar[2];
  DevCounts cnt;
};

#define SPIFFE_NOALLOC_SCRATCH_BYTES (352u * 1024u)
static_assert(sizeof(NoallocScratch) <= SPIFFE_NOALLOC_SCRATCH_BYTES, "no-alloc scratch too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[SPIFFE_NOALLOC_SCRATCH_BYTES];

#include <cstdio>
#include <mutex>

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
int g_noalloc_grid[NOALLOC_MAX_DEVICES];
// host staging for the tables, static so the call allocates nothing
double g_noalloc_omega[SPIFFE_NOALLOC_MAX_HALFSWEEPS];
double g_noalloc_crow[SPIFFE_NOALLOC_MAX_NR + 1], g_noalloc_drow[SPIFFE_NOALLOC_MAX_NR + 1];
} // namespace

extern "C" int spiffe_set_error(int code, const char *msg);

extern "C" int spiffe_gpu_solve_poisson_cyl_noalloc(const spiffe_mesh *mesh, double *psi, const double *rhs,
                                                    const int16_t *flags, double accuracy, int64_t iteration_limit,
                                                    int64_t *iterations, void *stream)
{
  char msg[256];
  if (!mesh || !psi || !flags)
    return spiffe_set_error(-1, "null argument");
  if (accuracy <= 0)
    return spiffe_set_error(-1, "accuracy is <= 0 in solve_poisson_cyl");
  if (iteration_limit <= 1)
    return spiffe_set_error(-1, "iteration_limit is <= 1 in solve_poisson_cyl");
  const int nz = mesh->nz, nr = mesh->nr;
  if (nz < 3 || nr < 4)
    return spiffe_set_error(-1, "mesh too small (need nz>=3, nr>=4)");
  if (iteration_limit > SPIFFE_NOALLOC_MAX_HALFSWEEPS) {
    snprintf(msg, sizeof(msg), "iteration_limit %lld exceeds the allocation-free maximum of %d",
             (long long)iteration_limit, SPIFFE_NOALLOC_MAX_HALFSWEEPS);
    return spiffe_set_error(-1, msg);
  }
  if (nr > SPIFFE_NOALLOC_MAX_NR) {
    snprintf(msg, sizeof(msg), "nr=%d exceeds the allocation-free maximum of %d", nr, SPIFFE_NOALLOC_MAX_NR);
    return spiffe_set_error(-1, msg);
  }
  const dim3 sblock(BX, BY), sgrid((nr - 1 + BX - 1) / BX, (nz + BY - 1) / BY);
  if ((size_t)sgrid.x * sgrid.y > SPIFFE_NOALLOC_MAX_PARTS) {
    snprintf(msg, sizeof(msg), "mesh of %d x %d nodes exceeds the allocation-free maximum of %d sum blocks", nz, nr,
             SPIFFE_NOALLOC_MAX_PARTS);
    return spiffe_set_error(-1, msg);
  }
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return spiffe_set_error(-2, "no current CUDA device");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  // every call, with the caller's device and context current: the device
  // address of the scratch array (its host-side name is not a device
  // address).  The lookup allocates nothing, and repeating it keeps the
  // address right after a device reset or under another context.
  NoallocScratch *sc = nullptr;
  {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the solver scratch failed: %s", cudaGetErrorString(e));
      return spiffe_set_error(-2, msg);
    }
    sc = (NoallocScratch *)p;
  }
  // the cooperative grid depends on the device only
  if (!g_noalloc_grid[dev]) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sor, RT, 0);
    if (per > 4)
      per = 4;
    int grid = sms * (per > 0 ? per : 1);
    if (grid > SPIFFE_NOALLOC_MAX_GRID)
      grid = SPIFFE_NOALLOC_MAX_GRID;
    g_noalloc_grid[dev] = grid;
  }
  // the tables, with the expressions of the instance path (poisson.c:342-361)
  const double dz = mesh->dz, dr = mesh->dr;
  const double rz = dz / dr;
  const double rj = (cos(SPIFFE_PI / nz) + rz * rz * cos(SPIFFE_PI / nr)) / (1 + rz * rz);
  double omega = 1.0;
  for (long long n = 0; n < iteration_limit; n++) {
    g_noalloc_omega[n] = omega;
    omega = n == 0 ? 1.0 / (1 - rj * rj / 2) : 1.0 / (1 - rj * rj * omega / 4);
  }
  for (int ir = 0; ir <= nr; ir++) {
    if (ir != 0) {
      g_noalloc_crow[ir] = 1 / (dr * dr) * (1 + 1. / (2 * ir));
      g_noalloc_drow[ir] = 1 / (dr * dr) * (1 - 1. / (2 * ir));
    } else
      g_noalloc_crow[ir] = g_noalloc_drow[ir] = 1 / (dr * dr);
  }
  cudaError_t e = cudaMemcpyAsync(sc->omega, g_noalloc_omega, sizeof(double) * iteration_limit,
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sc->crow, g_noalloc_crow, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sc->drow, g_noalloc_drow, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  // the array keeps the previous call's contents: clear what must start at zero
  if (e == cudaSuccess)
    e = cudaMemsetAsync(sc->bar, 0, sizeof(sc->bar), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(&sc->cnt, 0, sizeof(DevCounts), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(&sc->iterations, 0, sizeof(long long), s);
  if (e != cudaSuccess) {
    snprintf(msg, sizeof(msg), "staging the solver tables failed: %s", cudaGetErrorString(e));
    return spiffe_set_error(-2, msg);
  }
  DevMesh m{};
  m.nz = nz;
  m.nr = nr;
  m.pitch = nr + 1;
  m.zmin = mesh->zmin;
  m.zmax = mesh->zmax;
  m.rmax = mesh->rmax;
  m.dz = dz;
  m.dr = dr;
  m.dt = mesh->dt;
  m.lower_bc = mesh->lower_bc;
  m.upper_bc = mesh->upper_bc;
  m.right_bc = mesh->right_bc;
  m.left_bc = mesh->left_bc;
  m.modes = mesh->modes;
  // sum |rhs| over iz < nz, ir < nr-1 (poisson.c:333-336), as the instance path forms it
  if (rhs) {
    k_region_sum<<<sgrid, sblock, 0, s>>>(rhs, nz, nr - 1, nr + 1, 1, sc->part);
    spiffe_note_launches(1);
    k_finish_sum<<<1, 1024, 0, s>>>(sc->part, sgrid.x * sgrid.y, 1, &sc->driving);
    spiffe_note_launches(1);
  } else {
    cudaMemsetAsync(&sc->driving, 0, sizeof(double), s);
  }
  SorArgs a;
  a.Psi = psi;
  a.rhs = rhs;
  a.flags = flags;
  a.omega = sc->omega;
  a.a = 1 / (dz * dz);
  a.e = -2 * (1 / (dz * dz) + 1 / (dr * dr));
  a.crow = sc->crow;
  a.drow = sc->drow;
  const double c_axis = 1 / (dr * dr);
  a.c4_axis = 4 * c_axis;
  a.e2c_axis = a.e - 2 * c_axis;
  a.accuracy = accuracy;
  a.driving = &sc->driving;
  a.limit = iteration_limit;
  a.partials = sc->sor_part;
  a.bar_count = sc->bar;
  a.bar_gen = sc->bar + 1;
  a.st = nullptr;
  a.iterations_out = &sc->iterations;
  DevCounts *cnt = &sc->cnt;
  void *args[] = {&m, &a, &cnt};
  e = cudaLaunchCooperativeKernel((void *)k_sor, dim3(g_noalloc_grid[dev]), dim3(RT), args, 0, s);
  spiffe_note_launches(1);
  long long it = 0;
  unsigned err = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&it, &sc->iterations, sizeof(it), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&err, &sc->cnt.error, sizeof(err), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    snprintf(msg, sizeof(msg), "allocation-free SOR failed: %s", cudaGetErrorString(e));
    return spiffe_set_error(-2, msg);
  }
  if (err & SPIFFE_DEV_ERR_BARRIER)
    return spiffe_set_error(-4, "allocation-free SOR: grid barrier timed out");
  if (iterations)
    *iterations = it;
  return 0;
}
