// spiffe_b200/csrc/poisson_f32.cu -- Poisson correction of the split-precision form.
//
// add_poisson_correction (poisson_correction.c:73-454), solve_poisson_cyl
// (poisson.c:17-130) and compute_imposed_Efield (poisson_correction.c:456-562)
// for FP32 fields, with the charge, potential and residual kept in FP64.
//
// The solve runs the reference's red-black SOR with its Chebyshev factors
// and stop rule, but on the correction d = Psi - Psi0 of the warm start Psi0:
// the reference iterates Psi <- Psi - w (A Psi - rhs)/e node by node, which
// is affine in Psi, so with r0 = rhs - A Psi0 formed once in FP64 the same
// sweeps on d (residual A d - r0) produce the same iterates Psi0 + d.  The
// sweeps run in FP32 on d, which is small, and the result is added to Psi
// in FP64.  Each CTA of a cooperative launch holds a band of mesh rows of d,
// r0 and the node mask in shared memory for the whole solve (the FP32 mesh
// of a 3000 x 820 gun is 20 MB, which the 148 SMs' shared memory holds), so
// a half-sweep reads no global memory except the two neighbour rows that the
// adjacent CTAs updated; the rows of each colour are stored as separate
// contiguous halves so a warp's accesses are conflict-free.  The per-CTA
// |residual| sums are added in 64-bit fixed point inside the grid barrier's
// arrival atomic, so every CTA takes the same stop decision from an
// order-independent total.  When the residual has fallen 2^8-fold the
// correction is folded into Psi and the residual formed again in FP64
// (iterative refinement), so FP32 rounding of d never limits convergence.
#include "split32.cuh"
#include "modules.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

constexpr int BX = 32, BY = 8, RT = 256;

__device__ double block_sum_d(double v, double *sh)
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

// Apparent charge from the flux of E (poisson_correction.c:141-182, second
// pass :335-375), in FP64 from the FP32 fields.
__global__ void __launch_bounds__(BX *BY) k_apparent32(DevMesh m, DevFields32 f, const double *Az_, const double *Ari,
                                                        const double *Aro, int second, double *part)
{
  __shared__ double sh[BX * BY];
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  const double eps = SPIFFE_EPSILON_O;
  double qs = 0, cen = 0;
  if (ir < nr && iz < nz) {
    const size_t i = node(iz, ir, P);
    const double Az = Az_[ir], Ar_inner = Ari[ir], Ar_outer = Aro[ir];
    const double Ez0 = f.Ez[i], Ez1 = f.Ez[i + P], Er0 = f.Er[i], Er1 = f.Er[i + 1];
    double dQ;
    if (ir == 0)
      dQ = (Er1 * Ar_outer + (Ez1 - Ez0) * Az) * eps;
    else
      dQ = (Er1 * Ar_outer - Er0 * Ar_inner + (Ez1 - Ez0) * Az) * eps;
    if (surface_cell(m, f.flags[i], iz, ir)) {
      if (iz == 0)
        dQ += Ez0 * Az * eps;
      if (iz == nz - 1)
        dQ -= Ez1 * Az * eps;
      if (ir == nr - 1) {
        const double e = (double)f.Ez[i + 1] * Ar_outer * eps;
        dQ += second ? -e : e;
      }
      qs = dQ;
      f.Q[i] = 0;
    } else {
      f.Q[i] = dQ;
      cen = dQ * (iz * m.dz + m.zmin);
    }
  }
  const double s0 = block_sum_d(qs, sh), s1 = block_sum_d(cen, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int b = blockIdx.y * gridDim.x + blockIdx.x;
    part[2 * b] = s0;
    part[2 * b + 1] = s1;
  }
}

// The particles' own charge (:190-242) in fixed point: Qp[node] receives the
// removed charge of each non-metal node, Qreal the total.
__global__ void __launch_bounds__(RT) k_remove32(DevMesh m, DevFields32 f, DevBeam32 b, const DevCounts *cnt,
                                                  S32Scales sc, long long *qreal_fixed)
{
  __shared__ double sh[RT];
  const long ip = (long)blockIdx.x * RT + threadIdx.x;
  int nodes[4] = {-1, -1, -1, -1};
  long long q[4] = {0, 0, 0, 0};
  long long mine = 0;
  if (ip < (long)cnt->np && (b.status[ip] & S32_ACTIVE)) {
    const int nz = m.nz, nr = m.nr, P = m.pitch;
    const bool lsm = m.modes & SPIFFE_FL_LONGIT_SMEAR, rsm = m.modes & SPIFFE_FL_RADIAL_SMEAR;
    const bool ln = m.left_bc == SPIFFE_NEUMANN, rn = m.right_bc == SPIFFE_NEUMANN, un = m.upper_bc == SPIFFE_NEUMANN;
    const int32_t c = b.cell[ip];
    const int cz = s32_iz(c), cr = s32_ir(c);
    const float fz = b.fz[ip], fr = b.fr[ip];
    // (long) truncation toward zero of (z-zmin)/dz [+0.5] and r/dr [+0.5]
    int iz, ir;
    float zf, rf;
    {
      const float tz = lsm ? fz : fz + 0.5f, tr = rsm ? fr : fr + 0.5f;
      iz = cz + (tz >= 1.f);
      zf = tz - (float)(tz >= 1.f);
      ir = cr + (tr >= 1.f);
      rf = tr - (float)(tr >= 1.f);
      if (iz < 0 && zf > 0.f) {
        iz++;
        zf -= 1.f;
      }
      if (ir < 0 && rf > 0.f) {
        ir++;
        rf -= 1.f;
      }
    }
    if (iz >= 0 && iz < nz && ir >= 0 && ir < nr) {
      float fa, fb, frr, fl;
      if (rsm && ir != nr - 1) {
        fa = rf;
        fb = 1 - fa;
      } else {
        fb = 1;
        fa = 0;
      }
      if (lsm && iz != nz - 1) {
        frr = zf;
        fl = 1 - frr;
      } else {
        fl = 1;
        frr = 0;
      }
      const float Qs = b.Q[ip] * sc.sq_charge;
      const int16_t *F = f.flags;
      if (!((F[node(iz, ir, P)] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz - 1 && rn) || (ir >= nr - 1 && un))) {
        nodes[0] = (int)node(iz, ir, P);
        q[0] = __float2ll_rn(Qs * fb * fl);
      }
      if (!((F[node(iz + 1, ir, P)] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz && rn) || (ir >= nr - 1 && un))) {
        nodes[1] = (int)node(iz + 1, ir, P);
        q[1] = __float2ll_rn(Qs * fb * frr);
      }
      if (!((F[node(iz, ir + 1, P)] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz - 1 && rn) || (ir >= nr && un))) {
        nodes[2] = (int)node(iz, ir + 1, P);
        q[2] = __float2ll_rn(Qs * fa * fl);
      }
      if (!((F[node(iz + 1, ir + 1, P)] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz && rn) || (ir >= nr && un))) {
        nodes[3] = (int)node(iz + 1, ir + 1, P);
        q[3] = __float2ll_rn(Qs * fa * frr);
      }
      for (int k = 0; k < 4; k++)
        if (nodes[k] >= 0)
          mine += q[k];
    }
  }
  for (int k = 0; k < 4; k++) {
    // same grouping as the current deposition
    const unsigned grp = __match_any_sync(0xffffffffu, nodes[k]);
    const unsigned long long biased = (unsigned long long)(q[k] + (1LL << 42));
    const unsigned lo = (unsigned)(biased & ((1u << 22) - 1)), hi = (unsigned)(biased >> 22);
    const unsigned slo = __reduce_add_sync(grp, lo), shi = __reduce_add_sync(grp, hi);
    if (nodes[k] >= 0 && (threadIdx.x & 31) == __ffs(grp) - 1) {
      const long long tot = ((long long)shi << 22) + (long long)slo - (long long)__popc(grp) * (1LL << 42);
      if (tot)
        atomic_add_ll(f.Qp + nodes[k], tot);
    }
  }
  // exact integer total of the removed charge
  const double s = block_sum_d((double)mine, sh); // |per-block sum| < 2^53
  if (threadIdx.x == 0 && s != 0)
    atomic_add_ll(qreal_fixed, (long long)s);
}

// Q -= particle charge (the FP64 form's atomics on Q) over all nodes; partial
// sums of Q over iz < nz, ir < nr for Qerror (:244-256).
__global__ void __launch_bounds__(BX *BY) k_combine32(DevMesh m, DevFields32 f, double qQ, int space_charge,
                                                       double *part)
{
  __shared__ double sh[BX * BY];
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  double v = 0;
  if (ir <= m.nr && iz <= m.nz) {
    const size_t i = node(iz, ir, m.pitch);
    double q = f.Q[i];
    if (space_charge) {
      const long long p = f.Qp[i];
      if (p)
        q -= (double)p * qQ;
      f.Q[i] = q;
    }
    if (ir < m.nr && iz < m.nz)
      v = q;
  }
  const double s = block_sum_d(v, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    part[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

__global__ void k_finish_sum32(const double *part, int n, int stride, double *out)
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

__global__ void k_state32(PcState *st, const double *sc, const long long *qreal_fixed, double qQ, int space_charge,
                          double threshold)
{
  st->Qsurface = sc[0];
  st->centroid = sc[1];
  st->Qreal = space_charge ? (double)*qreal_fixed * qQ : 0.0;
  st->Qerror = sc[3];
  const double Qerror = st->Qerror, Qreal = st->Qreal;
  // error-charge threshold test (:258-265)
  const int skip = (threshold > 0 && fabs(Qerror) < threshold) ||
                   (threshold < 0 && (Qreal == 0 || fabs(Qerror / Qreal) < fabs(threshold)));
  st->do_solve = !skip;
}

// Q -> -Q/(V eps0) over iz < nz, ir < nr (:268-274)
__global__ void __launch_bounds__(BX *BY) k_scale32(DevMesh m, DevFields32 f, const double *volume, const PcState *st)
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
__global__ void __launch_bounds__(BX *BY) k_guess32(DevMesh m, DevFields32 f, int code, const PcState *st)
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
    f.Psi[i] = charge / (4 * SPIFFE_PI * SPIFFE_EPSILON_O * sqrt(zz * zz + rr * rr));
  } else if (code == 3)
    f.Psi[i] = 0;
}

// ---- the shared-memory SOR

struct Sor32Args {
  double *Psi;
  const double *rhs; // null: Laplace solve
  const uint8_t *umask;
  const float *omega;
  const float *crow, *drow; // per ir
  float a, e, inv_e, c4, e2c, inv_e2c;
  double a_d, e_d, c4_d, e2c_d, dr2_inv;
  double accuracy;
  long long limit;
  float *xbuf;                  // exchange rows [2][grid][2 sides][2 rows][2 parities][H]
  unsigned long long *arrive;   // barrier arrivals (low byte) and the first fixed-point sum
  unsigned long long *release;  // barrier generation (high 16 bits) and the first sum (low 48)
  unsigned long long *acc1;     // the second fixed-point sum
  unsigned long long *pub1;     // the second sum, published by the last CTA to arrive
  double *dpart;                // [grid][2] |rhs| and |r0| partials
  PcState *st;
  long long *iters_out;
  int lo, hi, cols, H, rows_per; // H: half-row length, a multiple of 4
};

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p)
{
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Bounded grid barrier that also sums two fixed-point values per CTA.  Each
// CTA adds the second value to *acc1 and then (v0 << 8) | 1 to *arrive, so
// the low byte of *arrive counts arrivals (at most 255 CTAs) and the rest
// accumulates the first sum; the last CTA to arrive reads and clears both
// accumulators, publishes the second sum in *pub1 and releases the others
// by storing the next generation (high 16 bits) with the first sum (low 48
// bits) in *release.  The fence before the arrival releases the CTA's
// earlier writes (the caller synchronises the CTA first, so they precede
// it); the acquire of *release (or the fence after the last arrival) makes
// every CTA's writes visible.  `gen` counts the barriers the calling thread
// has passed.  Returns false (and raises the device error bit) when the
// others do not arrive within the poll limit.
__device__ bool grid_sync_sum(const Sor32Args &s, unsigned long long v0, unsigned long long v1, unsigned &gen,
                              unsigned long long *t0, unsigned long long *t1, DevCounts *cnt, int *ok_sh)
{
  if (threadIdx.x == 0) {
    int ok = 1;
    gen = (gen + 1) & 0xffffu;
    unsigned long long old, tot0 = 0, tot1 = 0;
    const unsigned long long add = (v0 << 8) | 1ull;
    if (v1)
      asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(s.acc1), "l"(v1) : "memory");
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    asm volatile("atom.relaxed.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(s.arrive), "l"(add) : "memory");
    if ((old & 0xffull) == gridDim.x - 1) {
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      tot0 = (old >> 8) + v0;
      asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(tot1) : "l"(s.acc1) : "memory");
      const unsigned long long rel = ((unsigned long long)gen << 48) | (tot0 & 0xffffffffffffull);
      asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(s.acc1), "l"(0ull) : "memory");
      asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(s.pub1), "l"(tot1) : "memory");
      asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(s.arrive), "l"(0ull) : "memory");
      asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(s.release), "l"(rel) : "memory");
    } else {
      unsigned long long polls = 0, v;
      while (((v = ld_acquire64(s.release)) >> 48) != gen) {
        if (++polls > (1ull << 24)) {
          ok = 0;
          atomicOr(&cnt->error, SPIFFE_DEV_ERR_BARRIER);
          break;
        }
        if (polls > 256)
          __nanosleep(20);
      }
      tot0 = v & 0xffffffffffffull;
      asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(tot1) : "l"(s.pub1) : "memory");
    }
    if (t0)
      *t0 = tot0;
    if (t1)
      *t1 = tot1;
    *ok_sh = ok;
  }
  __syncthreads();
  return *ok_sh != 0;
}

// Band of rows of CTA b: [start, start+n) of the update rows lo..hi.
__device__ __forceinline__ void band(int rows, int b, int G, int &start, int &n)
{
  const int base = rows / G, rem = rows % G;
  n = base + (b < rem ? 1 : 0);
  start = b * base + (b < rem ? b : rem);
}

// r0 = rhs - A Psi (FP64, Psi read through L2) into B for the mesh rows
// iz0 .. iz0+nb-1 (B row i = mesh row iz0+i) that the SOR updates; adds this
// thread's share of sum |rhs| and sum |r0| over the band's own rows
// [own_lo, own_hi] to *drive and *rsum.
__device__ void form_r0(const DevMesh &m, const Sor32Args &s, float *B, int iz0, int nb, int own_lo, int own_hi,
                        double *drive, double *rsum)
{
  const int nz = m.nz, P = m.pitch, H = s.H, cols = s.cols;
  double d = 0, q = 0;
  for (int i = 0; i < nb; i++) {
    const int iz = iz0 + i;
    const bool upd = iz >= s.lo && iz <= s.hi, own = iz >= own_lo && iz <= own_hi;
    const long up = (iz == 0 && s.lo == 0) ? P : (iz == nz - 1 && s.hi == nz - 1 ? -P : P);
    const long dn = (iz == 0 && s.lo == 0) ? P : -P;
    for (int t = threadIdx.x; t < 2 * H; t += blockDim.x) {
      const int p = t / H, k = t - p * H, ir = 2 * k + p;
      float r0 = 0.f;
      if (upd && ir < cols) {
        const size_t j = node(iz, ir, P);
        const double rh = s.rhs ? s.rhs[j] : 0.0;
        if (own)
          d += fabs(rh);
        if (!(s.umask[j] & S32_U_METAL)) {
          const double psi = __ldcg(s.Psi + j), lr = __ldcg(s.Psi + j + up) + __ldcg(s.Psi + j + dn);
          double ap;
          if (ir == 0)
            ap = s.a_d * lr + s.c4_d * __ldcg(s.Psi + j + 1) + s.e2c_d * psi;
          else
            ap = s.a_d * lr + s.dr2_inv * (1 + 1. / (2 * ir)) * __ldcg(s.Psi + j + 1) +
                 s.dr2_inv * (1 - 1. / (2 * ir)) * __ldcg(s.Psi + j - 1) + s.e_d * psi;
          r0 = (float)(rh - ap);
          if (own)
            q += fabs(rh - ap);
        }
      }
      B[(i * 2 + p) * H + k] = r0;
    }
  }
  *drive += d;
  *rsum += q;
}

// The SOR update of four consecutive nodes of one colour in one row (nodes
// ir = 2(k0+i) + p): D row jd with neighbour rows uj, dj, B/M row jb.
// Returns the sum of their |residual|.  With UNDO it instead restores the
// values before that update: new = old(1-w) - w(nb - r0)/e, so
// old = (new + w(nb - r0)/e)/(1-w) (w > 1 after the first half-sweep).
template <bool UNDO>
__device__ __forceinline__ float sweep4(const Sor32Args &s, float *D, const float *B, const uint8_t *M,
                                        const float *CR, const float *DR, int jd, int uj, int dj, int jb, int p,
                                        int k0, float w)
{
  const int H = s.H;
  const int rs = (jd * 2 + p) * H + k0, ro = (jd * 2 + (p ^ 1)) * H + k0, rb = (jb * 2 + p) * H + k0;
  float4 sv = *reinterpret_cast<const float4 *>(D + rs);
  const float4 uv = *reinterpret_cast<const float4 *>(D + (uj * 2 + p) * H + k0);
  const float4 dv = *reinterpret_cast<const float4 *>(D + (dj * 2 + p) * H + k0);
  const float4 ov = *reinterpret_cast<const float4 *>(D + ro);
  const float4 bv = *reinterpret_cast<const float4 *>(B + rb);
  const uchar4 mv = *reinterpret_cast<const uchar4 *>(M + rb);
  const float4 cr = *reinterpret_cast<const float4 *>(CR + p * H + k0);
  const float4 dr = *reinterpret_cast<const float4 *>(DR + p * H + k0);
  // neighbours in r: the other colour's nodes ir-1 and ir+1
  float l0, l1, l2, l3, r0, r1, r2, r3;
  if (p == 0) {
    l0 = k0 > 0 ? D[ro - 1] : 0.f;
    l1 = ov.x;
    l2 = ov.y;
    l3 = ov.z;
    r0 = ov.x;
    r1 = ov.y;
    r2 = ov.z;
    r3 = ov.w;
  } else {
    l0 = ov.x;
    l1 = ov.y;
    l2 = ov.z;
    l3 = ov.w;
    r0 = ov.y;
    r1 = ov.z;
    r2 = ov.w;
    r3 = D[ro + 4];
  }
  const float a = s.a, e = s.e, we = w * s.inv_e;
  float acc = 0.f;
  if (UNDO) {
    const float inv1w = 1.f / (1.f - w);
    if (mv.x) {
      if (p == 0 && k0 == 0)
        sv.x = (sv.x + w * s.inv_e2c * (a * (uv.x + dv.x) + s.c4 * r0 - bv.x)) * inv1w;
      else
        sv.x = (sv.x + we * (a * (uv.x + dv.x) + cr.x * r0 + dr.x * l0 - bv.x)) * inv1w;
    }
    if (mv.y)
      sv.y = (sv.y + we * (a * (uv.y + dv.y) + cr.y * r1 + dr.y * l1 - bv.y)) * inv1w;
    if (mv.z)
      sv.z = (sv.z + we * (a * (uv.z + dv.z) + cr.z * r2 + dr.z * l2 - bv.z)) * inv1w;
    if (mv.w)
      sv.w = (sv.w + we * (a * (uv.w + dv.w) + cr.w * r3 + dr.w * l3 - bv.w)) * inv1w;
  } else {
    if (mv.x) {
      float res;
      if (p == 0 && k0 == 0) { // the axis node (poisson.c:386-387)
        res = a * (uv.x + dv.x) + s.c4 * r0 + s.e2c * sv.x - bv.x;
        sv.x -= w * s.inv_e2c * res;
      } else {
        res = a * (uv.x + dv.x) + cr.x * r0 + dr.x * l0 + e * sv.x - bv.x;
        sv.x -= we * res;
      }
      acc += fabsf(res);
    }
    if (mv.y) {
      const float res = a * (uv.y + dv.y) + cr.y * r1 + dr.y * l1 + e * sv.y - bv.y;
      sv.y -= we * res;
      acc += fabsf(res);
    }
    if (mv.z) {
      const float res = a * (uv.z + dv.z) + cr.z * r2 + dr.z * l2 + e * sv.z - bv.z;
      sv.z -= we * res;
      acc += fabsf(res);
    }
    if (mv.w) {
      const float res = a * (uv.w + dv.w) + cr.w * r3 + dr.w * l3 + e * sv.w - bv.w;
      sv.w -= we * res;
      acc += fabsf(res);
    }
  }
  *reinterpret_cast<float4 *>(D + rs) = sv;
  return acc;
}

// One colour over D rows jlo..jhi (mesh row iz = iz_first + jd - 2; B/M row
// jd - 1); |residual| summed over the own rows 2..nrow+1 only.
// With xo, a slot of an exchanged row (the first two and the last two own
// rows) also stores both colours of its four columns there, for the
// neighbouring CTAs (the other colour was final after the previous sweep).
template <bool UNDO>
__device__ float sweep_rows(const DevMesh &m, const Sor32Args &s, float *D, const float *B, const uint8_t *M,
                            const float *CR, const float *DR, int iz_first, int nrow, int jlo, int jhi, int c, float w,
                            float *xo = nullptr)
{
  const int nz = m.nz, Q = s.H >> 2, NT = blockDim.x, tid = threadIdx.x;
  const int slots = (jhi - jlo + 1) * Q, jstep = NT / Q, qstep = NT - jstep * Q;
  int jd = jlo + tid / Q, q = tid - (tid / Q) * Q;
  float acc = 0.f;
  for (int t = tid; t < slots; t += NT) {
    const int iz = iz_first + jd - 2;
    const int p = (c + iz) & 1;
    // Dirichlet end rows mirror their only neighbour (poisson.c:369-375, :404-410)
    const int uj = (iz == nz - 1 && s.hi == nz - 1) ? jd - 1 : jd + 1;
    const int dj = (iz == 0 && s.lo == 0) ? jd + 1 : jd - 1;
    const float r = sweep4<UNDO>(s, D, B, M, CR, DR, jd, uj, dj, jd - 1, p, q << 2, w);
    if (jd >= 2 && jd <= nrow + 1)
      acc += r;
    if (xo) {
      const int H = s.H;
      // side 0: rows 2, 3 for the CTA above; side 1: rows nrow, nrow+1 for the one below
      const bool s0 = jd <= 3, s1 = jd >= nrow;
      if (s0 || s1) {
        const float4 v0 = *reinterpret_cast<const float4 *>(D + (jd * 2) * H + 4 * q);
        const float4 v1 = *reinterpret_cast<const float4 *>(D + (jd * 2 + 1) * H + 4 * q);
        if (s0) {
          float *x = xo + (jd - 2) * 2 * H + 4 * q;
          __stcg(reinterpret_cast<float4 *>(x), v0);
          __stcg(reinterpret_cast<float4 *>(x + H), v1);
        }
        if (s1) {
          float *x = xo + 4 * H + (jd - nrow) * 2 * H + 4 * q;
          __stcg(reinterpret_cast<float4 *>(x), v0);
          __stcg(reinterpret_cast<float4 *>(x + H), v1);
        }
      }
    }
    q += qstep;
    jd += jstep;
    if (q >= Q) {
      q -= Q;
      jd++;
    }
  }
  return acc;
}

// Psi += d on the band's own updated nodes (FP64)
__device__ void fold_d(const Sor32Args &s, int P, const float *D, const uint8_t *M, int iz_first, int nrow)
{
  const int H = s.H, cols = s.cols;
  for (int j = 2; j <= nrow + 1; j++) {
    const int iz = iz_first + j - 2;
    for (int t = threadIdx.x; t < 2 * H; t += blockDim.x) {
      const int p = t / H, k = t - p * H, ir = 2 * k + p;
      const float d = D[(j * 2 + p) * H + k];
      if (ir < cols && M[((j - 1) * 2 + p) * H + k] && d != 0.f) {
        const size_t i = node(iz, ir, P);
        __stcg(s.Psi + i, __ldcg(s.Psi + i) + (double)d);
      }
    }
  }
}

__device__ __forceinline__ double block_sum2(double v, double *red, int slot)
{
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0)
    red[slot * 32 + (threadIdx.x >> 5)] = v;
  return v;
}

// solve_poisson_cyl (poisson.c:17-130) on the correction d of the warm
// start.  Each round runs one half-sweep of each colour between two grid
// barriers: a CTA's band carries two halo rows on each side, the colour-0
// sweep also updates the nearer halo row (from exactly the inputs the
// neighbour uses, so with the same result), and the colour-1 sweep then
// needs nothing from the neighbours.  Both half-sweeps' |residual| sums
// arrive with the barrier, so the reference's stop test runs after every
// half-sweep; when it fires after colour 0, the colour-1 update of the
// round is undone.
constexpr int SOR_NT = 1024; // threads per CTA of the shared-memory kernel

__global__ void __launch_bounds__(SOR_NT) k_sor32(DevMesh m, Sor32Args s, DevCounts *cnt)
{
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[64];
  __shared__ int ok_sh, stop_sh, undo_sh, rebase_sh;
  __shared__ double total_sh, thr_sh, quantum_sh, base_sh, p0_sh, p1_sh;
  __shared__ unsigned long long t0_sh, t1_sh;
  __shared__ long long result_sh;
  if (s.st && !s.st->do_solve)
    return;
  const int nz = m.nz, P = m.pitch, H = s.H, Q = s.H >> 2, cols = s.cols, R = s.rows_per;
  const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x, NT = blockDim.x;
  int start, nrow;
  band(s.hi - s.lo + 1, b, G, start, nrow);
  const int iz_first = s.lo + start;
  // shared layout (32-bit offsets): D[(R+4)][2][H] d for mesh rows
  // iz_first-2 .. iz_first+R+1 (D row iz - iz_first + 2), B[(R+2)][2][H] r0
  // and M[(R+2)][2][H] node mask for rows iz_first-1 .. (B row iz -
  // iz_first + 1), CR/DR[2][H] row coefficients; row j's nodes of parity p
  // are the contiguous run (j*2+p)*H .. +H
  float *D = (float *)smem;
  float *B = D + (R + 4) * 2 * H;
  float *CR = B + (R + 2) * 2 * H;
  float *DR = CR + 2 * H;
  uint8_t *M = (uint8_t *)(DR + 2 * H);
  for (int t = tid; t < (R + 4) * 2 * H; t += NT)
    D[t] = 0.f;
  for (int t = tid; t < 2 * H; t += NT) {
    const int p = t / H, k = t - p * H, ir = 2 * k + p;
    CR[t] = ir < cols ? s.crow[ir] : 0.f;
    DR[t] = ir < cols ? s.drow[ir] : 0.f;
  }
  for (int i = 0; i < nrow + 2; i++) {
    const int iz = iz_first - 1 + i;
    const bool upd = iz >= s.lo && iz <= s.hi;
    for (int t = tid; t < 2 * H; t += NT) {
      const int p = t / H, k = t - p * H, ir = 2 * k + p;
      M[(i * 2 + p) * H + k] = upd && ir < cols && !(s.umask[node(iz, ir, P)] & S32_U_METAL) ? 1 : 0;
    }
  }
  const int iz_last = iz_first + nrow - 1;
  double drive = 0, r0sum = 0;
  form_r0(m, s, B, iz_first - 1, nrow + 2, iz_first, iz_last, &drive, &r0sum);
  // rows outside lo..hi that the driving sum still covers (iz < nz)
  if (s.rhs) {
    const bool first = b == 0, last = b == G - 1;
    for (int iz = 0; iz < nz; iz++) {
      if (iz >= s.lo && iz <= s.hi)
        continue;
      if ((iz < s.lo && !first) || (iz > s.hi && !last))
        continue;
      for (int ir = tid; ir < cols; ir += NT)
        drive += fabs(s.rhs[node(iz, ir, P)]);
    }
  }
  // fixed-order block sums of the |rhs| and |r0| partials
  block_sum2(drive, red, 0);
  block_sum2(r0sum, red, 1);
  __syncthreads();
  if (tid == 0) {
    double t = 0, t2 = 0;
    for (int w = 0; w < (NT + 31) / 32; w++) {
      t += red[w];
      t2 += red[32 + w];
    }
    if (G > 1) {
      __stcg(s.dpart + 2 * b, t);
      __stcg(s.dpart + 2 * b + 1, t2);
    } else {
      thr_sh = s.accuracy * t;
      base_sh = t2;
    }
  }
  unsigned gen = 0;
  __syncthreads();
  if (G > 1) {
    if (!grid_sync_sum(s, 0ull, 0ull, gen, nullptr, nullptr, cnt, &ok_sh))
      return;
    if (tid == 0) {
      double d = 0, qq = 0;
      for (int i = 0; i < G; i++) {
        d += __ldcg(s.dpart + 2 * i);
        qq += __ldcg(s.dpart + 2 * i + 1);
      }
      thr_sh = s.accuracy * d;
      base_sh = qq;
    }
  }
  if (tid == 0) {
    quantum_sh = fmax(fmax(base_sh, thr_sh), 1e-280) / 1073741824.0;
    rebase_sh = 0;
    result_sh = -1;
    total_sh = 0;
  }
  __syncthreads();
  // sweeps of the first colour cover the nearer halo rows when there are neighbours
  const int jlo0 = G > 1 ? 1 : 2, jhi0 = G > 1 ? nrow + 2 : nrow + 1;
  for (long long n0 = 0; n0 < s.limit; n0 += 2) {
    if (rebase_sh) {
      // iterative refinement: Psi += d in FP64, r0 = rhs - A Psi in FP64 once
      // every band has folded its d in, and the sweeps go on from d = 0
      fold_d(s, P, D, M, iz_first, nrow);
      __syncthreads();
      if (G > 1 && !grid_sync_sum(s, 0ull, 0ull, gen, nullptr, nullptr, cnt, &ok_sh))
        return;
      double d0 = 0, q0 = 0;
      form_r0(m, s, B, iz_first - 1, nrow + 2, iz_first, iz_last, &d0, &q0);
      for (int t = tid; t < (R + 4) * 2 * H; t += NT)
        D[t] = 0.f;
      __syncthreads();
    }
    const bool two = n0 + 1 < s.limit;
    const float w0 = s.omega[n0], w1 = two ? s.omega[n0 + 1] : 0.f;
    const float acc0 = sweep_rows<false>(m, s, D, B, M, CR, DR, iz_first, nrow, jlo0, jhi0, 0, w0);
    __syncthreads();
    // the colour-1 sweep also writes the exchanged rows for the neighbours
    float *xo = G > 1 ? s.xbuf + (size_t)((n0 >> 1) & 1) * G * 8 * H + (size_t)b * 8 * H : nullptr;
    const float acc1 =
        two ? sweep_rows<false>(m, s, D, B, M, CR, DR, iz_first, nrow, 2, nrow + 1, 1, w1, xo) : 0.f;
    block_sum2((double)acc0, red, 0);
    block_sum2((double)acc1, red, 1);
    __syncthreads();
    if (tid < 32) {
      // fixed-order warp reduction of the per-warp partials
      const int nw = (NT + 31) / 32;
      double t = tid < nw ? red[tid] : 0.0, t2 = tid < nw ? red[32 + tid] : 0.0;
      for (int o = 16; o > 0; o >>= 1) {
        t += __shfl_down_sync(0xffffffffu, t, o);
        t2 += __shfl_down_sync(0xffffffffu, t2, o);
      }
      if (tid == 0) {
        p0_sh = t;
        p1_sh = t2;
      }
    }
    double total0, total1;
    unsigned long long tf0 = 0, tf1 = 0;
    if (G > 1) {
      // this CTA's |residual| sums in quanta of 2^-30 of the larger of the
      // refinement base and the stop threshold, capped at 2^40 quanta
      unsigned long long q0 = 0, q1 = 0;
      if (tid == 0) {
        const double x0 = p0_sh / quantum_sh, x1 = p1_sh / quantum_sh;
        if (p0_sh != 0)
          q0 = x0 >= 1099511627776.0 ? 1099511627776ull : ((unsigned long long)llrint(x0) | 1ull);
        if (p1_sh != 0)
          q1 = x1 >= 1099511627776.0 ? 1099511627776ull : ((unsigned long long)llrint(x1) | 1ull);
      }
      if (!grid_sync_sum(s, q0, q1, gen, &t0_sh, &t1_sh, cnt, &ok_sh))
        return;
      // the neighbours' rows into the halo rows
      const float *xi = s.xbuf + (size_t)((n0 >> 1) & 1) * G * 8 * H;
      for (int t = tid; t < 8 * Q; t += NT) {
        const int side = t / (4 * Q), r = t - side * 4 * Q;
        if (side == 0 && b > 0) {
          const float4 v = __ldcg(reinterpret_cast<const float4 *>(xi + (size_t)(b - 1) * 8 * H + 4 * H) + r);
          *reinterpret_cast<float4 *>(D + (r / (2 * Q)) * 2 * H + 4 * (r % (2 * Q))) = v;
        } else if (side == 1 && b < G - 1) {
          const float4 v = __ldcg(reinterpret_cast<const float4 *>(xi + (size_t)(b + 1) * 8 * H) + r);
          *reinterpret_cast<float4 *>(D + (nrow + 2 + r / (2 * Q)) * 2 * H + 4 * (r % (2 * Q))) = v;
        }
      }
      tf0 = t0_sh;
      tf1 = t1_sh;
      total0 = (double)tf0 * quantum_sh;
      total1 = (double)tf1 * quantum_sh;
    } else {
      __syncthreads();
      total0 = p0_sh;
      total1 = p1_sh;
      tf0 = total0 != 0;
      tf1 = total1 != 0;
    }
    if (tid == 0) {
      const bool stop0 = n0 > 0 && (total0 < thr_sh || tf0 == 0);
      const bool stop1 = two && (total1 < thr_sh || tf1 == 0);
      stop_sh = stop0 || stop1;
      undo_sh = stop0 && two;
      if (stop0) {
        result_sh = n0;
        total_sh = total0;
      } else if (stop1) {
        result_sh = n0 + 1;
        total_sh = total1;
      } else {
        total_sh = two ? total1 : total0;
        // Iterative refinement: once the residual has fallen 2^8-fold below
        // the last FP64 residual (the base), fold d into Psi and form the
        // residual again in FP64 before FP32 rounding of the growing d
        // limits it.  The fixed-point quantum of the residual sums is 2^-30
        // of the larger of the base and the stop threshold, so the stop test
        // keeps its resolution as the base follows the residual down; a
        // per-CTA sum is capped at 2^40 quanta (a barrier word holds 255).
        rebase_sh = total_sh < base_sh * (1.0 / 256);
        if (rebase_sh)
          base_sh = total_sh;
        quantum_sh = fmax(fmax(base_sh, thr_sh), 1e-280) / 1073741824.0;
      }
    }
    __syncthreads();
    if (stop_sh) {
      if (undo_sh) {
        sweep_rows<true>(m, s, D, B, M, CR, DR, iz_first, nrow, 2, nrow + 1, 1, w1);
        __syncthreads();
      }
      break;
    }
  }
  fold_d(s, P, D, M, iz_first, nrow);
  if (b == 0 && tid == 0) {
    const long long result = result_sh;
    if (s.iters_out)
      *s.iters_out = result;
    if (s.st) {
      s.st->iterations = result;
      s.st->residual = total_sh;
    }
    cnt->sor_halfsweeps += result >= 0 ? result + 1 : s.limit;
    cnt->sor_solves += 1;
  }
}

// Ez, Er -= grad Psi (:288-326) with the FDTD boundary copies; FP64 gradient.
__global__ void __launch_bounds__(BX *BY) k_subtract32(DevMesh m, DevFields32 f, const PcState *st)
{
  if (!st->do_solve)
    return;
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (ir > nr || iz > nz)
    return;
  const size_t i = node(iz, ir, P);
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;
  const uint8_t u = f.umask[i];
  const int16_t fl = f.flags[i];
  (void)u;
  if (ir < nr && iz >= 1 && iz <= nz - 1) {
    float v = f.Ez[i];
    if (!(fl & SPIFFE_FL_EZ_ZERO))
      v = (float)((double)v + (f.Psi[i] - f.Psi[i - P]) / m.dz);
    if (ir == nr - 1)
      v = 0.f;
    f.Ez[i] = v;
    if (iz == 1)
      f.Ez[node(0, ir, P)] = ir == nr - 1 ? 0.f : (leftN ? v : -v);
    if (iz == nz - 1)
      f.Ez[node(nz, ir, P)] = ir == nr - 1 ? 0.f : (rightN ? v : -v);
  }
  if (iz <= nz - 1) {
    const bool zero_row = (leftN && iz == 0) || (rightN && iz == nz - 1);
    if (ir >= 1) {
      float v = f.Er[i];
      if (!(fl & SPIFFE_FL_ER_ZERO))
        v = (float)((double)v + (f.Psi[i] - f.Psi[i - 1]) / m.dr);
      f.Er[i] = zero_row ? 0.f : v;
      if (ir == 1)
        f.Er[node(iz, 0, P)] = zero_row ? 0.f : -v;
    }
  }
}

// EzImposed, ErImposed = -factor grad PsiImposed (:523-561)
__global__ void __launch_bounds__(BX *BY) k_imposed32(DevMesh m, DevFields32 f, double ff)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (ir > nr || iz > nz)
    return;
  const size_t i = node(iz, ir, P);
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;
  const int16_t fl = f.flags[i];
  if (ir < nr && iz >= 1 && iz <= nz - 1) {
    float v = f.EzImposed[i];
    if (!(fl & SPIFFE_FL_EZ_ZERO))
      v = (float)(-ff * (f.PsiImposed[i] - f.PsiImposed[i - P]) / m.dz);
    if (ir == nr - 1)
      v = 0.f;
    f.EzImposed[i] = v;
    if (iz == 1)
      f.EzImposed[node(0, ir, P)] = ir == nr - 1 ? 0.f : (leftN ? v : -v);
    if (iz == nz - 1)
      f.EzImposed[node(nz, ir, P)] = ir == nr - 1 ? 0.f : (rightN ? v : -v);
  }
  if (iz <= nz - 1) {
    const bool zero_row = (leftN && iz == 0) || (rightN && iz == nz - 1);
    if (ir >= 1) {
      float v = f.ErImposed[i];
      if (!(fl & SPIFFE_FL_ER_ZERO))
        v = (float)(-ff * (f.PsiImposed[i] - f.PsiImposed[i - 1]) / m.dr);
      f.ErImposed[i] = zero_row ? 0.f : v;
      if (ir == 1)
        f.ErImposed[node(iz, 0, P)] = zero_row ? 0.f : -v;
    }
  }
}

// shared bytes of a band of R rows: d with two halo rows a side, r0 and the
// mask with one, the row coefficients
size_t sor_smem(int R, int H)
{
  return (size_t)(R + 4) * 2 * H * 4 + (size_t)(R + 2) * 2 * H * 4 + 2 * (size_t)2 * H * 4 + (size_t)(R + 2) * 2 * H;
}

int sor_threads(int R, int H)
{
  const int slots = (R + 2) * (H / 4);
  return std::min(SOR_NT, std::max(128, (slots + 31) / 32 * 32));
}

} // namespace

extern "C" int s32_poisson_setup(const DevMesh *m, Poisson32Work *w, long long np_capacity, cudaStream_t s)
{
  const int nr = m->nr, nz = m->nz;
  const double dr = m->dr, dz = m->dz, dr2 = dr * dr, drdz = dr * dz;
  std::vector<double> Az(nr + 1), Ari(nr + 1), Aro(nr + 1), vol(nr + 1);
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
  std::vector<float> crow(nr + 1), drow(nr + 1);
  for (int ir = 0; ir <= nr; ir++) {
    crow[ir] = ir ? (float)(1 / dr2 * (1 + 1. / (2 * ir))) : (float)(1 / dr2);
    drow[ir] = ir ? (float)(1 / dr2 * (1 - 1. / (2 * ir))) : (float)(1 / dr2);
  }
  // SOR launch shape: the band of rows of every CTA must fit in shared memory
  int dev = 0, sms = 0, max_smem = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int rows = (m->right_bc == SPIFFE_DIRICHLET ? nz - 1 : nz - 2) - (m->left_bc == SPIFFE_DIRICHLET ? 0 : 1) + 1;
  const int cols = nr - 1, H = ((cols + 2) / 2 + 3) / 4 * 4; // half-row (one colour), a multiple of 4
  const size_t budget = (size_t)max_smem - 1024;
  // one CTA when the mesh fits one SM (no grid barriers); otherwise bands of
  // at least two rows (the halo exchange carries two rows) over all SMs
  int G = 1;
  if (sor_smem(rows, H) > budget || (size_t)rows * 2 * H > 65536) {
    G = std::min(sms, rows / 2);
    while (G < rows / 2 && sor_smem((rows + G - 1) / G, H) > budget)
      G++;
  }
  cudaError_t e = cudaSuccess;
  int occ = 0;
  const int R = (rows + G - 1) / G;
  if (G < 1 || G > sms || G > 255 || sor_smem(R, H) > budget)
    return (int)cudaErrorInvalidConfiguration; // the mesh does not fit the shared-memory bands
  w->grid = G;
  w->rows_per = R;
  w->smem = sor_smem(R, H);
  w->threads = sor_threads(R, H);
  e = cudaFuncSetAttribute(k_sor32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w->smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sor32, w->threads, w->smem);
  if (e == cudaSuccess && occ < 1)
    e = cudaErrorInvalidConfiguration;
  w->half = H;
  const size_t gx = (nr + 1 + BX - 1) / BX, gy = (nz + 1 + BY - 1) / BY;
  size_t parts = std::max<size_t>(2 * gx * gy, 4096);
  (void)np_capacity;
  if (e == cudaSuccess && !w->Az) {
    e = cudaMalloc(&w->Az, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->Ari, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->Aro, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->volume, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->crow, sizeof(float) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->drow, sizeof(float) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&w->scalars, sizeof(double) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&w->qreal_fixed, sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&w->st, sizeof(PcState));
    if (e == cudaSuccess) e = cudaMemsetAsync(w->st, 0, sizeof(PcState), s);
    if (e == cudaSuccess) e = cudaMalloc(&w->iters, sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&w->bar, sizeof(unsigned) * 2);
    if (e == cudaSuccess) e = cudaMalloc(&w->rsum, sizeof(unsigned long long) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&w->dpart, sizeof(double) * (size_t)sms * 2); // |rhs|, |r0| per CTA
    if (e == cudaSuccess) e = cudaMalloc(&w->xbuf, sizeof(float) * (size_t)2 * sms * 8 * H); // exchange rows
    if (e == cudaSuccess) e = cudaMalloc(&w->part, sizeof(double) * parts);
    w->part_n = parts;
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->Az, Az.data(), sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->Ari, Ari.data(), sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->Aro, Aro.data(), sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->volume, vol.data(), sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->crow, crow.data(), sizeof(float) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->drow, drow.data(), sizeof(float) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return (int)e;
}

extern "C" void s32_poisson_free(Poisson32Work *w)
{
  void *p[] = {w->Az, w->Ari, w->Aro, w->volume, w->crow, w->drow, w->scalars, w->qreal_fixed, w->st,
               w->iters, w->bar, w->rsum, w->dpart, w->xbuf, w->part, w->omega};
  for (void *q : p)
    cudaFree(q);
  *w = Poisson32Work();
}

static int ensure_omega32(const DevMesh *m, Poisson32Work *w, long long limit, cudaStream_t s)
{
  if (w->omega_n >= limit)
    return 0;
  cudaFree(w->omega);
  w->omega = nullptr;
  cudaError_t e = cudaMalloc(&w->omega, sizeof(float) * (size_t)limit);
  if (e != cudaSuccess)
    return (int)e;
  // Chebyshev acceleration (poisson.c:342-346, :117-119), in FP64 then rounded
  const double rz = m->dz / m->dr;
  const double rj = (cos(SPIFFE_PI / m->nz) + rz * rz * cos(SPIFFE_PI / m->nr)) / (1 + rz * rz);
  std::vector<float> om((size_t)limit);
  double omega = 1.0;
  for (long long n = 0; n < limit; n++) {
    om[(size_t)n] = (float)omega;
    omega = n == 0 ? 1.0 / (1 - rj * rj / 2) : 1.0 / (1 - rj * rj * omega / 4);
  }
  e = cudaMemcpyAsync(w->omega, om.data(), sizeof(float) * (size_t)limit, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  w->omega_n = limit;
  return (int)e;
}

extern "C" int s32_sor(const DevMesh *m, Poisson32Work *w, double *Psi, const double *rhs, const uint8_t *umask,
                       double accuracy, long long limit, PcState *st, DevCounts *cnt, cudaStream_t s)
{
  int rc = ensure_omega32(m, w, limit, s);
  if (rc)
    return rc;
  const double dz2 = m->dz * m->dz, dr2 = m->dr * m->dr;
  Sor32Args a{};
  a.Psi = Psi;
  a.rhs = rhs;
  a.umask = umask;
  a.omega = w->omega;
  a.crow = w->crow;
  a.drow = w->drow;
  a.a_d = 1 / dz2;
  a.e_d = -2 * (1 / dz2 + 1 / dr2);
  a.c4_d = 4 / dr2;
  a.e2c_d = a.e_d - 2 / dr2;
  a.dr2_inv = 1 / dr2;
  a.a = (float)a.a_d;
  a.e = (float)a.e_d;
  a.inv_e = (float)(1 / a.e_d);
  a.c4 = (float)a.c4_d;
  a.e2c = (float)a.e2c_d;
  a.inv_e2c = (float)(1 / a.e2c_d);
  a.accuracy = accuracy;
  a.limit = limit;
  a.xbuf = w->xbuf;
  a.arrive = w->rsum;
  a.release = w->rsum + 1;
  a.acc1 = w->rsum + 2;
  a.pub1 = w->rsum + 3;
  a.dpart = w->dpart;
  a.st = st;
  a.iters_out = w->iters;
  a.lo = m->left_bc == SPIFFE_DIRICHLET ? 0 : 1;
  a.hi = m->right_bc == SPIFFE_DIRICHLET ? m->nz - 1 : m->nz - 2;
  a.cols = m->nr - 1;
  a.H = w->half;
  a.rows_per = w->rows_per;
  cudaError_t e = cudaMemsetAsync(w->bar, 0, sizeof(unsigned) * 2, s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(w->rsum, 0, sizeof(unsigned long long) * 4, s);
  if (e != cudaSuccess)
    return (int)e;
  DevMesh mm = *m;
  void *args[] = {&mm, &a, &cnt};
  e = cudaLaunchCooperativeKernel((const void *)k_sor32, dim3(w->grid), dim3(w->threads), args, w->smem, s);
  spiffe_note_launches(1);
  return (int)e;
}

extern "C" int s32_poisson_correction(const DevMesh *m, const DevFields32 *f, const DevBeam32 *b, DevCounts *cnt,
                                      long long np_bound, const PoissonHostOptions *o, const S32Scales *sc,
                                      Poisson32Work *w, cudaStream_t s)
{
  const dim3 block(BX, BY), grid((m->nr + 1 + BX - 1) / BX, (m->nz + 1 + BY - 1) / BY);
  const int nblk = grid.x * grid.y;
  const bool sc_on = o->space_charge && np_bound > 0;
  k_apparent32<<<grid, block, 0, s>>>(*m, *f, w->Az, w->Ari, w->Aro, 0, w->part);
  k_finish_sum32<<<1, 1024, 0, s>>>(w->part, nblk, 2, w->scalars + 0);
  k_finish_sum32<<<1, 1024, 0, s>>>(w->part + 1, nblk, 2, w->scalars + 1);
  spiffe_note_launches(3);
  cudaError_t e = cudaMemsetAsync(w->qreal_fixed, 0, sizeof(long long), s);
  if (e != cudaSuccess)
    return (int)e;
  if (sc_on) {
    e = cudaMemsetAsync(f->Qp, 0, sizeof(long long) * (size_t)(m->nz + 1) * m->pitch, s);
    if (e != cudaSuccess)
      return (int)e;
    k_remove32<<<blocks_for(np_bound, RT), RT, 0, s>>>(*m, *f, *b, cnt, *sc, w->qreal_fixed);
    spiffe_note_launches(1);
  }
  k_combine32<<<grid, block, 0, s>>>(*m, *f, sc->qQ, sc_on ? 1 : 0, w->part);
  k_finish_sum32<<<1, 1024, 0, s>>>(w->part, nblk, 1, w->scalars + 3);
  k_state32<<<1, 1, 0, s>>>(w->st, w->scalars, w->qreal_fixed, sc->qQ, o->space_charge, o->error_charge_threshold);
  k_scale32<<<grid, block, 0, s>>>(*m, *f, w->volume, w->st);
  spiffe_note_launches(4);
  if (o->guess_code) {
    k_guess32<<<grid, block, 0, s>>>(*m, *f, o->guess_code, w->st);
    spiffe_note_launches(1);
  }
  int rc = s32_sor(m, w, f->Psi, f->Q, f->umask, o->accuracy, o->maximum_iterations, w->st, cnt, s);
  if (rc)
    return rc;
  k_subtract32<<<grid, block, 0, s>>>(*m, *f, w->st);
  // the reference recomputes the apparent charge afterwards (:333-439); the
  // particles have not moved, so their charge per node is the same Qp
  k_apparent32<<<grid, block, 0, s>>>(*m, *f, w->Az, w->Ari, w->Aro, 1, w->part);
  k_combine32<<<grid, block, 0, s>>>(*m, *f, sc->qQ, sc_on ? 1 : 0, w->part);
  spiffe_note_launches(3);
  return (int)cudaGetLastError();
}

extern "C" int s32_poisson_report(Poisson32Work *w, spiffe_poisson_report *rep, cudaStream_t s)
{
  PcState st;
  double drv[8];
  cudaMemcpyAsync(&st, w->st, sizeof(st), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(drv, w->scalars, sizeof(drv), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  rep->ran = st.do_solve;
  rep->iterations = st.iterations;
  rep->Qreal = st.Qreal;
  rep->Qerror = st.Qerror;
  rep->Qsurface = st.Qsurface;
  rep->residual = st.residual;
  rep->driving = 0;
  return (int)e;
}

extern "C" int s32_imposed_field(const DevMesh *m, const DevFields32 *f, double factor, cudaStream_t s)
{
  const dim3 block(BX, BY), grid((m->nr + 1 + BX - 1) / BX, (m->nz + 1 + BY - 1) / BY);
  k_imposed32<<<grid, block, 0, s>>>(*m, *f, factor);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}
