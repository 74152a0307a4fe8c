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
// a round of half-sweeps reads no global memory except the halo rows that the
// adjacent CTAs updated; the rows of each colour are stored as separate
// contiguous halves so a warp's accesses are conflict-free.  A band carries
// a halo deep enough for several half-sweeps per grid barrier (temporal
// blocking).  The per-CTA |residual| sums of every half-sweep are added in
// 64-bit fixed point with the barrier's arrival, so every CTA takes the
// same stop decision from order-independent totals.  When the residual has fallen 2^8-fold the
// correction is folded into Psi and the residual formed again in FP64
// (iterative refinement), so FP32 rounding of d never limits convergence.
#include "split32.cuh"
#include "modules.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

constexpr int BX = 32, BY = 8, RT = 256;

__device__ bool surface_cell(const DevMesh &m, int16_t fl, int iz, int ir)
{
  return (fl & SPIFFE_FL_IS_METAL) || (iz == 0 && m.left_bc == SPIFFE_NEUMANN) ||
         (iz == m.nz - 1 && m.right_bc == SPIFFE_NEUMANN) || (ir == m.nr - 1 && m.upper_bc == SPIFFE_NEUMANN);
}

// The particles' own charge (:190-242) in fixed point: Qp[node] receives the
// removed charge of each non-metal node, Qreal the total.
__global__ void __launch_bounds__(RT) k_remove32(DevMesh m, DevFields32 f, DevBeam32 b, const DevCounts *cnt,
                                                  S32Scales sc, long long *qreal_fixed)
{
  __shared__ long long sh[RT / 32];
  const long ip = (long)blockIdx.x * RT + threadIdx.x;
  const bool lsm = m.modes & SPIFFE_FL_LONGIT_SMEAR, rsm = m.modes & SPIFFE_FL_RADIAL_SMEAR;
  int nodes[4] = {-1, -1, -1, -1};
  long long q[4] = {0, 0, 0, 0};
  long long mine = 0;
  if (ip < (long)cnt->np && (b.status[ip] & S32_ACTIVE)) {
    const int nz = m.nz, nr = m.nr, P = m.pitch;
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
#pragma unroll
  for (int k = 0; k < 4; k++) {
    // slots 1 and 3 carry charge only with longitudinal smearing, 2 and 3
    // only with radial smearing (their weight is zero otherwise); the flags
    // are the mesh's, the same in every lane
    if (((k & 1) && !lsm) || ((k & 2) && !rsm))
      continue;
    // same grouping as the current deposition; cell-sorted particles
    // usually share the node across the warp, which one vote settles
    const int nd0 = __shfl_sync(0xffffffffu, nodes[k], 0);
    const unsigned grp =
        __all_sync(0xffffffffu, nodes[k] == nd0) ? 0xffffffffu : __match_any_sync(0xffffffffu, nodes[k]);
    const unsigned long long biased = (unsigned long long)(q[k] + (1LL << 42));
    const unsigned lo = (unsigned)(biased & ((1u << 22) - 1)), hi = (unsigned)(biased >> 22);
    const unsigned slo = __reduce_add_sync(grp, lo), shi = __reduce_add_sync(grp, hi);
    if (nodes[k] >= 0 && (threadIdx.x & 31) == __ffs(grp) - 1) {
      const long long tot = ((long long)shi << 22) + (long long)slo - (long long)__popc(grp) * (1LL << 42);
      if (tot)
        atomic_add_ll(f.Qp + nodes[k], tot);
    }
  }
  // exact integer total of the removed charge: warp sums, then the CTA's
  for (int o = 16; o > 0; o >>= 1)
    mine += __shfl_down_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = mine;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int w = 0; w < RT / 32; w++)
      s += sh[w];
    if (s)
      atomic_add_ll(qreal_fixed, s);
  }
}

// One pass of the correction's charge: the apparent charge from the flux of
// E (poisson_correction.c:141-182, second pass :335-375) in FP64 from the
// FP32 fields, minus the particles' fixed-point charge per node (the FP64
// form's subtraction on Q, :190-242), and on the first pass the solver's
// right-hand side -Q/(V eps0) over iz < nz, ir < nr (:268-274) with the
// per-block sums of the surface charge, its centroid moment and the error
// charge (:244-256) taken before the scaling.  The scaling is unconditional:
// the pass after the solve recomputes every node it touched, so a solve
// skipped by the threshold test leaves the same Q.  Nodes outside iz < nz,
// ir < nr keep their Q minus the particles' charge.
__global__ void __launch_bounds__(BX *BY) k_charge32(DevMesh m, DevFields32 f, const double *Az_, const double *Ari,
                                                      const double *Aro, const double *volume, int second, double qQ,
                                                      int space_charge, double *part)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  const double eps = SPIFFE_EPSILON_O;
  double qs = 0, cen = 0, qe = 0;
  if (ir <= nr && iz <= nz) {
    const size_t i = node(iz, ir, P);
    const bool inner = ir < nr && iz < nz;
    double q;
    if (inner) {
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
        q = 0;
      } else {
        q = dQ;
        cen = dQ * (iz * m.dz + m.zmin);
      }
    } else {
      q = f.Q[i];
    }
    if (space_charge) {
      const long long pq = f.Qp[i];
      if (pq)
        q -= (double)pq * qQ;
    }
    if (inner)
      qe = q;
    f.Q[i] = (!second && inner) ? -q / (volume[ir] * SPIFFE_EPSILON_O) : q;
  }
  if (second)
    return;
  // fixed-order block sums of (qs, cen, qe)
  __shared__ double sh[3][BX * BY / 32];
  for (int o = 16; o > 0; o >>= 1) {
    qs += __shfl_down_sync(0xffffffffu, qs, o);
    cen += __shfl_down_sync(0xffffffffu, cen, o);
    qe += __shfl_down_sync(0xffffffffu, qe, o);
  }
  const int t = threadIdx.y * BX + threadIdx.x;
  if ((t & 31) == 0) {
    sh[0][t >> 5] = qs;
    sh[1][t >> 5] = cen;
    sh[2][t >> 5] = qe;
  }
  __syncthreads();
  if (t < 3) {
    double v = 0;
    for (int w = 0; w < BX * BY / 32; w++)
      v += sh[t][w];
    part[3 * (blockIdx.y * gridDim.x + blockIdx.x) + t] = v;
  }
}

// The grid's sums of k_charge32's partials (fixed order) into sc[0]
// (Qsurface), sc[1] (centroid moment), sc[3] (Qerror), then the correction's
// state and the error-charge threshold decision.
__global__ void k_charge_state32(const double *part, int n, double *sc, PcState *st, const long long *qreal_fixed,
                                 double qQ, int space_charge, double threshold)
{
  __shared__ double sh[3][1024];
  double v[3] = {0, 0, 0};
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    for (int k = 0; k < 3; k++)
      v[k] += part[3 * (size_t)i + k];
  for (int k = 0; k < 3; k++)
    sh[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 3; k++)
        sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sc[0] = sh[0][0];
    sc[1] = sh[1][0];
    sc[3] = sh[2][0];
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
  float *xbuf;                  // exchange rows [2][grid][2 sides][depth rows][2 parities][H]
  unsigned long long *count;    // barrier arrivals, monotonic over the launch
  unsigned long long *slots;    // [3][SOR_SLOTS] fixed-point sums, one set per barrier in rotation
  double *dpart;                // [grid][2] |rhs| and |r0| partials
  PcState *st;
  long long *iters_out;
  int lo, hi, cols, H, rows_per; // H: half-row length, a multiple of 4
};

constexpr int SOR_SLOTS = 8; // sums carried by one barrier: one per half-sweep of a round, and sum |e d|

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p)
{
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p)
{
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Bounded grid barrier for thread 0 of every CTA (the caller synchronises
// the CTA before and after).  Barrier number `gen` (counted by the caller
// from 1) adds this CTA's NV fixed-point values to slot set gen % 3, then,
// after a fence that releases the CTA's earlier writes, one arrival to the
// monotonic counter; it is passed once the counter reaches grid * gen, and
// the acquire of that read makes every CTA's writes and sums visible.  The
// sums of barrier gen are read between barriers gen and gen + 1, so CTA 0
// clears set (gen - 1) % 3 once past barrier gen, before its next arrival;
// barrier gen + 2 adds into it only after passing gen + 1.  Returns false
// (and raises the device error bit) when the others do not arrive within
// the poll limit.
template <int NV>
__device__ bool grid_barrier(const Sor32Args &s, const unsigned long long *v, unsigned gen, DevCounts *cnt)
{
  if (NV > 0) {
    unsigned long long *set = s.slots + (size_t)(gen % 3) * SOR_SLOTS;
#pragma unroll
    for (int k = 0; k < NV; k++)
      if (v[k])
        asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(set + k), "l"(v[k]) : "memory");
  }
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(s.count), "l"(1ull) : "memory");
  const unsigned long long target = (unsigned long long)gridDim.x * gen;
  unsigned long long polls = 0;
  while (ld_acquire64(s.count) < target) {
    if (++polls > (1ull << 24)) {
      atomicOr(&cnt->error, SPIFFE_DEV_ERR_BARRIER);
      return false;
    }
    if (polls > 64)
      __nanosleep(20);
  }
  if (blockIdx.x == 0) {
    unsigned long long *old = s.slots + (size_t)((gen + 2) % 3) * SOR_SLOTS;
#pragma unroll
    for (int k = 0; k < SOR_SLOTS; k++)
      asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(old + k), "l"(0ull) : "memory");
  }
  return true;
}

// Band of rows of CTA b: [start, start+n) of the update rows lo..hi.
__device__ __forceinline__ void band(int rows, int b, int G, int &start, int &n)
{
  const int base = rows / G, rem = rows % G;
  n = base + (b < rem ? 1 : 0);
  start = b * base + (b < rem ? b : rem);
}

// r0 = rhs - A Psi (FP64, Psi read through L2) into B for the mesh rows
// iz0 .. iz0+nb-1 (B row i = mesh row iz0+i) that the SOR updates; a node
// that the SOR does not update (metal, outside rows lo..hi, ir >= cols)
// gets NaN, which marks it for the sweeps.  Adds this thread's share of
// sum |rhs| and sum |r0| over the band's own rows [own_lo, own_hi] to
// *drive and *rsum.
__device__ void form_r0(const DevMesh &m, const Sor32Args &s, float *B, int iz0, int nb, int own_lo, int own_hi,
                        double *drive, double *rsum)
{
  const int nz = m.nz, P = m.pitch, H = s.H, cols = s.cols;
  double d = 0, q = 0;
#pragma unroll 4
  for (int i = 0; i < nb; i++) {
    const int iz = iz0 + i;
    const bool upd = iz >= s.lo && iz <= s.hi, own = iz >= own_lo && iz <= own_hi;
    const long up = (iz == 0 && s.lo == 0) ? P : (iz == nz - 1 && s.hi == nz - 1 ? -P : P);
    const long dn = (iz == 0 && s.lo == 0) ? P : -P;
    for (int t = threadIdx.x; t < 2 * H; t += blockDim.x) {
      const int p = t / H, k = t - p * H, ir = 2 * k + p;
      float r0 = __int_as_float(0x7fc00000); // quiet NaN: not updated
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
          else {
            const double h = 0.5 / ir; // = 1/(2 ir), correctly rounded either way
            ap = s.a_d * lr + s.dr2_inv * (1 + h) * __ldcg(s.Psi + j + 1) + s.dr2_inv * (1 - h) * __ldcg(s.Psi + j - 1) +
                 s.e_d * psi;
          }
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

// A thread's share of the sweeps: one column group -- the four nodes of
// each colour half-row at half-row offset 4q, i.e. mesh columns 8q..8q+7 --
// on a run of rows of the band, with the row coefficients of those columns
// held in registers for the whole solve.
struct Strip {
  int q, g, ng;              // column group, row group, row groups in use
  int off0, off1;            // offsets of the column group in the parity-0 and parity-1 half rows
  float4 cr0, cr1, dr0, dr1; // c(ir) and d(ir) of the eight columns (the axis node: 4/dr^2 and 0)
  float ex, iex;             // diagonal of column 8q and its inverse (e - 2c on the axis)
};

// The SOR update (or, with UNDO, its inverse) of one node: res = A d - r0
// with the diagonal term, d -= w res / e; a node whose r0 is NaN is left
// alone.  UNDO restores the value before the update from the value after
// it: new = old (1-w) - w (nb - r0)/e, so old = (new + w (nb - r0)/e)/(1-w)
// (w > 1 after the first half-sweep).
template <bool UNDO>
__device__ __forceinline__ void sor_node(float &x, float a, float ud, float c, float r, float dl, float l, float b,
                                         float e, float wie, float inv1w, float &acc)
{
  const float nb = fmaf(a, ud, fmaf(c, r, fmaf(dl, l, -b))); // neighbours - r0
  if (b == b) {
    if (UNDO) {
      x = fmaf(wie, nb, x) * inv1w;
    } else {
      const float res = fmaf(e, x, nb);
      x = fmaf(-wie, res, x);
      acc += fabsf(res);
    }
  }
}

// One row of one colour for a strip: D row j (mesh row iz), neighbour rows
// uj, dj, B row j - 1; P is the parity of the row's nodes of this colour.
// With LOAD_OD the other colour of the row (o) and the row below (d) are
// loaded here, otherwise the caller passes them; u returns the row above.
// Returns the sum of |residual|.  With x0/x1 the row's new values of both
// colours are also stored there for the neighbouring CTAs.
template <int P, bool UNDO, bool DSUM, bool LOAD_OD>
__device__ __forceinline__ float sor_row(const Sor32Args &s, const Strip &t, float *D, const float *B, int j, int uj,
                                         int dj, float4 &o, float4 &d, float4 &u, float wie, float wiex, float inv1w,
                                         float *dsum, float *x0, float *x1)
{
  const int H2 = 2 * s.H, so = P ? t.off1 : t.off0, oo = P ? t.off0 : t.off1;
  float *row = D + j * H2;
  float4 sv = *reinterpret_cast<const float4 *>(row + so);
  if (LOAD_OD) {
    o = *reinterpret_cast<const float4 *>(row + oo);
    d = *reinterpret_cast<const float4 *>(D + dj * H2 + so);
  }
  // the fifth neighbour in r: node 8q-1 (parity 0; read but weighted 0 on
  // the axis) or node 8q+8 (parity 1; beyond the mesh for the last group,
  // whose node is not updated)
  const float nbr = P ? row[oo + 4] : row[oo - 1];
  u = *reinterpret_cast<const float4 *>(D + uj * H2 + so);
  const float4 b = *reinterpret_cast<const float4 *>(B + (j - 1) * H2 + so);
  const float4 c = P ? t.cr1 : t.cr0, dl = P ? t.dr1 : t.dr0;
  const float a = s.a, e = s.e;
  float acc = 0.f;
  if (P == 0) {
    sor_node<UNDO>(sv.x, a, u.x + d.x, c.x, o.x, dl.x, nbr, b.x, t.ex, wiex, inv1w, acc);
    sor_node<UNDO>(sv.y, a, u.y + d.y, c.y, o.y, dl.y, o.x, b.y, e, wie, inv1w, acc);
    sor_node<UNDO>(sv.z, a, u.z + d.z, c.z, o.z, dl.z, o.y, b.z, e, wie, inv1w, acc);
    sor_node<UNDO>(sv.w, a, u.w + d.w, c.w, o.w, dl.w, o.z, b.w, e, wie, inv1w, acc);
  } else {
    sor_node<UNDO>(sv.x, a, u.x + d.x, c.x, o.y, dl.x, o.x, b.x, e, wie, inv1w, acc);
    sor_node<UNDO>(sv.y, a, u.y + d.y, c.y, o.z, dl.y, o.y, b.y, e, wie, inv1w, acc);
    sor_node<UNDO>(sv.z, a, u.z + d.z, c.z, o.w, dl.z, o.z, b.z, e, wie, inv1w, acc);
    sor_node<UNDO>(sv.w, a, u.w + d.w, c.w, nbr, dl.w, o.w, b.w, e, wie, inv1w, acc);
  }
  *reinterpret_cast<float4 *>(row + so) = sv;
  if (DSUM)
    *dsum += fabsf(sv.x) + fabsf(sv.y) + fabsf(sv.z) + fabsf(sv.w);
  if (x0) {
    __stcg(reinterpret_cast<float4 *>(x0 + so), sv);
    __stcg(reinterpret_cast<float4 *>(x0 + oo), o);
  }
  if (x1) {
    __stcg(reinterpret_cast<float4 *>(x1 + so), sv);
    __stcg(reinterpret_cast<float4 *>(x1 + oo), o);
  }
  return acc;
}

// Rows j0..j1 of a strip in pairs, the first of parity P0 (rows alternate
// parity).  The second row of a pair takes its other colour from the first
// row's row above and its row below from the first row's other colour (the
// sweep changes neither), except where a Dirichlet end row mirrors its
// neighbour.  Adds |residual| and, with DSUM, |d| over own rows to acc, dacc.
template <int P0, bool UNDO, int HD, bool DSUM>
__device__ __forceinline__ void strip_rows(const DevMesh &m, const Sor32Args &s, const Strip &t, float *D,
                                           const float *B, int iz_first, int nrow, int j0, int j1, float wie, float wiex,
                                           float inv1w, float *xo, float &acc, float &dacc)
{
  const int nz = m.nz, H2 = 2 * s.H;
  const bool lo0 = s.lo == 0, hin = s.hi == nz - 1;
  for (int j = j0; j <= j1; j += 2) {
    float4 oA, dA, uA;
    int ujA;
    {
      const int iz = iz_first + j - HD;
      // Dirichlet end rows mirror their only neighbour (poisson.c:369-375, :404-410)
      ujA = (iz == nz - 1 && hin) ? j - 1 : j + 1;
      const int dj = (iz == 0 && lo0) ? j + 1 : j - 1;
      float *x0 = nullptr, *x1 = nullptr;
      if (xo) {
        if (j < 2 * HD)
          x0 = xo + (j - HD) * H2;
        if (j >= nrow)
          x1 = xo + HD * H2 + (j - nrow) * H2;
      }
      float ds = 0.f;
      const float r = sor_row<P0, UNDO, DSUM, true>(s, t, D, B, j, ujA, dj, oA, dA, uA, wie, wiex, inv1w, &ds, x0, x1);
      if (j >= HD && j < HD + nrow) {
        acc += r;
        dacc += ds;
      }
    }
    const int jj = j + 1;
    if (jj <= j1) {
      const int iz = iz_first + jj - HD;
      const int uj = (iz == nz - 1 && hin) ? jj - 1 : jj + 1;
      const int dj = (iz == 0 && lo0) ? jj + 1 : jj - 1;
      constexpr int P1 = P0 ^ 1;
      float4 o = uA, d = oA, u;
      if (ujA != jj) // the first row mirrored: its row above was not this row
        o = *reinterpret_cast<const float4 *>(D + jj * H2 + (P1 ? t.off0 : t.off1));
      if (dj != j) // this row mirrors: its row below is the row above
        d = *reinterpret_cast<const float4 *>(D + dj * H2 + (P1 ? t.off1 : t.off0));
      float *x0 = nullptr, *x1 = nullptr;
      if (xo) {
        if (jj < 2 * HD)
          x0 = xo + (jj - HD) * H2;
        if (jj >= nrow)
          x1 = xo + HD * H2 + (jj - nrow) * H2;
      }
      float ds = 0.f;
      const float r = sor_row<P1, UNDO, DSUM, false>(s, t, D, B, jj, uj, dj, o, d, u, wie, wiex, inv1w, &ds, x0, x1);
      if (jj >= HD && jj < HD + nrow) {
        acc += r;
        dacc += ds;
      }
    }
  }
}

// One colour c over D rows jlo..jhi (mesh row iz = iz_first + j - HD; B row
// j - 1).  The rows are cut into runs of an even length, one per row group,
// so every thread of a warp starts on a row of the same parity.  Returns
// this thread's sum of |residual| over the own rows HD..HD+nrow-1 and, with
// DSUM, their sum of |d| in *dsum.  With xo, the first HD and the last HD
// own rows also go to the exchange buffer (side 0: rows HD.., side 1: rows
// nrow..).
template <bool UNDO, int HD, bool DSUM = false>
__device__ __forceinline__ float sweep_rows(const DevMesh &m, const Sor32Args &s, const Strip &t, float *D,
                                            const float *B, int iz_first, int nrow, int jlo, int jhi, int c, float w,
                                            float *xo = nullptr, float *dsum = nullptr)
{
  float acc = 0.f, dacc = 0.f;
  if (t.g < t.ng) {
    const int n = jhi - jlo + 1, per = 2 * ((n + 2 * t.ng - 1) / (2 * t.ng));
    const int j0 = jlo + t.g * per, j1 = min(jhi, j0 + per - 1);
    const float wie = w * s.inv_e, wiex = w * t.iex, inv1w = UNDO ? 1.f / (1.f - w) : 0.f;
    if (((c + iz_first + j0 - HD) & 1) == 0)
      strip_rows<0, UNDO, HD, DSUM>(m, s, t, D, B, iz_first, nrow, j0, j1, wie, wiex, inv1w, xo, acc, dacc);
    else
      strip_rows<1, UNDO, HD, DSUM>(m, s, t, D, B, iz_first, nrow, j0, j1, wie, wiex, inv1w, xo, acc, dacc);
  }
  if (DSUM)
    *dsum = dacc;
  return acc;
}

// Psi += d on the band's own nodes (FP64); own rows are D rows hd ..
// hd+nrow-1.  Nodes the SOR does not update keep d = 0.  Four rows' loads
// are issued before their stores.
__device__ void fold_d(const Sor32Args &s, int P, const float *D, int iz_first, int nrow, int hd)
{
  const int H = s.H, cols = s.cols;
  for (int t = threadIdx.x; t < 2 * H; t += blockDim.x) {
    const int p = t / H, k = t - p * H, ir = 2 * k + p;
    if (ir >= cols)
      continue;
    for (int j = hd; j < hd + nrow; j += 4) {
      double v[4];
      float dd[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        dd[u] = j + u < hd + nrow ? D[((j + u) * 2 + p) * H + k] : 0.f;
        v[u] = dd[u] != 0.f ? __ldcg(s.Psi + node(iz_first + j + u - hd, ir, P)) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (dd[u] != 0.f)
          __stcg(s.Psi + node(iz_first + j + u - hd, ir, P), v[u] + (double)dd[u]);
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
// start.  Each round runs HD half-sweeps (colours 0, 1, 0, ...) between two
// grid barriers: a CTA's band carries HD halo rows on each side, sweep k of
// the round also updates the HD-1-k nearest halo rows (from exactly the
// inputs the neighbour uses, so with the same result), and the last sweep
// needs nothing from the neighbours.  Every half-sweep's |residual| sum
// arrives with the barrier, so the reference's stop test runs after every
// half-sweep; when it fires before the last sweep of the round, the later
// sweeps are undone in reverse order over the rows they updated, before
// the neighbours' rows replace the halo.
constexpr int SOR_NT = 768; // most threads per CTA of the shared-memory kernel (80 registers each)

template <int HD>
__global__ void __launch_bounds__(SOR_NT) k_sor32(DevMesh m, Sor32Args s, DevCounts *cnt)
{
  static_assert(HD % 2 == 0 && HD + 1 <= SOR_SLOTS, "rounds of an even number of half-sweeps");
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[64];
  __shared__ float redf[HD + 1][32];
  __shared__ float om_sh[2][HD]; // Chebyshev factors of this round and the next
  __shared__ int ok_sh, stop_sh, nundo_sh, rebase_sh;
  __shared__ double total_sh, thr_sh, quantum_sh, base_sh;
  __shared__ long long result_sh;
  if (s.st && !s.st->do_solve)
    return;
  const int nz = m.nz, P = m.pitch, H = s.H, Q = s.H >> 2, cols = s.cols, R = s.rows_per;
  const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x, NT = blockDim.x;
  const bool halo = G > 1;
  int start, nrow;
  band(s.hi - s.lo + 1, b, G, start, nrow);
  const int iz_first = s.lo + start;
  // shared layout (32-bit words): D[(R+2HD)][2][H] d for mesh rows
  // iz_first-HD .. iz_first+R+HD-1 (D row iz - iz_first + HD) and
  // B[(R+2HD-2)][2][H] r0 (NaN where not updated) for rows iz_first-HD+1 ..
  // (B row = D row - 1); row j's nodes of parity p are the contiguous run
  // (j*2+p)*H .. +H
  float *D = (float *)smem;
  float *B = D + (R + 2 * HD) * 2 * H;
  for (int t = tid; t < (R + 2 * HD) * 2 * H; t += NT)
    D[t] = 0.f;
  Strip st;
  st.ng = NT / Q;
  st.q = tid % Q;
  st.g = tid / Q;
  st.off0 = 4 * st.q;
  st.off1 = H + 4 * st.q;
  {
    const float *cr = s.crow, *dr = s.drow;
    float c0[4], c1[4], d0[4], d1[4];
    for (int i = 0; i < 4; i++) {
      const int ir0 = 8 * st.q + 2 * i, ir1 = ir0 + 1;
      c0[i] = ir0 < cols ? cr[ir0] : 0.f;
      d0[i] = ir0 < cols ? dr[ir0] : 0.f;
      c1[i] = ir1 < cols ? cr[ir1] : 0.f;
      d1[i] = ir1 < cols ? dr[ir1] : 0.f;
    }
    if (st.q == 0) { // the axis node (poisson.c:386-387)
      c0[0] = s.c4;
      d0[0] = 0.f;
    }
    st.cr0 = make_float4(c0[0], c0[1], c0[2], c0[3]);
    st.cr1 = make_float4(c1[0], c1[1], c1[2], c1[3]);
    st.dr0 = make_float4(d0[0], d0[1], d0[2], d0[3]);
    st.dr1 = make_float4(d1[0], d1[1], d1[2], d1[3]);
    st.ex = st.q == 0 ? s.e2c : s.e;
    st.iex = st.q == 0 ? s.inv_e2c : s.inv_e;
  }
  const int iz_last = iz_first + nrow - 1;
  double drive = 0, r0sum = 0;
  form_r0(m, s, B, iz_first - (HD - 1), nrow + 2 * (HD - 1), iz_first, iz_last, &drive, &r0sum);
  // rows outside lo..hi that the driving sum still covers (iz < nz): the
  // first CTA takes those below lo, the last those above hi
  if (s.rhs) {
    if (b == 0)
      for (int iz = 0; iz < s.lo; iz++)
        for (int ir = tid; ir < cols; ir += NT)
          drive += fabs(s.rhs[node(iz, ir, P)]);
    if (b == G - 1)
      for (int iz = s.hi + 1; iz < nz; iz++)
        for (int ir = tid; ir < cols; ir += NT)
          drive += fabs(s.rhs[node(iz, ir, P)]);
  }
  // fixed-order block sums of the |rhs| and |r0| partials
  block_sum2(drive, red, 0);
  block_sum2(r0sum, red, 1);
  __syncthreads();
  unsigned gen = 0; // barriers passed (thread 0)
  if (tid == 0) {
    double t = 0, t2 = 0;
    for (int w = 0; w < (NT + 31) / 32; w++) {
      t += red[w];
      t2 += red[32 + w];
    }
    int ok = 1;
    if (halo) {
      __stcg(s.dpart + 2 * b, t);
      __stcg(s.dpart + 2 * b + 1, t2);
      ok = grid_barrier<0>(s, nullptr, ++gen, cnt);
      t = t2 = 0;
      for (int i = 0; i < G; i++) {
        t += __ldcg(s.dpart + 2 * i);
        t2 += __ldcg(s.dpart + 2 * i + 1);
      }
    }
    ok_sh = ok;
    thr_sh = s.accuracy * t;
    if (b == 0 && s.st)
      s.st->driving = t;
    base_sh = t2;
    quantum_sh = fmax(fmax(base_sh, thr_sh), 1e-280) / 1073741824.0;
    rebase_sh = 0;
    result_sh = -1;
    total_sh = 0;
  }
  __syncthreads();
  if (tid < HD)
    om_sh[0][tid] = tid < s.limit ? s.omega[tid] : 0.f;
  __syncthreads();
  if (!ok_sh)
    return;
  const int nw = (NT + 31) / 32, Q2 = 2 * Q;
  // the halo rows a thread fetches: elements tid + u NT (u < PRE) of the 2HD
  // rows x 2Q float4s of the neighbours' exchanged rows (rows 0..HD-1 from
  // the CTA before, HD..2HD-1 from the one after), as row and column
  constexpr int PRE = 3;
  const int ne = 2 * HD * Q2;
  int er[PRE], ec[PRE];
#pragma unroll
  for (int u = 0; u < PRE; u++) {
    er[u] = (tid + u * NT) / Q2;
    ec[u] = tid + u * NT - er[u] * Q2;
  }
  for (long long n0 = 0; n0 < s.limit; n0 += HD) {
    const int keff = (int)(s.limit - n0 < HD ? s.limit - n0 : HD);
    const bool last = n0 + HD >= s.limit;
    // the last sweep of a round also writes the exchanged rows for the neighbours
    float *xo = halo ? s.xbuf + (size_t)((n0 / HD) & 1) * G * 4 * HD * H + (size_t)b * 4 * HD * H : nullptr;
    const int rb = (int)((n0 / HD) & 1);
    // the next round's factors load while this one sweeps
    const float om_next = tid < HD && n0 + HD + tid < s.limit ? __ldg(s.omega + n0 + HD + tid) : 0.f;
#pragma unroll 1
    for (int k = 0; k < HD; k++) {
      float v = 0.f;
      if (k < keff) {
        const int ext = halo ? HD - 1 - k : 0;
        if (k == HD - 1) { // the last sweep also sums |d| over the own nodes it updates
          float ds = 0.f;
          v = sweep_rows<false, HD, true>(m, s, st, D, B, iz_first, nrow, HD, HD + nrow - 1, 1, om_sh[rb][k], xo,
                                          &ds);
          for (int o = 16; o > 0; o >>= 1)
            ds += __shfl_down_sync(0xffffffffu, ds, o);
          if ((tid & 31) == 0)
            redf[HD][tid >> 5] = ds;
        } else {
          v = sweep_rows<false, HD>(m, s, st, D, B, iz_first, nrow, HD - ext, HD + nrow - 1 + ext, k & 1,
                                    om_sh[rb][k]);
        }
      } else if (k == HD - 1 && (tid & 31) == 0) {
        redf[HD][tid >> 5] = 0.f;
      }
      // fixed-order sums: per warp in FP32 here, across warps in FP64 by warp 0 below
      for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
      if ((tid & 31) == 0)
        redf[k][tid >> 5] = v;
      if (k == HD - 1 && tid < HD)
        om_sh[rb ^ 1][tid] = om_next;
      __syncthreads();
    }
    double part[HD + 1]; // |residual| of each half-sweep, then |d| after the last
    if (tid < 32) {
#pragma unroll
      for (int k = 0; k <= HD; k++) {
        double v = tid < nw ? (double)redf[k][tid] : 0.0;
        for (int o = 16; o > 0; o >>= 1)
          v += __shfl_down_sync(0xffffffffu, v, o);
        part[k] = v;
      }
    }
    float4 pre[PRE];
#pragma unroll
    for (int u = 0; u < PRE; u++)
      pre[u] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float *xi = s.xbuf + (size_t)((n0 / HD) & 1) * G * 4 * HD * H;
    if (halo) {
      if (tid == 0) {
        // this CTA's |residual| sums in quanta of 2^-30 of the larger of the
        // refinement base and the stop threshold, capped at 2^40 quanta, and
        // its |e| sum |d| in quanta 2^12 times larger, capped at 2^50
        unsigned long long qv[HD + 1];
#pragma unroll
        for (int k = 0; k < HD; k++) {
          const double x = part[k] / quantum_sh;
          qv[k] = part[k] == 0 ? 0ull
                               : (x >= 1099511627776.0 ? 1099511627776ull : ((unsigned long long)llrint(x) | 1ull));
        }
        const double xd = part[HD] * fabs(s.e_d) / (quantum_sh * 4096.0);
        qv[HD] = xd >= 1125899906842624.0 ? 1125899906842624ull : (unsigned long long)llrint(xd);
        ok_sh = grid_barrier<HD + 1>(s, qv, ++gen, cnt);
      }
      __syncthreads();
      if (!ok_sh)
        return;
      // the neighbours' rows, held in registers until the stop test has run
      if (!last) {
#pragma unroll
        for (int u = 0; u < PRE; u++) {
          const int nb_ = er[u] < HD ? b - 1 : b + 1;
          if (tid + u * NT < ne && nb_ >= 0 && nb_ < G)
            pre[u] = __ldcg(reinterpret_cast<const float4 *>(xi + (size_t)nb_ * 4 * HD * H +
                                                             (er[u] < HD ? 2 * HD * H : 0)) +
                            (er[u] < HD ? er[u] : er[u] - HD) * Q2 + ec[u]);
        }
      }
    }
    if (tid == 0) {
      double tot[HD + 1];
      unsigned long long tq[HD + 1];
      const unsigned long long *set = s.slots + (size_t)(gen % 3) * SOR_SLOTS;
#pragma unroll
      for (int k = 0; k <= HD; k++) {
        if (halo) {
          tq[k] = ld_relaxed64(set + k);
          tot[k] = (double)tq[k] * quantum_sh * (k == HD ? 4096.0 : 1.0);
        } else {
          tot[k] = k == HD ? part[k] * fabs(s.e_d) : part[k];
          tq[k] = part[k] != 0;
        }
      }
      // the first half-sweep of the round that meets the stop rule (unrolled
      // selects keep the arrays in registers)
      int ks = -1;
      double tks = 0, tlast = 0;
#pragma unroll
      for (int k = 0; k < HD; k++) {
        if (ks < 0 && k < keff && n0 + k > 0 && (tot[k] < thr_sh || tq[k] == 0)) {
          ks = k;
          tks = tot[k];
        }
        if (k == keff - 1)
          tlast = tot[k];
      }
      stop_sh = ks >= 0;
      rebase_sh = 0;
      if (ks >= 0) {
        nundo_sh = keff - 1 - ks;
        result_sh = n0 + ks;
        total_sh = tks;
      } else {
        total_sh = tlast;
        // Iterative refinement: fold d into Psi and form the residual again
        // in FP64 once the residual has fallen 2^8-fold below the last FP64
        // residual (the base), or to within 2^11 of the FP32 rounding noise
        // of its own terms.  That noise is about 2^-21 |e| sum |d| (each
        // node's residual cancels terms of size |e d| rounded to 2^-24);
        // near it the FP32 residual sums lag the true ones and delay the
        // stop rule (by up to 6 % of the half-sweeps on a 1400 x 200 gun mesh
        // with a trigger 2^3 above the noise; within 2 half-sweeps of the
        // FP64 count at 2^11).  The fixed-point quantum of the residual sums
        // is 2^-30 of the larger of the base and the stop threshold, so the
        // stop test keeps its resolution as the base follows the residual down.
        if (!last && (total_sh < base_sh * (1.0 / 256) || total_sh < tot[HD] * (1.0 / 1024))) {
          rebase_sh = 1;
          base_sh = total_sh;
        }
        quantum_sh = fmax(fmax(base_sh, thr_sh), 1e-280) / 1073741824.0;
      }
    }
    __syncthreads();
    if (stop_sh) {
      for (int u = nundo_sh; u > 0; u--) {
        const int k = keff - 1 - nundo_sh + u; // the latest sweep not yet undone
        const int ext = halo ? HD - 1 - k : 0;
        sweep_rows<true, HD>(m, s, st, D, B, iz_first, nrow, HD - ext, HD + nrow - 1 + ext, k & 1, om_sh[rb][k]);
        __syncthreads();
      }
      break;
    }
    if (rebase_sh) {
      // Psi += d in FP64, then r0 = rhs - A Psi in FP64 once every band has
      // folded its d in, and the sweeps go on from d = 0
      fold_d(s, P, D, iz_first, nrow, HD);
      __syncthreads();
      if (halo) {
        if (tid == 0)
          ok_sh = grid_barrier<0>(s, nullptr, ++gen, cnt);
        __syncthreads();
        if (!ok_sh)
          return;
      }
      double d0 = 0, q0 = 0;
      form_r0(m, s, B, iz_first - (HD - 1), nrow + 2 * (HD - 1), iz_first, iz_last, &d0, &q0);
      for (int t = tid; t < (R + 2 * HD) * 2 * H; t += NT)
        D[t] = 0.f;
      __syncthreads();
      continue;
    }
    if (halo && !last) {
      // halo rows 0..HD-1 from the CTA before, nrow+HD.. from the one after;
      // the exchange rows hold both parities in D's row layout
#pragma unroll
      for (int u = 0; u < PRE; u++) {
        const int nb_ = er[u] < HD ? b - 1 : b + 1;
        if (tid + u * NT < ne && nb_ >= 0 && nb_ < G)
          *reinterpret_cast<float4 *>(D + (er[u] < HD ? er[u] : nrow + er[u]) * 2 * H + 4 * ec[u]) = pre[u];
      }
      for (int t = tid + PRE * NT; t < ne; t += NT) { // wide meshes: the rest directly
        const int r = t / Q2, cc = t - r * Q2;
        const int nb_ = r < HD ? b - 1 : b + 1;
        if (nb_ < 0 || nb_ >= G)
          continue;
        const float4 v = __ldcg(reinterpret_cast<const float4 *>(xi + (size_t)nb_ * 4 * HD * H +
                                                                 (r < HD ? 2 * HD * H : 0)) + (r < HD ? r : r - HD) * Q2 + cc);
        *reinterpret_cast<float4 *>(D + (r < HD ? r : nrow + r) * 2 * H + 4 * cc) = v;
      }
      __syncthreads();
    }
  }
  fold_d(s, P, D, iz_first, nrow, HD);
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

// shared bytes of a band of R rows: d with hd halo rows a side, r0 with hd - 1
size_t sor_smem(int R, int H, int hd)
{
  const size_t row = (size_t)2 * H * 4;
  return (R + 2 * hd) * row + (R + 2 * hd - 2) * row;
}

// threads of a CTA: one per column group (H/4 of them) per row group, with
// as many row groups as fit in SOR_NT threads and as runs of two rows need;
// 0 when a half row has more than SOR_NT column groups
int sor_threads(int R, int H, int hd)
{
  const int Q = H / 4, groups = std::min(SOR_NT / std::max(Q, 1), (R + 2 * hd - 2 + 1) / 2);
  if (Q > SOR_NT || groups < 1)
    return 0;
  return (groups * Q + 31) / 32 * 32;
}

const void *sor_kernel(int hd)
{
  return hd == 4 ? (const void *)k_sor32<4> : (const void *)k_sor32<2>;
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
  // dynamic shared memory a CTA of depth h may use: the opt-in limit less
  // the kernel's own static shared memory
  auto budget_of = [&](int h) -> size_t {
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, sor_kernel(h)) != cudaSuccess)
      return 0;
    return (size_t)max_smem > fa.sharedSizeBytes ? (size_t)max_smem - fa.sharedSizeBytes : 0;
  };
  // One CTA when the mesh fits one SM (no grid barriers); otherwise bands
  // of at least `hd` rows (the halo exchange carries hd rows) over all SMs,
  // with four half-sweeps per barrier where the deeper halo fits, else two
  // (six measured slower on the 3000 x 820 gun: the extra halo rows cost
  // more than the barriers they save).
  int G = 0, hd = 4;
  for (int h : {4, 2})
    if (sor_smem(rows, H, h) <= budget_of(h) && (size_t)rows * 2 * H <= 65536) {
      G = 1;
      hd = h;
      break;
    }
  if (G == 0)
    for (int h : {4, 2}) {
      const size_t budget = budget_of(h);
      int g = std::min(sms, rows / h);
      while (g < rows / h && sor_smem((rows + g - 1) / g, H, h) > budget)
        g++;
      if (g >= 1 && g <= sms && sor_smem((rows + g - 1) / g, H, h) <= budget) {
        G = g;
        hd = h;
        break;
      }
    }
  cudaError_t e = cudaSuccess;
  int occ = 0;
  if (G < 1)
    return (int)cudaErrorInvalidConfiguration; // the mesh does not fit the shared-memory bands
  const int R = (rows + G - 1) / G;
  w->grid = G;
  w->depth = hd;
  w->rows_per = R;
  w->smem = sor_smem(R, H, hd);
  w->threads = sor_threads(R, H, hd);
  if (w->threads < 1)
    return (int)cudaErrorInvalidConfiguration; // a half row wider than one CTA's threads
  // the attribute is process-wide: set it to the kernel's limit (the same
  // value for every instance), not to this instance's band, so that setting
  // up another instance cannot lower it under this one's launch
  e = cudaFuncSetAttribute(sor_kernel(hd), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget_of(hd));
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sor_kernel(hd), w->threads, w->smem);
  if (e == cudaSuccess && occ < 1)
    e = cudaErrorInvalidConfiguration;
  w->half = H;
  const size_t gx = (nr + 1 + BX - 1) / BX, gy = (nz + 1 + BY - 1) / BY;
  size_t parts = std::max<size_t>(3 * gx * gy, 4096);
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
    if (e == cudaSuccess) e = cudaMalloc(&w->bar, sizeof(unsigned long long) * 48); // counter, sum slots
    if (e == cudaSuccess) e = cudaMalloc(&w->dpart, sizeof(double) * (size_t)sms * 2); // |rhs|, |r0| per CTA
    if (e == cudaSuccess) e = cudaMalloc(&w->xbuf, sizeof(float) * (size_t)2 * sms * 16 * H); // exchange rows, 4 a side
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
  s32_mg_free(&w->mg);
  void *p[] = {w->Az, w->Ari, w->Aro, w->volume, w->crow, w->drow, w->scalars, w->qreal_fixed, w->st,
               w->iters, w->bar, w->dpart, w->xbuf, w->part, w->omega};
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
  a.count = w->bar;
  a.slots = w->bar + 16; // another 128-byte line than the polled counter
  a.dpart = w->dpart;
  a.st = st;
  a.iters_out = w->iters;
  a.lo = m->left_bc == SPIFFE_DIRICHLET ? 0 : 1;
  a.hi = m->right_bc == SPIFFE_DIRICHLET ? m->nz - 1 : m->nz - 2;
  a.cols = m->nr - 1;
  a.H = w->half;
  a.rows_per = w->rows_per;
  cudaError_t e = cudaMemsetAsync(w->bar, 0, sizeof(unsigned long long) * 48, s);
  if (e != cudaSuccess)
    return (int)e;
  DevMesh mm = *m;
  void *args[] = {&mm, &a, &cnt};
  e = cudaLaunchCooperativeKernel(sor_kernel(w->depth), dim3(w->grid), dim3(w->threads), args, w->smem, s);
  spiffe_note_launches(1);
  return (int)e;
}

extern "C" int s32_solve(const DevMesh *m, Poisson32Work *w, double *Psi, const double *rhs, const uint8_t *umask,
                         double accuracy, long long limit, PcState *st, DevCounts *cnt, cudaStream_t s)
{
  if (w->solver == SPIFFE_POISSON_MULTIGRID && w->mg.nlev >= 2)
    return s32_mg_solve(m, &w->mg, w->crow, w->drow, Psi, rhs, umask, accuracy, limit, st, w->iters, cnt, s);
  return s32_sor(m, w, Psi, rhs, umask, accuracy, limit, st, cnt, s);
}

extern "C" int s32_poisson_correction(const DevMesh *m, const DevFields32 *f, const DevBeam32 *b, DevCounts *cnt,
                                      long long np_bound, const PoissonHostOptions *o, const S32Scales *sc,
                                      Poisson32Work *w, cudaStream_t s)
{
  const dim3 block(BX, BY), grid((m->nr + 1 + BX - 1) / BX, (m->nz + 1 + BY - 1) / BY);
  const int nblk = grid.x * grid.y;
  const bool sc_on = o->space_charge && np_bound > 0;
  // the particles' charge first (it reads only the beam), then one pass of
  // apparent charge, particle charge, sums and right-hand side
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
  k_charge32<<<grid, block, 0, s>>>(*m, *f, w->Az, w->Ari, w->Aro, w->volume, 0, sc->qQ, sc_on ? 1 : 0, w->part);
  k_charge_state32<<<1, 1024, 0, s>>>(w->part, nblk, w->scalars, w->st, w->qreal_fixed, sc->qQ, o->space_charge,
                                      o->error_charge_threshold);
  spiffe_note_launches(2);
  if (o->guess_code) {
    k_guess32<<<grid, block, 0, s>>>(*m, *f, o->guess_code, w->st);
    spiffe_note_launches(1);
  }
  int rc = s32_solve(m, w, f->Psi, f->Q, f->umask, o->accuracy, o->maximum_iterations, w->st, cnt, s);
  if (rc)
    return rc;
  k_subtract32<<<grid, block, 0, s>>>(*m, *f, w->st);
  // the reference recomputes the apparent charge afterwards (:333-439); the
  // particles have not moved, so their charge per node is the same Qp
  k_charge32<<<grid, block, 0, s>>>(*m, *f, w->Az, w->Ari, w->Aro, w->volume, 1, sc->qQ, sc_on ? 1 : 0, nullptr);
  spiffe_note_launches(2);
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
  rep->driving = st.driving;
  return (int)e;
}

extern "C" int s32_imposed_field(const DevMesh *m, const DevFields32 *f, double factor, cudaStream_t s)
{
  const dim3 block(BX, BY), grid((m->nr + 1 + BX - 1) / BX, (m->nz + 1 + BY - 1) / BY);
  k_imposed32<<<grid, block, 0, s>>>(*m, *f, factor);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}
