// spiffe_b200/csrc/multigrid_f32.cu -- multigrid Poisson solve of the split-precision form.
//
// The problem is solve_poisson_cyl's (poisson.c:17-130): the five-point
// cylindrical operator on the nodes that routine updates (rows lo..hi,
// columns 0..nr-2, not metal; the axis row of coefficients 4c and e - 2c;
// mirrored end rows for a "Dirichlet" end), every other node held.  The
// reference relaxes it with red-black SOR to its stop rule
// sum|residual| < accuracy sum|rhs|; on the meshes of the RF and DC guns
// that rule is out of reach within its 1000 half-sweeps.  Here the same
// equations are solved by FP64 iterative refinement around FP32 multigrid
// V-cycles:
//
//   r = rhs - A Psi in FP64; stop when sum|r| < accuracy * sum|rhs|
//   (sum|rhs| over iz < nz, ir < nr-1, as poisson.c:40-43 forms it; a
//   Laplace solve, rhs absent, measures against its first residual);
//   u = V-cycle(r) in FP32;  Psi += u in FP64;  repeat.
//
// Levels: level 0 is the mesh; level l+1 holds the nodes 2I, 2J of level l
// (node (I, J) of level l+1 is unknown when node (2I, 2J) of level l is).
// Transfers are bilinear interpolation P and its volume-weighted adjoint
// R = (1/4) Vc^-1 P^T Vf (Vf, Vc: annulus volumes, the axis node's 1/8 of
// the first ring's), and the coarse operators are the Galerkin products
// R A P, built once per mesh on the host in FP64 (nine-point stencils).
// Metal irises and electrodes stay in the coarse operators that way;
// operators rediscretised on the coarse nodes instead lose them and the
// V-cycle then reduces the residual only 0.6x per cycle on the 1.6-cell gun
// against 0.1-0.17x with the Galerkin operators.  Smoothing is red-black
// Gauss-Seidel on level 0 and four-colour Gauss-Seidel (colour (I&1, J&1))
// on the nine-point levels, nu sweeps before and after each coarse
// correction; the last pre-smoothing colour leaves a zero residual at its
// own nodes, so the restriction evaluates the residual only at the others.
//
// One cooperative launch runs the whole solve.  Levels with more than
// MG_TAIL_NODES nodes are worked by every CTA with grid barriers between the
// colour sweeps; on the nine-point ones each CTA owns a band of rows, so the
// two colours of one row parity, which depend on each other only within a
// row, need a CTA barrier between them and a grid barrier only before the
// other parity (two grid barriers a sweep, not four, same update order).
// The residual pass also makes level 0's first colour-0 sweep (from u = 0
// it needs no neighbours) and the last post-smoothing sweep adds u to Psi,
// saving two passes and two barriers a cycle.  The smaller levels, down to
// the coarsest (solved exactly by its precomputed inverse when it has at
// most MG_MAX_DIRECT unknowns, else by Gauss-Seidel sweeps), are worked by
// CTA 0 alone with CTA barriers while the others wait at the next grid
// barrier.  Data written inside the launch are read after the acquire of a
// grid barrier.  The sums that drive the stop rule are per-CTA partials
// added in the same order by every CTA, so every CTA takes the same
// decision and the result does not depend on timing.  Every barrier wait is
// bounded; on time-out the kernel raises SPIFFE_DEV_ERR_BARRIER and every
// CTA returns.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <system_error>
#include <thread>
#include <vector>

#include "modules.cuh"
#include "split32.cuh"

namespace {

constexpr int MG_NT = 1024;           // threads per CTA
constexpr int MG_TAIL_NODES = 3000;   // levels at most this large are worked by CTA 0 alone
constexpr int MG_MIN_UNKNOWNS = 64;   // coarsening stops at this many unknowns
constexpr int MG_NODES_PER_CTA = 8192; // mesh nodes per CTA below one CTA per SM
constexpr int MG_MAX_DIRECT = 1024;   // a coarsest level of at most this many unknowns is solved exactly
enum { MG_INVD = 8, MG_DIAG = 9 };

struct Mg32Args {
  double *Psi;
  const double *rhs; // null: Laplace solve
  const uint8_t *umask;
  float *u0, *f0;
  const float *crow, *drow;
  int nz, P0, lo, hi, cols;
  float a, c4, e, e2c, inv_e, inv_e2c;   // level-0 operator in FP32
  double a_d, e_d, c4_d, e2c_d, dr2_inv; // and in FP64 for the residual
  int nlev, tail, nu0, nu, coarse_sweeps, max_cycles;
  const float *cinv; // the coarsest level's inverse, cn x cn row-major (null: coarse sweeps)
  const int *cidx;   // its unknowns' array indices on that level
  int cn;
  double accuracy;
  MgLevel lev[MG_MAX_LEVELS];
  unsigned long long *bar; // [0] arrivals, [16] abort
  double *part;            // [grid][2]
  PcState *st;
  long long *iters_out;
};

__device__ __forceinline__ unsigned long long mg_ld_acquire(const unsigned long long *p)
{
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long mg_ld_relaxed(const unsigned long long *p)
{
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier over a monotonic arrival counter (barrier number gen, counted
// from 1 by every thread alike).  Bounded: after 2^24 polls, or once another
// CTA has given up, it returns false in every thread of the CTA.
__device__ bool mg_grid_sync(const Mg32Args &a, unsigned &gen, DevCounts *cnt)
{
  __shared__ int ok_sh;
  gen++;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(a.bar), "l"(1ull) : "memory");
    const unsigned long long target = (unsigned long long)gridDim.x * gen;
    unsigned long long polls = 0;
    while (mg_ld_acquire(a.bar) < target) {
      if (mg_ld_relaxed(a.bar + 16)) {
        ok = 0;
        break;
      }
      if (++polls > (1ull << 24)) {
        atomicOr(&cnt->error, SPIFFE_DEV_ERR_BARRIER);
        asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(a.bar + 16), "l"(1ull) : "memory");
        ok = 0;
        break;
      }
      if (polls > 32)
        __nanosleep(32);
    }
    ok_sh = ok;
  }
  __syncthreads();
  return ok_sh != 0;
}

// ---- level 0: the mesh, five-point operator

__device__ __forceinline__ bool unknown0(const Mg32Args &a, int iz, int ir, size_t j)
{
  return iz >= a.lo && iz <= a.hi && ir < a.cols && !(a.umask[j] & S32_U_METAL);
}

// neighbour sum of the level-0 operator at an unknown node (poisson.c:57-117)
__device__ __forceinline__ float nb0(const Mg32Args &a, const float *u, int iz, int ir, size_t j)
{
  const long P = a.P0;
  const float up = (iz == a.nz - 1 && a.hi == a.nz - 1) ? *(u + j - P) : *(u + j + P);
  const float dn = (iz == 0 && a.lo == 0) ? *(u + j + P) : *(u + j - P);
  if (ir == 0)
    return a.a * (up + dn) + a.c4 * *(u + j + 1);
  return a.a * (up + dn) + __ldg(a.crow + ir) * *(u + j + 1) + __ldg(a.drow + ir) * *(u + j - 1);
}

__device__ __forceinline__ float res0(const Mg32Args &a, int iz, int ir)
{
  const size_t j = node(iz, ir, a.P0);
  if (!unknown0(a, iz, ir, j))
    return 0.f;
  return *(a.f0 + j) - nb0(a, a.u0, iz, ir, j) - (ir ? a.e : a.e2c) * *(a.u0 + j);
}

// Four consecutive columns c0 .. c0+3 of a level-0 row: what a colour
// sweep reads: 16-byte loads of u on the row and its two neighbours, of f
// and of the mask; the scalars left and right of the group.
struct Cols0 {
  float4 um, dm, u, f;
  uchar4 mk;
  float left, right;
  int j, iz, c0; // j: array index (level 0 has fewer than 2^31 nodes)
};

__device__ __forceinline__ void cols0_load(const Mg32Args &a, long t, int G, Cols0 &k)
{
  const long P = a.P0;
  const int row = (int)(t / G), g = (int)(t - (long)row * G);
  k.iz = a.lo + row;
  k.c0 = 4 * g;
  k.j = (int)node(k.iz, k.c0, a.P0);
  const bool top = k.iz == a.nz - 1 && a.hi == a.nz - 1, bottom = k.iz == 0 && a.lo == 0;
  k.um = *reinterpret_cast<const float4 *>(a.u0 + (top ? k.j - P : k.j + P));
  k.dm = *reinterpret_cast<const float4 *>(a.u0 + (bottom ? k.j + P : k.j - P));
  k.u = *reinterpret_cast<const float4 *>(a.u0 + k.j);
  k.f = *reinterpret_cast<const float4 *>(a.f0 + k.j);
  k.mk = *reinterpret_cast<const uchar4 *>(a.umask + k.j);
  k.left = k.c0 > 0 ? a.u0[k.j - 1] : 0.f;
  k.right = a.u0[k.j + 4];
}

// New values of the group's nodes of colour c ((iz+ir)%2 == c); fin keeps
// the others' values.  Bit q of the result: node c0+q is an unknown.
// Every index into the small arrays is a compile-time constant, so they
// live in registers.
__device__ __forceinline__ unsigned cols0_relax(const Mg32Args &a, int c, const Cols0 &k, float fin[4])
{
  const float uu[6] = {k.left, k.u.x, k.u.y, k.u.z, k.u.w, k.right};
  const float ups[4] = {k.um.x, k.um.y, k.um.z, k.um.w}, dns[4] = {k.dm.x, k.dm.y, k.dm.z, k.dm.w};
  const float fs[4] = {k.f.x, k.f.y, k.f.z, k.f.w};
  const uint8_t ms[4] = {k.mk.x, k.mk.y, k.mk.z, k.mk.w};
  fin[0] = k.u.x;
  fin[1] = k.u.y;
  fin[2] = k.u.z;
  fin[3] = k.u.w;
  unsigned unk = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int ir = k.c0 + q;
    if (ir >= a.cols || (ms[q] & S32_U_METAL))
      continue;
    unk |= 1u << q;
    if (((k.iz + ir) & 1) != c)
      continue;
    float nb;
    if (ir == 0)
      nb = a.a * (ups[q] + dns[q]) + a.c4 * uu[q + 2];
    else
      nb = a.a * (ups[q] + dns[q]) + __ldg(a.crow + ir) * uu[q + 2] + __ldg(a.drow + ir) * uu[q];
    fin[q] = (fs[q] - nb) * (ir ? a.inv_e : a.inv_e2c);
  }
  return unk;
}

// One colour c of red-black Gauss-Seidel on level 0: nodes with (iz+ir)%2 ==
// c, a group of four columns per task; the group's other two nodes, which
// this colour's updates only read, are left as they are.  With FOLD (the
// V-cycle's last sweep) the thread also adds the group's four final values
// to Psi in FP64: the other colour's are final before this sweep and its own
// after it.
template <bool FOLD>
__device__ void smooth0(const Mg32Args &a, int c, long t0, long dt)
{
  const int G = (a.cols + 3) >> 2; // column groups per row
  const long n = (long)(a.hi - a.lo + 1) * G;
  for (long t = t0; t < n; t += dt) {
    Cols0 k;
    cols0_load(a, t, G, k);
    float fin[4];
    const unsigned unk = cols0_relax(a, c, k, fin);
#pragma unroll
    for (int q = 0; q < 4; q++)
      if ((unk >> q & 1) && ((k.iz + k.c0 + q) & 1) == c)
        a.u0[k.j + q] = fin[q];
    if (FOLD)
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (unk >> q & 1)
          a.Psi[k.j + q] = a.Psi[k.j + q] + (double)fin[q];
  }
}

// ---- levels >= 1: nine-point Galerkin operators

__device__ __forceinline__ float nb9(const MgLevel &L, size_t idx, size_t plane)
{
  const float *u = L.u, *c = L.coef;
  const long P = L.P;
  float s = __ldg(c + idx) * *(u + idx - P - 1);
  s += __ldg(c + plane + idx) * *(u + idx - P);
  s += __ldg(c + 2 * plane + idx) * *(u + idx - P + 1);
  s += __ldg(c + 3 * plane + idx) * *(u + idx - 1);
  s += __ldg(c + 4 * plane + idx) * *(u + idx + 1);
  s += __ldg(c + 5 * plane + idx) * *(u + idx + P - 1);
  s += __ldg(c + 6 * plane + idx) * *(u + idx + P);
  s += __ldg(c + 7 * plane + idx) * *(u + idx + P + 1);
  return s;
}

__device__ __forceinline__ float res9(const MgLevel &L, int I, int J)
{
  const size_t plane = (size_t)(L.Z + 2) * L.P, idx = (size_t)(I + 1) * L.P + J + 1;
  if (__ldg(L.coef + MG_INVD * plane + idx) == 0.f)
    return 0.f;
  return *(L.f + idx) - __ldg(L.coef + MG_DIAG * plane + idx) * (*(L.u + idx) + nb9(L, idx, plane));
}

// one colour (cz, cr) = (c >> 1, c & 1) of Gauss-Seidel on a nine-point level
__device__ void smooth9(const MgLevel &L, int c, long t0, long dt)
{
  const int cz = c >> 1, cr = c & 1;
  const int Zh = (L.Z - cz + 1) >> 1, Rh = (L.R - cr + 1) >> 1;
  const long n = (long)Zh * Rh;
  const size_t plane = (size_t)(L.Z + 2) * L.P;
  for (long t = t0; t < n; t += dt) {
    const int q = (int)(t / Rh);
    const int I = 2 * q + cz, J = 2 * (int)(t - (long)q * Rh) + cr;
    const size_t idx = (size_t)(I + 1) * L.P + J + 1;
    const float id = __ldg(L.coef + MG_INVD * plane + idx);
    if (id == 0.f)
      continue;
    L.u[idx] = *(L.f + idx) * id - nb9(L, idx, plane);
  }
}

// Two colours (cz, cr) then (cz, 1-cr) of Gauss-Seidel on a nine-point level
// over this CTA's rows (a band of ceil(Z / grid) rows).  A node of colour
// (cz, 1-cr) reads the just-updated colour (cz, cr) only at its left and
// right neighbours, in its own row, so a CTA barrier between the two
// colours suffices; the colours of the other row parity read rows I +- 1
// and follow a grid barrier.  The update order, and so every value, is the
// four-colour sweep's.
__device__ void smooth9_rows(const MgLevel &L, int cz, int cr)
{
  const int nbl = (L.Z + (int)gridDim.x - 1) / (int)gridDim.x;
  const int I0 = (int)blockIdx.x * nbl, I1 = min(I0 + nbl, L.Z);
  const int r0 = I0 + ((I0 & 1) != cz); // first own row of parity cz
  const int nrows = r0 < I1 ? (I1 - r0 + 1) >> 1 : 0;
  const size_t plane = (size_t)(L.Z + 2) * L.P;
  for (int h = 0; h < 2; h++) {
    const int c = h ? 1 - cr : cr;
    const int Rh = (L.R - c + 1) >> 1;
    const long n = (long)nrows * Rh;
    for (long t = threadIdx.x; t < n; t += blockDim.x) {
      const int q = (int)(t / Rh);
      const int I = r0 + 2 * q, J = 2 * (int)(t - (long)q * Rh) + c;
      const size_t idx = (size_t)(I + 1) * L.P + J + 1;
      const float id = __ldg(L.coef + MG_INVD * plane + idx);
      if (id == 0.f)
        continue;
      L.u[idx] = *(L.f + idx) * id - nb9(L, idx, plane);
    }
    __syncthreads();
  }
}

// f of level C from the residual of level 0 (C = lev[1]), u of C cleared.
// Level 0's last colour (1) has a zero residual: only (iz+ir) even nodes.
__device__ void restrict0(const Mg32Args &a, long t0, long dt)
{
  const MgLevel &C = a.lev[1];
  const long n = (long)C.Z * C.R;
  const size_t plane = (size_t)(C.Z + 2) * C.P;
  for (long t = t0; t < n; t += dt) {
    const int I = (int)(t / C.R), J = (int)(t - (long)I * C.R);
    const size_t idx = (size_t)(I + 1) * C.P + J + 1;
    float s = 0.f;
    if (__ldg(C.coef + MG_INVD * plane + idx) != 0.f && (C.cz != 2 || C.cr != 2)) {
      // semi-coarsened: the three fine nodes along the coarsened direction
      const float w[3] = {__ldg(C.rw + 3 * J), __ldg(C.rw + 3 * J + 1), __ldg(C.rw + 3 * J + 2)};
      const int iz = C.cz * I, ir = C.cr * J;
#pragma unroll
      for (int d = -1; d <= 1; d++) {
        const int z = C.cz == 2 ? iz + d : iz, r = C.cr == 2 ? ir + d : ir;
        if (z < 0 || z > a.nz || r < 0)
          continue;
        s += (C.cz == 2 ? (d ? 0.5f : 1.f) * w[1] : w[d + 1]) * res0(a, z, r);
      }
    } else if (__ldg(C.coef + MG_INVD * plane + idx) != 0.f) {
      const float w0 = __ldg(C.rw + 3 * J), w1 = __ldg(C.rw + 3 * J + 1), w2 = __ldg(C.rw + 3 * J + 2);
      const int iz = 2 * I, ir = 2 * J;
      s = w1 * res0(a, iz, ir);
      if (iz > 0) {
        if (ir > 0)
          s += 0.5f * w0 * res0(a, iz - 1, ir - 1);
        s += 0.5f * w2 * res0(a, iz - 1, ir + 1);
      }
      if (iz < a.nz) {
        if (ir > 0)
          s += 0.5f * w0 * res0(a, iz + 1, ir - 1);
        s += 0.5f * w2 * res0(a, iz + 1, ir + 1);
      }
    }
    C.f[idx] = s;
    C.u[idx] = 0.f;
  }
}

// f of level C = lev[l+1] from the residual of F = lev[l], u of C cleared.
// F's last colour (3: odd, odd) has a zero residual: its four diagonal
// neighbours of (2I, 2J) are skipped.
__device__ void restrict9(const MgLevel &F, const MgLevel &C, long t0, long dt)
{
  const long n = (long)C.Z * C.R;
  const size_t plane = (size_t)(C.Z + 2) * C.P;
  for (long t = t0; t < n; t += dt) {
    const int I = (int)(t / C.R), J = (int)(t - (long)I * C.R);
    const size_t idx = (size_t)(I + 1) * C.P + J + 1;
    float s = 0.f;
    if (__ldg(C.coef + MG_INVD * plane + idx) != 0.f && (C.cz != 2 || C.cr != 2)) {
      // semi-coarsened: the three fine nodes along the coarsened direction
      const float w[3] = {__ldg(C.rw + 3 * J), __ldg(C.rw + 3 * J + 1), __ldg(C.rw + 3 * J + 2)};
      const int i = C.cz * I, j = C.cr * J;
#pragma unroll
      for (int d = -1; d <= 1; d++) {
        const int z = C.cz == 2 ? i + d : i, r = C.cr == 2 ? j + d : j;
        if (z < 0 || z >= F.Z || r < 0 || r >= F.R)
          continue;
        s += (C.cz == 2 ? (d ? 0.5f : 1.f) * w[1] : w[d + 1]) * res9(F, z, r);
      }
    } else if (__ldg(C.coef + MG_INVD * plane + idx) != 0.f) {
      const float w0 = __ldg(C.rw + 3 * J), w1 = __ldg(C.rw + 3 * J + 1), w2 = __ldg(C.rw + 3 * J + 2);
      const int i = 2 * I, j = 2 * J;
      s = w1 * res9(F, i, j);
      if (j > 0)
        s += w0 * res9(F, i, j - 1);
      if (j + 1 < F.R)
        s += w2 * res9(F, i, j + 1);
      if (i > 0)
        s += 0.5f * w1 * res9(F, i - 1, j);
      if (i + 1 < F.Z)
        s += 0.5f * w1 * res9(F, i + 1, j);
    }
    C.f[idx] = s;
    C.u[idx] = 0.f;
  }
}

// bilinear correction from level C at node (i, j) of the level above
// (linear along a direction C does not coarsen: the node itself)
__device__ __forceinline__ float interp(const MgLevel &C, int i, int j)
{
  const bool hz = C.cz == 2 && (i & 1), hr = C.cr == 2 && (j & 1); // half-way nodes
  const int I = C.cz == 2 ? i >> 1 : i, J = C.cr == 2 ? j >> 1 : j;
  const float *u = C.u + (size_t)(I + 1) * C.P + J + 1;
  float v;
  if (hr)
    v = 0.5f * (*(u) + *(u + 1));
  else
    v = *(u);
  if (hz) {
    const float *w = u + C.P;
    v = 0.5f * v + 0.5f * (hr ? 0.5f * (*(w) + *(w + 1)) : *(w));
  }
  return v;
}

__device__ void prolong0(const Mg32Args &a, long t0, long dt)
{
  const MgLevel &C = a.lev[1];
  const long n = (long)(a.hi - a.lo + 1) * a.cols;
  for (long t = t0; t < n; t += dt) {
    const int row = (int)(t / a.cols), ir = (int)(t - (long)row * a.cols), iz = a.lo + row;
    const size_t j = node(iz, ir, a.P0);
    if (a.umask[j] & S32_U_METAL)
      continue;
    a.u0[j] = *(a.u0 + j) + interp(C, iz, ir);
  }
}

__device__ void prolong9(const MgLevel &F, const MgLevel &C, long t0, long dt)
{
  const long n = (long)F.Z * F.R;
  const size_t plane = (size_t)(F.Z + 2) * F.P;
  for (long t = t0; t < n; t += dt) {
    const int i = (int)(t / F.R), j = (int)(t - (long)i * F.R);
    const size_t idx = (size_t)(i + 1) * F.P + j + 1;
    if (__ldg(F.coef + MG_INVD * plane + idx) == 0.f)
      continue;
    F.u[idx] = *(F.u + idx) + interp(C, i, j);
  }
}

__shared__ float mg_coarse_f[MG_MAX_DIRECT]; // the coarsest level's f, gathered for its exact solve

// Levels l0 .. nlev-1 below a restriction into l0, by CTA 0 alone with CTA
// barriers: descent, the coarsest level's solve, ascent back to l0.
__device__ void sub_cycle(const Mg32Args &a, int l0)
{
  const MgLevel *lv = a.lev;
  const long t0 = threadIdx.x, dt = blockDim.x;
  const int L = a.nlev;
  for (int l = l0; l < L - 1; l++) {
    for (int k = 0; k < a.nu; k++)
      for (int c = 0; c < 4; c++) {
        smooth9(lv[l], c, t0, dt);
        __syncthreads();
      }
    restrict9(lv[l], lv[l + 1], t0, dt);
    __syncthreads();
  }
  if (a.cinv) {
    // the coarsest level solved exactly: u = A^-1 f over its unknowns
    float *fc = mg_coarse_f;
    const MgLevel &C = lv[L - 1];
    for (int i = (int)t0; i < a.cn; i += (int)dt)
      fc[i] = C.f[a.cidx[i]];
    __syncthreads();
    // a warp per row: coalesced reads of the row, the lanes' partial sums
    // added by shuffles
    const int lane = (int)t0 & 31, warp = (int)t0 >> 5, nwarps = (int)dt >> 5;
    for (int i = warp; i < a.cn; i += nwarps) {
      const float *row = a.cinv + (size_t)i * a.cn;
      float acc = 0.f;
      for (int k = lane; k < a.cn; k += 32)
        acc += __ldg(row + k) * fc[k];
      for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_down_sync(0xffffffffu, acc, o);
      if (lane == 0)
        C.u[a.cidx[i]] = acc;
    }
    __syncthreads();
  } else {
    for (int k = 0; k < a.coarse_sweeps; k++)
      for (int c = 0; c < 4; c++) {
        smooth9(lv[L - 1], c, t0, dt);
        __syncthreads();
      }
  }
  for (int l = L - 2; l >= l0; l--) {
    prolong9(lv[l], lv[l + 1], t0, dt);
    __syncthreads();
    for (int k = 0; k < a.nu; k++)
      for (int c = 3; c >= 0; c--) {
        smooth9(lv[l], c, t0, dt);
        __syncthreads();
      }
  }
}

// One V-cycle on (u0, f0), u0 = 0 on entry.
__device__ bool vcycle(const Mg32Args &a, unsigned &gen, DevCounts *cnt)
{
  const long gt0 = (long)blockIdx.x * blockDim.x + threadIdx.x, gdt = (long)gridDim.x * blockDim.x;
  const int T = a.tail; // 1 <= T <= nlev - 1
  // the first colour-0 sweep from u0 = 0 was made by residual64
  for (int k = 0; k < a.nu0; k++)
    for (int c = k ? 0 : 1; c < 2; c++) {
      smooth0<false>(a, c, gt0, gdt);
      if (!mg_grid_sync(a, gen, cnt))
        return false;
    }
  restrict0(a, gt0, gdt);
  if (!mg_grid_sync(a, gen, cnt))
    return false;
  // grid-wide nine-point levels 1 .. T-1
  for (int l = 1; l < T; l++) {
    for (int k = 0; k < a.nu; k++)
      for (int cz = 0; cz < 2; cz++) { // colours (cz, 0), (cz, 1)
        smooth9_rows(a.lev[l], cz, 0);
        if (!mg_grid_sync(a, gen, cnt))
          return false;
      }
    restrict9(a.lev[l], a.lev[l + 1], gt0, gdt);
    if (!mg_grid_sync(a, gen, cnt))
      return false;
  }
  // levels T .. nlev-1 by CTA 0 while the others wait
  if (blockIdx.x == 0)
    sub_cycle(a, T);
  if (!mg_grid_sync(a, gen, cnt))
    return false;
  for (int l = T - 1; l >= 1; l--) {
    prolong9(a.lev[l], a.lev[l + 1], gt0, gdt);
    if (!mg_grid_sync(a, gen, cnt))
      return false;
    for (int k = 0; k < a.nu; k++)
      for (int cz = 1; cz >= 0; cz--) { // colours (cz, 1), (cz, 0)
        smooth9_rows(a.lev[l], cz, 1);
        if (!mg_grid_sync(a, gen, cnt))
          return false;
      }
  }
  prolong0(a, gt0, gdt);
  if (!mg_grid_sync(a, gen, cnt))
    return false;
  for (int k = 0; k < a.nu0; k++)
    for (int c = 1; c >= 0; c--) {
      if (k == a.nu0 - 1 && c == 0)
        smooth0<true>(a, c, gt0, gdt); // Psi += u0 on the way
      else
        smooth0<false>(a, c, gt0, gdt);
      if (!mg_grid_sync(a, gen, cnt))
        return false;
    }
  return true;
}

// r = rhs - A Psi in FP64 over the unknown nodes into f0 (rounded), and u0
// as the first colour-0 Gauss-Seidel sweep from u0 = 0 leaves it: f0 / e at
// (iz+ir) even nodes (their neighbour sum is zero), 0 at the others; this
// thread's sum |r| and, with first, sum |rhs| over iz < nz, ir < nr-1.
__device__ void residual64(const Mg32Args &a, bool first, double *rs, double *ds)
{
  const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x, dt = (long)gridDim.x * blockDim.x;
  const long n = (long)a.nz * a.cols, P = a.P0;
  double r_acc = 0, d_acc = 0;
  for (long t = t0; t < n; t += dt) {
    const int iz = (int)(t / a.cols), ir = (int)(t - (long)iz * a.cols);
    const size_t j = node(iz, ir, a.P0);
    const double rh = a.rhs ? a.rhs[j] : 0.0;
    if (first)
      d_acc += fabs(rh);
    if (!unknown0(a, iz, ir, j))
      continue;
    const double up = (iz == a.nz - 1 && a.hi == a.nz - 1) ? *(a.Psi + j - P) : *(a.Psi + j + P);
    const double dn = (iz == 0 && a.lo == 0) ? *(a.Psi + j + P) : *(a.Psi + j - P);
    const double psi = *(a.Psi + j);
    double ap;
    if (ir == 0)
      ap = a.a_d * (up + dn) + a.c4_d * *(a.Psi + j + 1) + a.e2c_d * psi;
    else {
      const double h = 0.5 / ir;
      ap = a.a_d * (up + dn) + a.dr2_inv * (1 + h) * *(a.Psi + j + 1) +
           a.dr2_inv * (1 - h) * *(a.Psi + j - 1) + a.e_d * psi;
    }
    const double r = rh - ap;
    r_acc += fabs(r);
    const float rf = (float)r;
    a.f0[j] = rf;
    a.u0[j] = (a.nu0 && !((iz + ir) & 1)) ? rf * (ir ? a.inv_e : a.inv_e2c) : 0.f;
  }
  *rs = r_acc;
  *ds = d_acc;
}

__device__ void fold(const Mg32Args &a)
{
  const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x, dt = (long)gridDim.x * blockDim.x;
  const long n = (long)a.nz * a.cols;
  for (long t = t0; t < n; t += dt) {
    const int iz = (int)(t / a.cols), ir = (int)(t - (long)iz * a.cols);
    const size_t j = node(iz, ir, a.P0);
    if (unknown0(a, iz, ir, j))
      a.Psi[j] = *(a.Psi + j) + (double)*(a.u0 + j);
  }
}

// CTA sums of two doubles into part[blockIdx][0..1] (fixed order)
__device__ void block_sums(const Mg32Args &a, double x, double y)
{
  __shared__ double sh[2][MG_NT / 32];
  for (int o = 16; o > 0; o >>= 1) {
    x += __shfl_down_sync(0xffffffffu, x, o);
    y += __shfl_down_sync(0xffffffffu, y, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sh[0][w] = x;
    sh[1][w] = y;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sx = 0, sy = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
      sx += sh[0][k];
      sy += sh[1][k];
    }
    a.part[2 * blockIdx.x] = sx;
    a.part[2 * blockIdx.x + 1] = sy;
  }
}

// the grid's totals, formed in the same order by every CTA
__device__ void grid_totals(const Mg32Args &a, double *tx, double *ty)
{
  __shared__ double tot[2];
  if (threadIdx.x < 32) {
    double x = 0, y = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += 32) {
      x += __ldcg(a.part + 2 * k);
      y += __ldcg(a.part + 2 * k + 1);
    }
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_down_sync(0xffffffffu, x, o);
      y += __shfl_down_sync(0xffffffffu, y, o);
    }
    if (threadIdx.x == 0) {
      tot[0] = x;
      tot[1] = y;
    }
  }
  __syncthreads();
  *tx = tot[0];
  *ty = tot[1];
}

__global__ void __launch_bounds__(MG_NT) k_mg32(Mg32Args a, DevCounts *cnt)
{
  if (a.st && !a.st->do_solve)
    return;
  unsigned gen = 0;
  double drive = 0, total = 0;
  long long cycles = 0;
  bool conv = false;
  for (;;) {
    const bool first = cycles == 0;
    double rs, ds;
    residual64(a, first, &rs, &ds);
    block_sums(a, rs, ds);
    if (!mg_grid_sync(a, gen, cnt))
      return;
    double dsum;
    grid_totals(a, &total, &dsum);
    if (first)
      drive = a.rhs ? dsum : total; // poisson.c:40-43; a Laplace solve: its first residual
    if (total == 0 || total < a.accuracy * drive) {
      conv = true;
      break;
    }
    if (cycles >= a.max_cycles)
      break;
    // (the partials are rewritten only after the V-cycle's first barrier,
    // which every CTA reaches after reading them)
    if (!vcycle(a, gen, cnt))
      return;
    if (a.nu0 == 0) { // no sweep to fold into
      fold(a);
      if (!mg_grid_sync(a, gen, cnt))
        return;
    }
    cycles++;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const long long result = conv ? cycles : -1;
    if (a.iters_out)
      *a.iters_out = result;
    if (a.st) {
      a.st->iterations = result;
      a.st->residual = total;
      a.st->driving = drive;
    }
    cnt->mg_cycles += cycles;
    cnt->sor_solves += 1;
  }
}

// ---- host: the level hierarchy

// fn(lo, hi) over [0, n) in contiguous chunks on up to 16 host threads (the
// hierarchy of a 2.5M-node mesh takes over half a second on one core)
template <class Fn>
void parallel_rows(int n, Fn fn)
{
  const int nt = std::max(1, std::min({16, (int)std::thread::hardware_concurrency(), n / 8}));
  if (nt <= 1) {
    fn(0, n);
    return;
  }
  std::vector<std::thread> pool;
  const int chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; t++) {
    const int lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi)
      continue;
    try {
      pool.emplace_back(fn, lo, hi);
    } catch (const std::system_error &) {
      fn(lo, hi); // no thread to be had: this chunk on the caller's thread
    }
  }
  for (std::thread &th : pool)
    th.join();
}

// level-0 operator as nine-point rows (only the five-point entries are
// nonzero): coefficient of node (iz+dz, ir+dr) at k = (dz+1)*3 + (dr+1)
struct Stencil {
  int Z = 0, R = 0;
  std::vector<double> c; // [9][Z*R]
  std::vector<uint8_t> unk;
  double &at(int k, int i, int j) { return c[(size_t)k * Z * R + (size_t)i * R + j]; }
  double at(int k, int i, int j) const { return c[(size_t)k * Z * R + (size_t)i * R + j]; }
};

void fine_stencil(const DevMesh &m, const int16_t *flags, int lo, int hi, Stencil &S)
{
  const int nz = m.nz, nr = m.nr, cols = nr - 1;
  S.Z = nz + 1;
  S.R = nr + 1;
  S.c.assign((size_t)9 * S.Z * S.R, 0.0);
  S.unk.assign((size_t)S.Z * S.R, 0);
  for (int iz = lo; iz <= hi; iz++)
    for (int ir = 0; ir < cols; ir++)
      if (!(flags[(size_t)iz * (nr + 1) + ir] & (SPIFFE_FL_IS_SURFACE | SPIFFE_FL_IS_INSIDE)))
        S.unk[(size_t)iz * S.R + ir] = 1;
  const double a = 1 / (m.dz * m.dz), dr2 = m.dr * m.dr;
  const double e = -2 * (1 / (m.dz * m.dz) + 1 / dr2);
  // each node writes only its own stencil row
  parallel_rows(hi - lo + 1, [&](int r0, int r1) {
  for (int iz = lo + r0; iz < lo + r1; iz++)
    for (int ir = 0; ir < cols; ir++) {
      if (!S.unk[(size_t)iz * S.R + ir])
        continue;
      double cu = a, cd = a;
      int zu = iz + 1, zd = iz - 1;
      if (iz == 0 && lo == 0) { // mirrored end rows (poisson.c:67-84, :102-118)
        zd = iz + 1;
      } else if (iz == nz - 1 && hi == nz - 1) {
        zu = iz - 1;
      }
      double cr, cl, dg;
      if (ir == 0) {
        cr = 4 / dr2;
        cl = 0;
        dg = e - 2 / dr2;
      } else {
        cr = 1 / dr2 * (1 + 1. / (2 * ir));
        cl = 1 / dr2 * (1 - 1. / (2 * ir));
        dg = e;
      }
      auto add = [&](int z2, int r2, double v) {
        if (v == 0 || z2 < 0 || z2 >= S.Z || r2 < 0 || r2 >= S.R || !S.unk[(size_t)z2 * S.R + r2])
          return;
        S.at((z2 - iz + 1) * 3 + (r2 - ir + 1), iz, ir) += v;
      };
      add(zu, ir, cu);
      add(zd, ir, cd);
      add(iz, ir + 1, cr);
      add(iz, ir - 1, cl);
      S.at(4, iz, ir) = dg;
    }
  });
}

// annulus weight of column j of a level of spacing 1 (the axis node: 1/8)
inline double vol(int j) { return j ? (double)j : 0.125; }

// Galerkin R A P from level F to C (nodes cz I, cr J of F: cz, cr = 2 to
// coarsen a direction, 1 to keep it); restriction weights rw[J][3] for F
// columns cr J - 1, cr J, cr J + 1 (with cz = 2 the z weights 1/2, 1, 1/2
// apply on top)
void galerkin(const Stencil &F, Stencil &C, std::vector<double> &rw, int cz, int cr)
{
  C.Z = cz == 2 ? (F.Z + 1) / 2 : F.Z;
  C.R = cr == 2 ? (F.R + 1) / 2 : F.R;
  C.c.assign((size_t)9 * C.Z * C.R, 0.0);
  C.unk.assign((size_t)C.Z * C.R, 0);
  for (int I = 0; I < C.Z; I++)
    for (int J = 0; J < C.R; J++)
      C.unk[(size_t)I * C.R + J] = F.unk[(size_t)(cz * I) * F.R + cr * J];
  rw.assign((size_t)3 * C.R, 0.0);
  for (int J = 0; J < C.R; J++)
    for (int dj = -1; dj <= 1; dj++) {
      const int j = cr * J + dj;
      if (j < 0 || j >= F.R || (cr == 1 && dj))
        continue;
      // in fine units: coarse spacing 2, Vc(J) = 2 vc with vc = 2J (axis:
      // 1/4); coarse spacing 1, Vc(J) = vol(J) = 2 vc
      const double vc = cr == 2 ? (J ? 2.0 * J : 0.25) : 0.5 * vol(J);
      rw[(size_t)3 * J + dj + 1] = (dj ? 0.5 : 1.0) * vol(j) / (4 * vc);
    }
  auto cunk = [&](int I, int J) { return I >= 0 && I < C.Z && J >= 0 && J < C.R && C.unk[(size_t)I * C.R + J]; };
  // coarse rows in parallel: each node writes only its own stencil and flag,
  // and reads the neighbours' flags as they were before any hold below (a
  // coupling to a node held here is removed by the pass after, so the
  // stencils do not depend on the order the rows are done in)
  const std::vector<uint8_t> unk0 = C.unk;
  auto cunk0 = [&](int I, int J) { return I >= 0 && I < C.Z && J >= 0 && J < C.R && unk0[(size_t)I * C.R + J]; };
  parallel_rows(C.Z, [&](int I0, int I1) {
  for (int I = I0; I < I1; I++)
    for (int J = 0; J < C.R; J++) {
      if (!C.unk[(size_t)I * C.R + J])
        continue;
      double acc[9] = {0};
      const int dz0 = cz == 2 ? -1 : 0, dr0 = cr == 2 ? -1 : 0;
      for (int di = dz0; di <= -dz0; di++)
        for (int dj = dr0; dj <= -dr0; dj++) {
          const int i = cz * I + di, j = cr * J + dj;
          if (i < 0 || i >= F.Z || j < 0 || j >= F.R || !F.unk[(size_t)i * F.R + j])
            continue;
          const double r = (di ? 0.5 : 1.0) * rw[(size_t)3 * J + dj + 1];
          for (int k = 0; k < 9; k++) {
            const double v = F.at(k, i, j);
            if (v == 0)
              continue;
            const int ni = i + k / 3 - 1, nj = j + k % 3 - 1; // an unknown fine node
            // its coarse parents (bilinear interpolation; along a direction
            // kept, the node itself)
            const bool hz = cz == 2 && (ni & 1), hr = cr == 2 && (nj & 1);
            const int pz0 = cz == 2 ? ni >> 1 : ni, pr0 = cr == 2 ? nj >> 1 : nj;
            const int nzp = hz ? 2 : 1, nrp = hr ? 2 : 1;
            const double wz = hz ? 0.5 : 1.0, wr = hr ? 0.5 : 1.0;
            for (int pz = 0; pz < nzp; pz++)
              for (int pr = 0; pr < nrp; pr++) {
                const int K = pz0 + pz, Lc = pr0 + pr;
                if (!cunk0(K, Lc))
                  continue;
                acc[(K - I + 1) * 3 + (Lc - J + 1)] += r * v * wz * wr;
              }
          }
        }
      for (int k = 0; k < 9; k++)
        C.at(k, I, J) = acc[k];
      if (!(acc[4] < 0)) { // not a proper diagonal: hold the node
        C.unk[(size_t)I * C.R + J] = 0;
        for (int k = 0; k < 9; k++)
          C.at(k, I, J) = 0;
      }
    }
  });
  // couplings to nodes that were held above (after every row's hold)
  parallel_rows(C.Z, [&](int I0, int I1) {
    for (int I = I0; I < I1; I++)
      for (int J = 0; J < C.R; J++)
        for (int k = 0; k < 9; k++)
          if (C.at(k, I, J) != 0 && !cunk(I + k / 3 - 1, J + k % 3 - 1))
            C.at(k, I, J) = 0;
  });
}

size_t unknowns(const Stencil &S)
{
  size_t n = 0;
  for (uint8_t u : S.unk)
    n += u;
  return n;
}

} // namespace

extern "C" void s32_mg_free(Mg32Work *w)
{
  cudaFree(w->mem);
  cudaFree(w->cinv);
  cudaFree(w->cidx);
  *w = Mg32Work();
}

namespace {
// The inverse of the coarsest level's operator over its unknowns (Gauss-Jordan
// with partial pivoting in FP64), for the exact coarse solve; false when the
// level has more than MG_MAX_DIRECT unknowns or the matrix is singular.
bool coarse_inverse(const Stencil &S, int P, std::vector<float> &inv, std::vector<int> &idx)
{
  std::vector<int> num((size_t)S.Z * S.R, -1);
  idx.clear();
  for (int I = 0; I < S.Z; I++)
    for (int J = 0; J < S.R; J++)
      if (S.unk[(size_t)I * S.R + J]) {
        num[(size_t)I * S.R + J] = (int)idx.size();
        idx.push_back((I + 1) * P + J + 1);
      }
  const int n = (int)idx.size();
  if (n == 0 || n > MG_MAX_DIRECT)
    return false;
  std::vector<double> A((size_t)n * n, 0.0), X((size_t)n * n, 0.0);
  for (int I = 0; I < S.Z; I++)
    for (int J = 0; J < S.R; J++) {
      const int r = num[(size_t)I * S.R + J];
      if (r < 0)
        continue;
      for (int k = 0; k < 9; k++) {
        const int i2 = I + k / 3 - 1, j2 = J + k % 3 - 1;
        if (i2 < 0 || i2 >= S.Z || j2 < 0 || j2 >= S.R)
          continue;
        const int c = num[(size_t)i2 * S.R + j2];
        if (c >= 0)
          A[(size_t)r * n + c] += S.at(k, I, J);
      }
    }
  for (int i = 0; i < n; i++)
    X[(size_t)i * n + i] = 1.0;
  for (int col = 0; col < n; col++) {
    int piv = col;
    for (int r = col + 1; r < n; r++)
      if (std::fabs(A[(size_t)r * n + col]) > std::fabs(A[(size_t)piv * n + col]))
        piv = r;
    if (A[(size_t)piv * n + col] == 0)
      return false;
    if (piv != col)
      for (int k = 0; k < n; k++) {
        std::swap(A[(size_t)piv * n + k], A[(size_t)col * n + k]);
        std::swap(X[(size_t)piv * n + k], X[(size_t)col * n + k]);
      }
    const double d = 1 / A[(size_t)col * n + col];
    for (int k = 0; k < n; k++) {
      A[(size_t)col * n + k] *= d;
      X[(size_t)col * n + k] *= d;
    }
    for (int r = 0; r < n; r++) {
      if (r == col)
        continue;
      const double fct = A[(size_t)r * n + col];
      if (fct == 0)
        continue;
      for (int k = 0; k < n; k++) {
        A[(size_t)r * n + k] -= fct * A[(size_t)col * n + k];
        X[(size_t)r * n + k] -= fct * X[(size_t)col * n + k];
      }
    }
  }
  inv.assign((size_t)n * n, 0.f);
  for (size_t k = 0; k < inv.size(); k++)
    inv[k] = (float)X[k];
  return true;
}
} // namespace

extern "C" int s32_mg_setup(const DevMesh *m, const int16_t *flags, Mg32Work *w, cudaStream_t s)
{
  s32_mg_free(w);
  const int lo = m->left_bc == SPIFFE_DIRICHLET ? 0 : 1;
  const int hi = m->right_bc == SPIFFE_DIRICHLET ? m->nz - 1 : m->nz - 2;
  std::vector<Stencil> lev(1);
  std::vector<std::vector<double>> rws(1);
  fine_stencil(*m, flags, lo, hi, lev[0]);
  // Semi-coarsening: where the spacing in one direction is at least twice
  // the other's, the operator couples nodes far more strongly along the
  // finer direction, point Gauss-Seidel smooths the error only along it,
  // and only that direction is coarsened (on a 165 x 357 gun mesh with
  // dz = 8 dr, 64 V-cycles a correction with both directions coarsened).
  std::vector<int> czs(1, 2), crs(1, 2);
  double sz = m->dz, sr = m->dr; // the finest level's spacings so far
  while ((int)lev.size() < MG_MAX_LEVELS) {
    const Stencil &F = lev.back();
    if (unknowns(F) <= (size_t)MG_MIN_UNKNOWNS)
      break;
    const int cz = sz >= 2 * sr ? 1 : 2, cr = sr >= 2 * sz ? 1 : 2;
    if ((cz == 2 && F.Z < 5) || (cr == 2 && F.R < 5))
      break;
    Stencil C;
    std::vector<double> rw;
    galerkin(F, C, rw, cz, cr);
    if (unknowns(C) == 0)
      break;
    lev.push_back(std::move(C));
    rws.push_back(std::move(rw));
    czs.push_back(cz);
    crs.push_back(cr);
    sz *= cz;
    sr *= cr;
  }
  const int L = (int)lev.size();
  if (L < 2)
    return (int)cudaErrorInvalidConfiguration; // a mesh too small to coarsen: the caller uses SOR
  // device layout: level 0's u0, f0 at the mesh pitch; per coarse level u,
  // f, MG_NCOEF coefficient planes of (Z+2) x P floats, rw of 3 R floats
  const size_t n0 = (size_t)(m->nz + 1) * m->pitch;
  size_t bytes = 2 * n0 * sizeof(float);
  std::vector<size_t> off(L), coff(L), roff(L);
  for (int l = 1; l < L; l++) {
    const int P = (lev[l].R + 2 + 31) / 32 * 32;
    const size_t plane = (size_t)(lev[l].Z + 2) * P;
    off[l] = bytes;
    bytes += 2 * plane * sizeof(float);
    coff[l] = bytes;
    bytes += MG_NCOEF * plane * sizeof(float);
    roff[l] = bytes;
    bytes += ((size_t)3 * lev[l].R * sizeof(float) + 255) / 256 * 256;
  }
  const size_t sums_off = bytes;
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_mg32, MG_NT, 0);
  if (e != cudaSuccess)
    return (int)e;
  if (per < 1)
    return (int)cudaErrorInvalidConfiguration;
  // one CTA per SM at most (every CTA resident), and no more CTAs than the
  // mesh gives work: a small mesh's solve then pays for fewer barrier
  // arrivals and leaves the other SMs to other instances' kernels
  const size_t mesh_nodes = (size_t)(m->nz + 1) * (m->nr + 1);
  const int grid = (int)std::min<size_t>((size_t)sms, std::max<size_t>(1, (mesh_nodes + MG_NODES_PER_CTA - 1) / MG_NODES_PER_CTA));
  bytes += (size_t)2 * grid * sizeof(double) + 32 * sizeof(unsigned long long) + sizeof(long long);
  char *mem = nullptr;
  e = cudaMalloc(&mem, bytes);
  if (e != cudaSuccess)
    return (int)e;
  e = cudaMemsetAsync(mem, 0, bytes, s); // halos, held nodes and level 0 start at zero
  w->mem = mem;
  w->bytes = bytes;
  w->nlev = L;
  w->grid = grid;
  w->threads = MG_NT;
  w->u0 = (float *)mem;
  w->f0 = (float *)mem + n0;
  w->part = (double *)(mem + sums_off);
  w->bar = (unsigned long long *)(mem + sums_off + (size_t)2 * grid * sizeof(double));
  w->iters = (long long *)(w->bar + 32);
  // the first level small enough for CTA 0 alone (at least level 1, at most the coarsest)
  int tail = L - 1;
  for (int l = 1; l < L; l++)
    if ((size_t)lev[l].Z * lev[l].R <= (size_t)MG_TAIL_NODES) {
      tail = l;
      break;
    }
  w->tail = tail;
  std::vector<float> hc, hr;
  for (int l = 1; l < L && e == cudaSuccess; l++) {
    const Stencil &S = lev[l];
    MgLevel &D = w->lev[l];
    D.Z = S.Z;
    D.R = S.R;
    D.cz = czs[l];
    D.cr = crs[l];
    D.P = (S.R + 2 + 31) / 32 * 32;
    const size_t plane = (size_t)(S.Z + 2) * D.P;
    D.u = (float *)(mem + off[l]);
    D.f = D.u + plane;
    D.coef = (const float *)(mem + coff[l]);
    D.rw = (const float *)(mem + roff[l]);
    hc.assign(MG_NCOEF * plane, 0.f);
    for (int I = 0; I < S.Z; I++)
      for (int J = 0; J < S.R; J++) {
        if (!S.unk[(size_t)I * S.R + J])
          continue;
        const size_t idx = (size_t)(I + 1) * D.P + J + 1;
        const double dg = S.at(4, I, J);
        int q = 0;
        for (int k = 0; k < 9; k++) {
          if (k == 4)
            continue;
          hc[(size_t)q * plane + idx] = (float)(S.at(k, I, J) / dg);
          q++;
        }
        hc[(size_t)MG_INVD * plane + idx] = (float)(1 / dg);
        hc[(size_t)MG_DIAG * plane + idx] = (float)dg;
      }
    hr.assign((size_t)3 * S.R, 0.f);
    for (size_t k = 0; k < hr.size(); k++)
      hr[k] = (float)rws[l][k];
    e = cudaMemcpyAsync(mem + coff[l], hc.data(), hc.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(mem + roff[l], hr.data(), hr.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaStreamSynchronize(s); // the host staging is reused by the next level
  }
  // the coarsest level's inverse for its exact solve
  std::vector<float> cinv;
  std::vector<int> cidx;
  if (e == cudaSuccess && coarse_inverse(lev[L - 1], w->lev[L - 1].P, cinv, cidx)) {
    e = cudaMalloc(&w->cinv, cinv.size() * sizeof(float));
    if (e == cudaSuccess)
      e = cudaMalloc(&w->cidx, cidx.size() * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(w->cinv, cinv.data(), cinv.size() * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(w->cidx, cidx.data(), cidx.size() * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaStreamSynchronize(s);
    w->cn = (int)cidx.size();
  }
  if (e != cudaSuccess)
    s32_mg_free(w);
  return (int)e;
}

// the solve on Psi with driving term rhs (null: Laplace), stop rule
// sum|r| < accuracy sum|rhs|, at most max_cycles V-cycles
extern "C" int s32_mg_solve(const DevMesh *m, Mg32Work *w, const float *crow, const float *drow, double *Psi,
                            const double *rhs, const uint8_t *umask, double accuracy, long long max_cycles,
                            PcState *st, long long *iters_out, DevCounts *cnt, cudaStream_t s)
{
  Mg32Args a{};
  a.Psi = Psi;
  a.rhs = rhs;
  a.umask = umask;
  a.u0 = w->u0;
  a.f0 = w->f0;
  a.crow = crow;
  a.drow = drow;
  a.nz = m->nz;
  a.P0 = m->pitch;
  a.lo = m->left_bc == SPIFFE_DIRICHLET ? 0 : 1;
  a.hi = m->right_bc == SPIFFE_DIRICHLET ? m->nz - 1 : m->nz - 2;
  a.cols = m->nr - 1;
  const double dz2 = m->dz * m->dz, dr2 = m->dr * m->dr;
  a.a_d = 1 / dz2;
  a.e_d = -2 * (1 / dz2 + 1 / dr2);
  a.c4_d = 4 / dr2;
  a.e2c_d = a.e_d - 2 / dr2;
  a.dr2_inv = 1 / dr2;
  a.a = (float)a.a_d;
  a.c4 = (float)a.c4_d;
  a.e = (float)a.e_d;
  a.e2c = (float)a.e2c_d;
  a.inv_e = (float)(1 / a.e_d);
  a.inv_e2c = (float)(1 / a.e2c_d);
  a.nlev = w->nlev;
  a.tail = w->tail;
  a.nu0 = 2;
  a.nu = 2;
  a.coarse_sweeps = 24;
  a.cinv = w->cinv;
  a.cidx = w->cidx;
  a.cn = w->cn;
  a.max_cycles = (int)std::min<long long>(max_cycles, 100);
  a.accuracy = accuracy;
  for (int l = 0; l < w->nlev; l++)
    a.lev[l] = w->lev[l];
  a.bar = w->bar;
  a.part = w->part;
  a.st = st;
  a.iters_out = iters_out ? iters_out : w->iters;
  cudaError_t e = cudaMemsetAsync(w->bar, 0, 32 * sizeof(unsigned long long), s);
  if (e != cudaSuccess)
    return (int)e;
  void *args[] = {&a, &cnt};
  e = cudaLaunchCooperativeKernel((const void *)k_mg32, dim3(w->grid), dim3(w->threads), args, 0, s);
  spiffe_note_launches(1);
  return (int)e;
}
