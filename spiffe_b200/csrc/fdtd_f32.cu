// spiffe_b200/csrc/fdtd_f32.cu -- FP32 Yee update of the split-precision form.
//
// The same update as advance_field_solutions (integrate.c:277-541) and the
// same one-writer-per-node structure as the FP64 kernels (each mesh node's
// final value, interior update or boundary copy, is written by exactly one
// thread), with these changes of representation:
//   * E and B are FP32 and dt is folded into the per-row metric factors;
//   * J arrives as 64-bit fixed point and is scaled by kJ = -dt qJ / eps0;
//     inside the integration loop the kernel zeroes J after reading it, so
//     the next step's deposition (fused into the push) starts from zero;
//   * the per-node flag tests and the FL_LAST_ACTIVE_PT row cut-offs are one
//     precomputed update-mask byte.
#include "split32.cuh"

#include <cmath>
#include <vector>

namespace {

constexpr int BX = 32, BY = 8;

struct Coef32 {
  const float *cpd, *cmd, *bzf;
  float fEr, topf, fEphi_dz, fEphi_dr, dt_dz, dt_dr, kJ;
  int zero_j;
  int reset_box; // this B kernel is the step's last: empty the current box
};

// rows [lo, hi] of the current box (lo > hi: no current anywhere)
__device__ __forceinline__ void jbox_rows(const int *jbox, int &lo, int &hi)
{
  lo = jbox[0];
  hi = jbox[1];
}

__device__ __forceinline__ void jbox_reset(int *jbox)
{
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
    jbox[0] = 0x7fffffff;
    jbox[1] = -1;
  }
}

// ---- the arithmetic of one node, each product and sum rounded on its own
// (no contraction), shared by the per-node, tiled and fused kernels so that
// all three give the same bits.
// Ez (integrate.c:323-344): ez + (kJ jz + (cp b1 - cm b0))
__device__ __forceinline__ float ez_next(float ez, float kJ, float jz, float cp, float b1, float cm, float b0)
{
  return __fadd_rn(ez, __fadd_rn(__fmul_rn(kJ, jz), __fsub_rn(__fmul_rn(cp, b1), __fmul_rn(cm, b0))));
}
// Er (integrate.c:362-368): er + (kJ jr - fEr (bP - b0))
__device__ __forceinline__ float er_next(float er, float kJ, float jr, float fEr, float bP, float b0)
{
  return __fadd_rn(er, __fsub_rn(__fmul_rn(kJ, jr), __fmul_rn(fEr, __fsub_rn(bP, b0))));
}
// dBphi (integrate.c:391-394): dt/dr (ez - ezm) - dt/dz (er - erm)
__device__ __forceinline__ float dbphi(float dt_dr, float ez, float ezm, float dt_dz, float er, float erm)
{
  return __fsub_rn(__fmul_rn(dt_dr, __fsub_rn(ez, ezm)), __fmul_rn(dt_dz, __fsub_rn(er, erm)));
}
__device__ __forceinline__ float half_step(float b, float dB) { return __fadd_rn(b, __fmul_rn(0.5f, dB)); }

// ---- TM update, one node at a time: the boundary rows and columns
// (copies to the axis, the top and the end rows) and the cells next to them.

// Ez and Er of node (iz, ir), 0 <= iz <= nz, 0 <= ir <= nr; J rows jlo..jhi
__device__ __forceinline__ void tm_e_node(const DevMesh &m, const DevFields32 &f, const Coef32 &c, int iz, int ir,
                                          int jlo, int jhi)
{
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  const size_t i = node(iz, ir, P);
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;
  const bool ez_row = ir < nr && iz >= 1 && iz <= nz - 1, er_row = iz <= nz - 1;
  // every load before any store, so no store can order the loads behind it;
  // J is read (and cleared) only on the rows a deposit touched
  const bool jrow = iz >= jlo && iz <= jhi;
  const uint8_t u = f.umask[i];
  const long long jz = jrow ? f.Jz[i] : 0, jr = jrow ? f.Jr[i] : 0;
  const float ez = ez_row ? f.Ez[i] : 0.f, er = er_row ? f.Er[i] : 0.f;
  const float b0 = f.Bphi[i];
  const float b1 = ez_row && ir < nr - 1 ? f.Bphi[i + 1] : 0.f;
  const float bP = er_row ? f.Bphi[i + P] : 0.f;
  const float cp = ir < nr - 1 ? c.cpd[ir] : 0.f, cm = ir < nr - 1 ? c.cmd[ir] : 0.f;
  // Ez (integrate.c:323-357)
  if (ez_row) {
    float v;
    if (ir == nr - 1) {
      v = 0.f;
    } else {
      v = ez;
      if (u & S32_U_EZ)
        v = ez_next(ez, c.kJ, (float)jz, cp, b1, cm, b0);
    }
    f.Ez[i] = v;
    if (iz == 1)
      f.Ez[node(0, ir, P)] = ir == nr - 1 ? 0.f : (leftN ? v : -v);
    if (iz == nz - 1)
      f.Ez[node(nz, ir, P)] = ir == nr - 1 ? 0.f : (rightN ? v : -v);
  }
  // Er (integrate.c:359-380)
  if (er_row) {
    const bool zero_row = (leftN && iz == 0) || (rightN && iz == nz - 1);
    if (ir >= 1 && ir <= nr - 1) {
      float v = er;
      if (u & S32_U_ER)
        v = er_next(er, c.kJ, (float)jr, c.fEr, bP, b0);
      f.Er[i] = zero_row ? 0.f : v;
      if (ir == 1)
        f.Er[node(iz, 0, P)] = zero_row ? 0.f : -v;
    } else if (ir == nr && zero_row) {
      f.Er[i] = 0.f;
    }
  }
  if (c.zero_j && jrow) {
    f.Jz[i] = 0;
    f.Jr[i] = 0;
  }
}

// Bphi and Bphi2 of node (iz, ir), 1 <= iz <= nz-1, 0 <= ir <= nr
__device__ __forceinline__ void tm_b_node(const DevMesh &m, const DevFields32 &f, const Coef32 &c, int iz, int ir)
{
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;
  const size_t i = node(iz, ir, P);
  float b = f.Bphi[i], b2;
  if (ir >= 1 && ir <= nr - 2) {
    const uint8_t u = f.umask[i];
    const float ez = f.Ez[i], ezm = f.Ez[i - 1], er = f.Er[i], erm = f.Er[i - P];
    if (u & S32_U_BPHI) {
      const float dB = dbphi(c.dt_dr, ez, ezm, c.dt_dz, er, erm);
      b2 = half_step(b, dB);
      b = __fadd_rn(b, dB);
      f.Bphi2[i] = b2;
      f.Bphi[i] = b;
    } else {
      b2 = f.Bphi2[i]; // the old half-step value is read only where it is kept
    }
    if (ir == 1) {
      f.Bphi[node(iz, 0, P)] = -b;
      f.Bphi2[node(iz, 0, P)] = -b2;
    }
    if (ir == nr - 2) {
      f.Bphi[node(iz, nr - 1, P)] = b * c.topf;
      f.Bphi2[node(iz, nr - 1, P)] = b2 * c.topf;
    }
    if (iz == 1 || iz == nz - 1) {
      // the end rows copy row 1 / row nz-1 after its axis and top copies (integrate.c:396-432)
      for (int side = 0; side < 2; side++) {
        if ((side == 0 && iz != 1) || (side == 1 && iz != nz - 1))
          continue;
        const int row = side == 0 ? 0 : nz;
        const float sg = (side == 0 ? leftN : rightN) ? 1.f : -1.f;
        f.Bphi[node(row, ir, P)] = sg * b;
        f.Bphi2[node(row, ir, P)] = sg * b2;
        if (ir == 1) {
          f.Bphi[node(row, 0, P)] = -sg * b;
          f.Bphi2[node(row, 0, P)] = -sg * b2;
        }
        if (ir == nr - 2) {
          f.Bphi[node(row, nr - 1, P)] = sg * b * c.topf;
          f.Bphi2[node(row, nr - 1, P)] = sg * b2 * c.topf;
        }
      }
    }
  } else if (ir == nr) {
    // column nr is never updated; the end rows still copy it
    b2 = f.Bphi2[i];
    if (iz == 1) {
      f.Bphi[node(0, nr, P)] = leftN ? b : -b;
      f.Bphi2[node(0, nr, P)] = leftN ? b2 : -b2;
    }
    if (iz == nz - 1) {
      f.Bphi[node(nz, nr, P)] = rightN ? b : -b;
      f.Bphi2[node(nz, nr, P)] = rightN ? b2 : -b2;
    }
  }
}

// ---- TM update, four columns per thread.  The launch has two kinds of
// blocks.  Interior tiles: a warp covers 32 groups of four consecutive
// columns of one row in 2 <= iz <= nz-2, every node of which is an ordinary
// interior node (no boundary copy); 16-byte loads and stores move four nodes
// at a time (rows start on 128-byte boundaries), every load is issued before
// the one shuffle that passes the neighbour column between lanes, so a thread
// waits for memory once.  Boundary blocks: one node per thread, with the
// per-node code above, over the rows and columns the tiles leave out; they
// take the first block indices, so they run beside the tiles.
constexpr int VX = 32, VY = 8, VW = 4; // lanes per row segment, rows per tile, columns per group

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }

// Work split of one TM kernel.  Groups g = 1..G cover columns 4..4G+3; the
// boundary columns are 0..left-1 and right..nr; rows 2..nz-2 are interior.
struct TmSplit {
  int G, tiles_x, tiles, left, right, W; // W: boundary nodes per interior row
  int nrows_b;                           // boundary rows (E: outside 2..nz-2; B: rows 1 and nz-1)
  long long nb;                          // boundary nodes in all
};

__host__ __device__ inline TmSplit tm_split(int nz, int nr, bool b_kernel)
{
  TmSplit t;
  const int last = b_kernel ? nr - 3 : nr - 2; // last column a group may reach
  t.G = last >= 7 ? (last - 3) / VW : 0;
  const int ni = nz - 3 > 0 ? nz - 3 : 0; // interior rows 2..nz-2
  t.tiles_x = (t.G + VX - 1) / VX;
  t.tiles = t.G > 0 ? t.tiles_x * ((ni + VY - 1) / VY) : 0;
  t.left = nr + 1 < VW ? nr + 1 : VW;
  t.right = t.G > 0 ? VW * t.G + VW : t.left;
  t.W = t.left + (nr + 1 - t.right);
  if (t.G == 0) // rows are boundary throughout
    t.W = nr + 1;
  if (b_kernel)
    t.nrows_b = nz >= 3 ? 2 : (nz == 2 ? 1 : 0);
  else
    t.nrows_b = (nz + 1) - ni;
  t.nb = (long long)t.nrows_b * (nr + 1) + (long long)ni * t.W;
  return t;
}

// boundary node k of the split -> (iz, ir)
__device__ __forceinline__ void tm_boundary_node(const TmSplit &t, int nz, int nr, bool b_kernel, long long k, int &iz,
                                                 int &ir)
{
  const long long nrow = (long long)t.nrows_b * (nr + 1);
  if (k < nrow) {
    const int r = (int)(k / (nr + 1));
    ir = (int)(k % (nr + 1));
    if (b_kernel)
      iz = r == 0 ? 1 : nz - 1;
    else
      iz = r < 2 ? r : nz - (t.nrows_b - 1 - r);
  } else {
    k -= nrow;
    iz = 2 + (int)(k / t.W);
    const int c = (int)(k % t.W);
    ir = t.G == 0 ? c : (c < t.left ? c : t.right + (c - t.left));
  }
}

__global__ void __launch_bounds__(VX *VY) k_tm_e32(DevMesh m, DevFields32 f, Coef32 c, TmSplit t)
{
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  int jlo, jhi;
  jbox_rows(f.jbox, jlo, jhi);
  // the boundary blocks come first, so they run beside the tiles, not after them
  const int nbb = (int)((t.nb + VX * VY - 1) / (VX * VY));
  if ((int)blockIdx.x < nbb) {
    const long long k = (long long)blockIdx.x * (VX * VY) + threadIdx.y * VX + threadIdx.x;
    if (k < t.nb) {
      int iz, ir;
      tm_boundary_node(t, nz, nr, false, k, iz, ir);
      tm_e_node(m, f, c, iz, ir, jlo, jhi);
    }
    return;
  }
  const int tile = blockIdx.x - nbb;
  const int tx = tile % t.tiles_x, ty = tile / t.tiles_x;
  const int g = 1 + tx * VX + threadIdx.x, iz = 2 + ty * VY + threadIdx.y;
  if (iz > nz - 2) // whole warps: a warp is one row segment
    return;
  const int ir0 = g * VW;
  const bool mine = g <= t.G, in_row = ir0 <= nr;
  const size_t i = node(iz, ir0, P);
  const bool jrow = iz >= jlo && iz <= jhi;
  // every load first; the next group's first Bphi comes from the next lane
  float4 b0 = make_float4(0.f, 0.f, 0.f, 0.f), ez = b0, er = b0, bP = b0, cp = b0, cm = b0;
  uchar4 u = make_uchar4(0, 0, 0, 0);
  longlong2 z01 = make_longlong2(0, 0), z23 = z01, r01 = z01, r23 = z01;
  float bnext = 0.f;
  if (in_row)
    b0 = ldg4(f.Bphi + i);
  if (mine) {
    u = __ldg(reinterpret_cast<const uchar4 *>(f.umask + i));
    ez = ld4(f.Ez + i);
    er = ld4(f.Er + i);
    bP = ldg4(f.Bphi + i + P);
    cp = ldg4(c.cpd + ir0);
    cm = ldg4(c.cmd + ir0);
    if (jrow) {
      z01 = *reinterpret_cast<const longlong2 *>(f.Jz + i);
      z23 = *reinterpret_cast<const longlong2 *>(f.Jz + i + 2);
      r01 = *reinterpret_cast<const longlong2 *>(f.Jr + i);
      r23 = *reinterpret_cast<const longlong2 *>(f.Jr + i + 2);
    }
    if (threadIdx.x == VX - 1)
      bnext = __ldg(f.Bphi + i + VW); // ir0 + 4 <= nr - 1: inside the row
  }
  const float bsh = __shfl_down_sync(0xffffffffu, b0.x, 1);
  if (!mine)
    return;
  if (threadIdx.x != VX - 1)
    bnext = bsh;
  const float jz0 = (float)z01.x, jz1 = (float)z01.y, jz2 = (float)z23.x, jz3 = (float)z23.y;
  const float jr0 = (float)r01.x, jr1 = (float)r01.y, jr2 = (float)r23.x, jr3 = (float)r23.y;
  // integrate.c:323-344 and :362-368 on four interior nodes
  if (u.x & S32_U_EZ) ez.x = ez_next(ez.x, c.kJ, jz0, cp.x, b0.y, cm.x, b0.x);
  if (u.y & S32_U_EZ) ez.y = ez_next(ez.y, c.kJ, jz1, cp.y, b0.z, cm.y, b0.y);
  if (u.z & S32_U_EZ) ez.z = ez_next(ez.z, c.kJ, jz2, cp.z, b0.w, cm.z, b0.z);
  if (u.w & S32_U_EZ) ez.w = ez_next(ez.w, c.kJ, jz3, cp.w, bnext, cm.w, b0.w);
  if (u.x & S32_U_ER) er.x = er_next(er.x, c.kJ, jr0, c.fEr, bP.x, b0.x);
  if (u.y & S32_U_ER) er.y = er_next(er.y, c.kJ, jr1, c.fEr, bP.y, b0.y);
  if (u.z & S32_U_ER) er.z = er_next(er.z, c.kJ, jr2, c.fEr, bP.z, b0.z);
  if (u.w & S32_U_ER) er.w = er_next(er.w, c.kJ, jr3, c.fEr, bP.w, b0.w);
  st4(f.Ez + i, ez);
  st4(f.Er + i, er);
  if (c.zero_j && jrow) {
    const longlong2 zero = make_longlong2(0, 0);
    *reinterpret_cast<longlong2 *>(f.Jz + i) = zero;
    *reinterpret_cast<longlong2 *>(f.Jz + i + 2) = zero;
    *reinterpret_cast<longlong2 *>(f.Jr + i) = zero;
    *reinterpret_cast<longlong2 *>(f.Jr + i + 2) = zero;
  }
}

__global__ void __launch_bounds__(VX *VY) k_tm_b32(DevMesh m, DevFields32 f, Coef32 c, TmSplit t)
{
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (c.reset_box)
    jbox_reset(f.jbox);
  const int nbb = (int)((t.nb + VX * VY - 1) / (VX * VY));
  if ((int)blockIdx.x < nbb) {
    const long long k = (long long)blockIdx.x * (VX * VY) + threadIdx.y * VX + threadIdx.x;
    if (k < t.nb) {
      int iz, ir;
      tm_boundary_node(t, nz, nr, true, k, iz, ir);
      tm_b_node(m, f, c, iz, ir);
    }
    return;
  }
  const int tile = blockIdx.x - nbb;
  const int tx = tile % t.tiles_x, ty = tile / t.tiles_x;
  const int g = 1 + tx * VX + threadIdx.x, iz = 2 + ty * VY + threadIdx.y;
  if (iz > nz - 2) // whole warps
    return;
  const int ir0 = g * VW;
  const bool mine = g <= t.G, in_row = ir0 <= nr;
  const size_t i = node(iz, ir0, P);
  // every load first; the previous group's last Ez comes from the previous lane
  float4 ez = make_float4(0.f, 0.f, 0.f, 0.f), er = ez, erm = ez, b = ez;
  uchar4 u = make_uchar4(0, 0, 0, 0);
  float eprev = 0.f;
  if (in_row)
    ez = ldg4(f.Ez + i);
  if (mine) {
    u = __ldg(reinterpret_cast<const uchar4 *>(f.umask + i));
    er = ldg4(f.Er + i);
    erm = ldg4(f.Er + i - P);
    b = ld4(f.Bphi + i);
    if (threadIdx.x == 0)
      eprev = __ldg(f.Ez + i - 1); // ir0 - 1 >= 3: inside the row
  }
  const float esh = __shfl_up_sync(0xffffffffu, ez.w, 1);
  if (!mine)
    return;
  if (threadIdx.x != 0)
    eprev = esh;
  // integrate.c:391-394 on four interior nodes
  const float dBx = dbphi(c.dt_dr, ez.x, eprev, c.dt_dz, er.x, erm.x);
  const float dBy = dbphi(c.dt_dr, ez.y, ez.x, c.dt_dz, er.y, erm.y);
  const float dBz = dbphi(c.dt_dr, ez.z, ez.y, c.dt_dz, er.z, erm.z);
  const float dBw = dbphi(c.dt_dr, ez.w, ez.z, c.dt_dz, er.w, erm.w);
  const bool ux = u.x & S32_U_BPHI, uy = u.y & S32_U_BPHI, uz = u.z & S32_U_BPHI, uw = u.w & S32_U_BPHI;
  float4 b2;
  b2.x = half_step(b.x, dBx);
  b2.y = half_step(b.y, dBy);
  b2.z = half_step(b.z, dBz);
  b2.w = half_step(b.w, dBw);
  if (ux && uy && uz && uw) {
    b.x = __fadd_rn(b.x, dBx);
    b.y = __fadd_rn(b.y, dBy);
    b.z = __fadd_rn(b.z, dBz);
    b.w = __fadd_rn(b.w, dBw);
    st4(f.Bphi2 + i, b2);
    st4(f.Bphi + i, b);
  } else {
    // a node that is not updated keeps both of its values (next to metal)
    if (ux) { f.Bphi2[i] = b2.x; f.Bphi[i] = __fadd_rn(b.x, dBx); }
    if (uy) { f.Bphi2[i + 1] = b2.y; f.Bphi[i + 1] = __fadd_rn(b.y, dBy); }
    if (uz) { f.Bphi2[i + 2] = b2.z; f.Bphi[i + 2] = __fadd_rn(b.z, dBz); }
    if (uw) { f.Bphi2[i + 3] = b2.w; f.Bphi[i + 3] = __fadd_rn(b.w, dBw); }
  }
}

// ---- TM update fused into one persistent kernel: E then B, row by row.
//
// Each block owns a band of rows [z0, z1) across the whole row and sweeps it
// in order of z.  Rows arrive in a ring of FS shared-memory stages by bulk
// copies (cp.async.bulk: one thread issues a row of each array and an
// mbarrier per stage counts the bytes in), so each SM keeps several rows in
// flight without a thread waiting on a load.  Row iz's E update reads Bphi
// of rows iz and iz+1; its B update reads the new Ez of the row and the new
// Er of rows iz and iz-1 (the latter kept in registers from the row before).
// Each node is then read once and written once: Ez, Er and Bphi read and
// written, Bphi2 written, the mask byte read and, on rows that hold
// current, J read and zeroed.
//
// Neighbouring bands meet at one row: band k's first B update needs the new
// Er of row z0-1, which band k-1 computes, and band k-1's last E update
// needs the old Bphi of row z0, which band k overwrites.  So each band first
// computes the new Er of its last row from the old values and publishes it
// (a row in global memory, then its flag set to the launch's epoch); a band
// waits for its neighbour's flag before its first B update, and so before it
// writes its first Bphi row.  The launch is cooperative (every band resident)
// and every wait is bounded: one that runs out sets SPIFFE_DEV_ERR_WAIT, and
// the block stops computing, drains its copies and returns.
constexpr bool FUSED_BY_DEFAULT = false;       // SPIFFE_FDTD_AUTO takes the fused kernel on large meshes
constexpr int FS = 4;                          // ring stages
constexpr unsigned long long WAIT_NS = 1000000000ull; // a wait gives up after one second

__device__ __forceinline__ unsigned long long now_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

struct FusedArgs {
  float *pub;          // bands x P: the new Er of each band's last row
  unsigned *flag;      // per band: the epoch its row was published for
  unsigned *arrivals;  // blocks that have read the current box (the last resets it)
  unsigned *err;
  int rows_per, bands;
  unsigned epoch;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_done(uint64_t *bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok)
               : "r"(smem_addr(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

// one row of an array, global -> shared, counted by the stage's mbarrier
// (16-byte aligned addresses, a multiple of 16 bytes: rows start on 128-byte
// boundaries and P is a multiple of 32)
__device__ __forceinline__ void bulk_row(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v)
{
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// bytes of one stage and its layout: Ez, Er, Bphi (floats), Jz, Jr (64-bit), mask
__host__ __device__ inline size_t fused_stage_bytes(int P) { return (size_t)29 * P; }
__host__ __device__ inline size_t fused_smem(int P) { return FS * fused_stage_bytes(P) + (size_t)16 * P + 8 * FS + 64; }

__global__ void k_tm_fused32(DevMesh m, DevFields32 f, Coef32 c, FusedArgs a)
{
  extern __shared__ __align__(128) unsigned char sm[];
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  const int tid = threadIdx.x;
  const int band = blockIdx.x;
  const int z0 = band * a.rows_per, z1 = min(z0 + a.rows_per, nz); // E rows z0..z1-1 (row nz is copies)
  const bool last_band = z1 == nz;
  const size_t SB = fused_stage_bytes(P);
  float *ezn = reinterpret_cast<float *>(sm + FS * SB);  // the row's new Ez (neighbour reads)
  float *bnx = ezn + P;                                   // old Bphi of row z1
  float *bnr = bnx + P;                                   // the row's new Bphi
  float *b2r = bnr + P;                                   // the row's new (or kept) Bphi2
  uint64_t *bar = reinterpret_cast<uint64_t *>(b2r + P);
  // [0] abort, [1] jlo, [2] jhi, [3 + st] rows issued into stage st
  volatile int *flags = reinterpret_cast<volatile int *>(bar + FS);
  auto stEz = [&](int st) { return reinterpret_cast<float *>(sm + st * SB); };
  auto stEr = [&](int st) { return reinterpret_cast<float *>(sm + st * SB + 4 * (size_t)P); };
  auto stB = [&](int st) { return reinterpret_cast<float *>(sm + st * SB + 8 * (size_t)P); };
  auto stJz = [&](int st) { return reinterpret_cast<long long *>(sm + st * SB + 12 * (size_t)P); };
  auto stJr = [&](int st) { return reinterpret_cast<long long *>(sm + st * SB + 20 * (size_t)P); };
  auto stU = [&](int st) { return sm + st * SB + 28 * (size_t)P; };
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;

  if (tid == 0) {
    flags[0] = 0;
    flags[1] = f.jbox[0];
    flags[2] = f.jbox[1];
    for (int st = 0; st < FS; st++) {
      mbar_init(bar + st);
      flags[3 + st] = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int jlo = flags[1], jhi = flags[2];
  if (tid == 0 && c.reset_box) {
    // the last block to have read the box empties it for the next deposit
    __threadfence();
    if (atomicAdd(a.arrivals, 1u) == (unsigned)a.bands - 1) {
      *a.arrivals = 0;
      f.jbox[0] = 0x7fffffff;
      f.jbox[1] = -1;
    }
  }
  auto jrow = [&](int iz) { return iz >= jlo && iz <= jhi; };
  // issue row iz into stage st (one thread)
  auto issue = [&](int iz, int st) {
    const size_t o = (size_t)iz * P;
    uint32_t bytes = 12u * (uint32_t)P + (uint32_t)P;
    const bool j = jrow(iz);
    if (j)
      bytes += 16u * (uint32_t)P;
    mbar_expect(bar + st, bytes);
    bulk_row(stEz(st), f.Ez + o, 4u * P, bar + st);
    bulk_row(stEr(st), f.Er + o, 4u * P, bar + st);
    bulk_row(stB(st), f.Bphi + o, 4u * P, bar + st);
    bulk_row(stU(st), f.umask + o, (uint32_t)P, bar + st);
    if (j) {
      bulk_row(stJz(st), f.Jz + o, 8u * P, bar + st);
      bulk_row(stJr(st), f.Jr + o, 8u * P, bar + st);
    }
    flags[3 + st] = flags[3 + st] + 1;
  };
  const int nrow = z1 - z0;
  if (tid == 0)
    for (int q = 0; q < FS && q < nrow; q++)
      issue(z0 + q, q);

  // the columns of this thread: 4 tid .. 4 tid + 3
  const int c0 = 4 * tid;
  const bool have = c0 < P;
  // old Bphi of row z1 (the next band's first row, or the copy row nz)
  if (have)
    for (int q = 0; q < 4; q++)
      bnx[c0 + q] = f.Bphi[(size_t)z1 * P + c0 + q];

  // the new Er of the band's last row, from the old values, for the next band
  auto er_of = [&](int iz, int ir, float er, long long jr, uint8_t u, float b0, float bP) {
    const bool zero_row = (leftN && iz == 0) || (rightN && iz == nz - 1);
    if (ir >= 1 && ir <= nr - 1) {
      float v = er;
      if (u & S32_U_ER)
        v = er_next(er, c.kJ, (float)jr, c.fEr, bP, b0);
      return zero_row ? 0.f : v;
    }
    if (ir == nr && zero_row)
      return 0.f;
    return er; // column 0 is set from column 1 by the caller; column nr and the padding keep their values
  };
  if (!last_band && have) {
    const int iz = z1 - 1;
    const size_t o = (size_t)iz * P;
    float v[4];
    for (int q = 0; q < 4; q++) {
      const int ir = c0 + q;
      const long long jr = jrow(iz) ? f.Jr[o + ir] : 0;
      v[q] = er_of(iz, ir, f.Er[o + ir], jr, f.umask[o + ir], f.Bphi[o + ir], bnx[ir]);
    }
    if (c0 == 0) { // column 0 copies column 1 (integrate.c:369-370)
      const bool zero_row = (leftN && iz == 0) || (rightN && iz == nz - 1);
      v[0] = zero_row ? 0.f : -v[1];
    }
    for (int q = 0; q < 4; q++)
      a.pub[(size_t)band * P + c0 + q] = v[q];
  }
  __syncthreads();
  if (tid == 0 && !last_band) {
    __threadfence();
    st_release(a.flag + band, a.epoch);
  }
  // the new Er of row z0-1 from the band before
  float erp[4] = {0.f, 0.f, 0.f, 0.f};
  if (band > 0) {
    if (tid == 0) {
      const unsigned long long t0 = now_ns();
      while (ld_acquire(a.flag + band - 1) != a.epoch)
        if (now_ns() - t0 > WAIT_NS) {
          atomicOr(a.err, SPIFFE_DEV_ERR_WAIT);
          flags[0] = 1;
          break;
        }
    }
    __syncthreads();
    if (have)
      for (int q = 0; q < 4; q++)
        erp[q] = __ldcg(a.pub + (size_t)(band - 1) * P + c0 + q);
  }

  for (int k = 0; k < nrow; k++) {
    const int iz = z0 + k, st = k % FS;
    const uint32_t par = (uint32_t)(k / FS) & 1u;
    // this row's stage and, inside the band, the next row's
    unsigned long long t0 = now_ns();
    while (!flags[0] && !mbar_done(bar + st, par))
      if (now_ns() - t0 > WAIT_NS) {
        atomicOr(a.err, SPIFFE_DEV_ERR_WAIT);
        flags[0] = 1;
      }
    const bool next_in = k + 1 < nrow;
    const int st1 = (k + 1) % FS;
    if (next_in) {
      t0 = now_ns();
      while (!flags[0] && !mbar_done(bar + st1, (uint32_t)((k + 1) / FS) & 1u))
        if (now_ns() - t0 > WAIT_NS) {
          atomicOr(a.err, SPIFFE_DEV_ERR_WAIT);
          flags[0] = 1;
        }
    }
    __syncthreads();
    const bool ok = !flags[0];
    const float *Ez = stEz(st), *Er = stEr(st), *B = stB(st);
    const float *Bn = next_in ? stB(st1) : bnx;
    const long long *Jz = stJz(st), *Jr = stJr(st);
    const uint8_t *U = stU(st);
    const bool jr_ = jrow(iz);
    // E (integrate.c:323-380), as tm_e_node
    float ezo[4], ero[4];
    const bool ez_row = iz >= 1 && iz <= nz - 1;
    const bool zero_row = (leftN && iz == 0) || (rightN && iz == nz - 1);
    if (ok && have) {
      for (int q = 0; q < 4; q++) {
        const int ir = c0 + q;
        const uint8_t u = U[ir];
        const float b0 = B[ir];
        float v = Ez[ir];
        if (ez_row && ir < nr) {
          if (ir == nr - 1)
            v = 0.f;
          else if (u & S32_U_EZ)
            v = ez_next(v, c.kJ, jr_ ? (float)Jz[ir] : 0.f, c.cpd[ir], B[ir + 1], c.cmd[ir], b0);
        }
        ezo[q] = v;
        ero[q] = er_of(iz, ir, Er[ir], jr_ ? Jr[ir] : 0, u, b0, Bn[ir]);
      }
      if (c0 == 0)
        ero[0] = zero_row ? 0.f : -ero[1];
      for (int q = 0; q < 4; q++)
        ezn[c0 + q] = ezo[q];
    }
    __syncthreads();
    // B (integrate.c:391-432), as tm_b_node: the row's values into bnr / b2r
    const bool b_row = iz >= 1 && iz <= nz - 1;
    if (ok && have && b_row) {
      for (int q = 0; q < 4; q++) {
        const int ir = c0 + q;
        const float b = B[ir];
        float bn = b, b2 = 0.f;
        if (ir >= 1 && ir <= nr - 2) {
          if (U[ir] & S32_U_BPHI) {
            const float dB = dbphi(c.dt_dr, ezo[q], ezn[ir - 1], c.dt_dz, ero[q], erp[q]);
            b2 = half_step(b, dB);
            bn = __fadd_rn(b, dB);
          } else {
            b2 = f.Bphi2[(size_t)iz * P + ir]; // kept where not updated
          }
        } else if (ir == nr) {
          b2 = f.Bphi2[(size_t)iz * P + ir];
        }
        bnr[ir] = bn;
        b2r[ir] = b2;
      }
    }
    __syncthreads();
    if (ok && have) {
      const size_t o = (size_t)iz * P;
      // Ez: the updated columns (ir < nr) of rows 1..nz-1, unchanged values elsewhere
      if (ez_row)
        st4(f.Ez + o + c0, make_float4(ezo[0], ezo[1], ezo[2], ezo[3]));
      st4(f.Er + o + c0, make_float4(ero[0], ero[1], ero[2], ero[3]));
      for (int side = 0; side < 2 && ez_row; side++) { // the end rows copy rows 1 and nz-1
        if ((side == 0 && iz != 1) || (side == 1 && iz != nz - 1))
          continue;
        const size_t e = (size_t)(side == 0 ? 0 : nz) * P;
        const bool neu = side == 0 ? leftN : rightN;
        for (int q = 0; q < 4; q++) {
          const int ir = c0 + q;
          if (ir < nr)
            f.Ez[e + ir] = ir == nr - 1 ? 0.f : (neu ? ezo[q] : -ezo[q]);
        }
      }
      if (b_row) {
        float bo[4], b2o[4];
        bool w2[4];
        for (int q = 0; q < 4; q++) {
          const int ir = c0 + q;
          bo[q] = bnr[ir];
          b2o[q] = b2r[ir];
          w2[q] = ir >= 1 && ir <= nr - 2 && (U[ir] & S32_U_BPHI);
          if (ir == 0) {
            bo[q] = -bnr[1];
            b2o[q] = -b2r[1];
            w2[q] = true;
          } else if (ir == nr - 1) {
            bo[q] = bnr[nr - 2] * c.topf;
            b2o[q] = b2r[nr - 2] * c.topf;
            w2[q] = true;
          }
        }
        st4(f.Bphi + o + c0, make_float4(bo[0], bo[1], bo[2], bo[3]));
        if (w2[0] && w2[1] && w2[2] && w2[3])
          st4(f.Bphi2 + o + c0, make_float4(b2o[0], b2o[1], b2o[2], b2o[3]));
        else
          for (int q = 0; q < 4; q++)
            if (w2[q])
              f.Bphi2[o + c0 + q] = b2o[q];
        for (int side = 0; side < 2; side++) { // end rows (integrate.c:396-432)
          if ((side == 0 && iz != 1) || (side == 1 && iz != nz - 1))
            continue;
          const size_t e = (size_t)(side == 0 ? 0 : nz) * P;
          const float sg = (side == 0 ? leftN : rightN) ? 1.f : -1.f;
          for (int q = 0; q < 4; q++) {
            const int ir = c0 + q;
            if (ir > nr)
              continue;
            float v, v2;
            if (ir == 0) {
              v = -sg * bnr[1];
              v2 = -sg * b2r[1];
            } else if (ir == nr - 1) {
              v = sg * bnr[nr - 2] * c.topf;
              v2 = sg * b2r[nr - 2] * c.topf;
            } else {
              v = sg * bnr[ir];
              v2 = sg * b2r[ir];
            }
            f.Bphi[e + ir] = v;
            f.Bphi2[e + ir] = v2;
          }
        }
      }
      if (c.zero_j && jr_) {
        const longlong2 zero = make_longlong2(0, 0);
        *reinterpret_cast<longlong2 *>(f.Jz + o + c0) = zero;
        *reinterpret_cast<longlong2 *>(f.Jz + o + c0 + 2) = zero;
        *reinterpret_cast<longlong2 *>(f.Jr + o + c0) = zero;
        *reinterpret_cast<longlong2 *>(f.Jr + o + c0 + 2) = zero;
      }
      for (int q = 0; q < 4; q++)
        erp[q] = ero[q];
    }
    __syncthreads();
    // the stage is free: the row FS ahead goes into it
    if (tid == 0 && !flags[0] && k + FS < nrow) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(z0 + k + FS, st);
    }
  }
  // the copy row nz holds no E update of its own, but its current is cleared
  if (last_band && c.zero_j && jrow(nz) && have && !flags[0]) {
    const size_t o = (size_t)nz * P;
    for (int q = 0; q < 4; q++) {
      f.Jz[o + c0 + q] = 0;
      f.Jr[o + c0 + q] = 0;
    }
  }
  // after a wait ran out: let every issued copy land before the block exits
  if (tid == 0 && flags[0]) {
    for (int st = 0; st < FS; st++) {
      const int n = flags[3 + st]; // copies into this stage: its phase n - 1 is the last
      const unsigned long long t0 = now_ns();
      if (n > 0)
        while (!mbar_done(bar + st, (uint32_t)(n - 1) & 1u) && now_ns() - t0 < WAIT_NS) {
        }
    }
  }
}

// Ephi (integrate.c:449-471)
__global__ void __launch_bounds__(BX *BY) k_te_e32(DevMesh m, DevFields32 f, Coef32 c)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (ir > nr || iz > nz)
    return;
  const size_t i = node(iz, ir, P);
  int jlo, jhi;
  jbox_rows(f.jbox, jlo, jhi);
  const bool jrow = iz >= jlo && iz <= jhi;
  const long long jphi = jrow ? f.Jphi[i] : 0;
  if (c.zero_j && jrow)
    f.Jphi[i] = 0;
  const bool zero = ir == 0 || (m.right_bc == SPIFFE_NEUMANN && iz == nz - 1) ||
                    (m.left_bc == SPIFFE_NEUMANN && iz == 0) || (m.upper_bc == SPIFFE_NEUMANN && ir == nr - 1);
  if (zero) {
    f.Ephi[i] = 0.f;
    return;
  }
  if (ir >= 1 && ir <= nr - 1 && iz <= nz - 1 && (f.umask[i] & S32_U_EPHI))
    f.Ephi[i] += c.kJ * (float)jphi + c.fEphi_dz * (f.Br[i + P] - f.Br[i]) - c.fEphi_dr * (f.Bz[i + 1] - f.Bz[i]);
}

// Br/Br2 and Bz/Bz2 (integrate.c:473-539)
__global__ void __launch_bounds__(BX *BY) k_te_b32(DevMesh m, DevFields32 f, Coef32 c)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (c.reset_box)
    jbox_reset(f.jbox);
  if (ir > nr || iz > nz)
    return;
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;
  const size_t i = node(iz, ir, P);
  const uint8_t u = f.umask[i];
  if (iz >= 1 && iz <= nz - 1) {
    float b = f.Br[i], b2 = f.Br2[i];
    if (ir <= nr - 1 && (u & S32_U_BR)) {
      const float dB = c.dt_dz * (f.Ephi[i] - f.Ephi[i - P]);
      b2 = b + 0.5f * dB;
      b += dB;
      f.Br2[i] = b2;
      f.Br[i] = b;
    }
    if (iz == nz - 1) {
      f.Br[node(nz, ir, P)] = rightN ? b : -b;
      f.Br2[node(nz, ir, P)] = rightN ? b2 : -b2;
    }
    if (iz == 1) {
      f.Br[node(0, ir, P)] = leftN ? b : -b;
      f.Br2[node(0, ir, P)] = leftN ? b2 : -b2;
    }
  }
  const bool zero_row = (rightN && iz == nz - 1) || (leftN && iz == 0);
  if (ir >= 1 && ir <= nr - 1) {
    float b = f.Bz[i], b2 = f.Bz2[i];
    if (iz <= nz - 1 && (u & S32_U_BZ)) {
      const float dB = c.bzf[ir] * ((float)(ir + 1) * f.Ephi[i] - (float)ir * f.Ephi[i - 1]);
      b2 = b + 0.5f * dB;
      b += dB;
    }
    f.Bz[i] = zero_row ? 0.f : b;
    f.Bz2[i] = zero_row ? 0.f : b2;
    if (ir == 1) {
      f.Bz[node(iz, 0, P)] = zero_row ? 0.f : b;
      f.Bz2[node(iz, 0, P)] = zero_row ? 0.f : b2;
    }
  } else if (ir == nr && zero_row) {
    f.Bz[i] = 0.f;
    f.Bz2[i] = 0.f;
  }
}

// ---- representation changes between the host's FP64 (pitch nr+1) arrays
// and the device's pitched arrays

__global__ void k_to_f32(int nz, int nr, int P, const double *src, float *dst)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  if (iz > nz || ir >= P)
    return;
  dst[node(iz, ir, P)] = ir <= nr ? (float)src[node(iz, ir, nr + 1)] : 0.f;
}

__global__ void k_from_f32(int nz, int nr, int P, const float *src, double *dst)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  if (iz > nz || ir > nr)
    return;
  dst[node(iz, ir, nr + 1)] = (double)src[node(iz, ir, P)];
}

__global__ void k_to_f64p(int nz, int nr, int P, const double *src, double *dst)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  if (iz > nz || ir >= P)
    return;
  dst[node(iz, ir, P)] = ir <= nr ? src[node(iz, ir, nr + 1)] : 0.0;
}

__global__ void k_from_f64p(int nz, int nr, int P, const double *src, double *dst)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  if (iz > nz || ir > nr)
    return;
  dst[node(iz, ir, nr + 1)] = src[node(iz, ir, P)];
}

__global__ void k_to_fixed(int nz, int nr, int P, const double *src, long long *dst, double inv_q)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  if (iz > nz || ir >= P)
    return;
  dst[node(iz, ir, P)] = ir <= nr ? __double2ll_rn(src[node(iz, ir, nr + 1)] * inv_q) : 0;
}

__global__ void k_from_fixed(int nz, int nr, int P, const long long *src, double *dst, double q)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  if (iz > nz || ir > nr)
    return;
  dst[node(iz, ir, nr + 1)] = (double)src[node(iz, ir, P)] * q;
}

__global__ void k_antenna32(long long *J, int *jbox, int P, int direction, long istart, long iend, long iposition,
                            long long v)
{
  const long i = istart + (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > iend)
    return;
  // antenna.c:398-415
  const int nd = direction == 1 ? (int)node((int)iposition, (int)i, P) : (int)node((int)i, (int)iposition, P);
  J[nd] += v;
  atomicMin(jbox, nd / P);
  atomicMax(jbox + 1, nd / P);
}

__global__ void k_jbox_set(int *jbox, int lo, int hi)
{
  jbox[0] = lo;
  jbox[1] = hi;
}

// a >>= shift with rounding to nearest: values in old quanta to quanta 2^shift times larger
__global__ void k_rescale_fixed(long long *a, size_t n, int shift)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const long long v = a[i];
  a[i] = shift >= 63 ? 0 : (v + (1LL << (shift - 1))) >> shift;
}

dim3 grid_for(const DevMesh *m, int cols) { return dim3((cols + BX - 1) / BX, (m->nz + 1 + BY - 1) / BY); }

} // namespace

// Per-row metric factors (dt folded in) and the update mask.
extern "C" int s32_fdtd_tables(const DevMesh *m, const int16_t *host_flags, Fdtd32Tables *t, uint8_t *d_umask,
                               cudaStream_t s)
{
  const int nz = m->nz, nr = m->nr, P = m->pitch;
  const double dti = m->dt, dr = m->dr, dz = m->dz;
  const double eps0 = SPIFFE_EPSILON_O, mu0 = SPIFFE_MU_O, factor = 1 / (eps0 * mu0);
  std::vector<float> cpd(nr + 1), cmd(nr + 1), bzf(nr + 1);
  std::vector<int> cut0(nr + 1), cut1(nr + 1);
  for (int ir = 0; ir <= nr; ir++) {
    const double rp = (ir + 0.5) * dr, rm = (ir - 0.5) * dr;
    double cp, cm;
    if (ir != 0) {
      cp = 2 * factor / (rp * rp - rm * rm);
      cm = rm * cp;
      cp = rp * cp;
    } else {
      cp = 4 * factor / dr;
      cm = 0;
    }
    cpd[ir] = (float)(dti * cp);
    cmd[ir] = (float)(dti * cm);
    bzf[ir] = ir >= 1 ? (float)(-2 * dti / (dr * (double)((long)(ir + 1) * (ir + 1) - (long)ir * ir))) : 0.f;
    int c0 = nz - 1, c1 = nz - 1;
    for (int iz = 0; iz < nz; iz++)
      if (host_flags[(size_t)iz * (nr + 1) + ir] & SPIFFE_FL_LAST_ACTIVE_PT) {
        c0 = iz;
        break;
      }
    for (int iz = 1; iz < nz; iz++)
      if (host_flags[(size_t)iz * (nr + 1) + ir] & SPIFFE_FL_LAST_ACTIVE_PT) {
        c1 = iz;
        break;
      }
    cut0[ir] = c0;
    cut1[ir] = c1;
  }
  std::vector<uint8_t> um((size_t)(nz + 1) * P, 0);
  for (int iz = 0; iz <= nz; iz++)
    for (int ir = 0; ir <= nr; ir++) {
      const int16_t fl = host_flags[(size_t)iz * (nr + 1) + ir];
      uint8_t u = 0;
      if (iz <= cut1[ir] && !(fl & SPIFFE_FL_EZ_ZERO)) u |= S32_U_EZ;
      if (iz <= cut0[ir] && !(fl & SPIFFE_FL_ER_ZERO)) u |= S32_U_ER;
      if (iz <= cut1[ir] && !(fl & SPIFFE_FL_BPHI_ZERO)) u |= S32_U_BPHI;
      if (iz <= cut0[ir] && !(fl & SPIFFE_FL_EPHI_ZERO)) u |= S32_U_EPHI;
      if (iz <= cut1[ir] && !(fl & SPIFFE_FL_BR_ZERO)) u |= S32_U_BR;
      if (iz <= cut0[ir] && !(fl & SPIFFE_FL_BZ_ZERO)) u |= S32_U_BZ;
      if (fl & SPIFFE_FL_IS_METAL) u |= S32_U_METAL;
      bool clean = true;
      for (int z = iz - 1; z <= iz + 1 && clean; z++)
        for (int r = ir; r <= ir + 1 && clean; r++)
          if (z >= 0 && z <= nz && r <= nr && host_flags[(size_t)z * (nr + 1) + r])
            clean = false;
      if (clean) u |= S32_U_CLEAN;
      um[(size_t)iz * P + ir] = u;
    }
  t->fEr = (float)(dti / (mu0 * eps0 * dz));
  t->topf = (float)((m->rmax - dr / 2) / (m->rmax + dr / 2));
  t->fEphi = (float)(dti * factor);
  cudaError_t e = cudaSuccess;
  if (!t->cpd) {
    e = cudaMalloc(&t->cpd, sizeof(float) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&t->cmd, sizeof(float) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&t->bzf, sizeof(float) * (nr + 1));
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->cpd, cpd.data(), sizeof(float) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->cmd, cmd.data(), sizeof(float) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->bzf, bzf.data(), sizeof(float) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_umask, um.data(), um.size(), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s); // the host vectors go out of scope
  t->fused = -1; // planned again for this mesh at the next step
  return (int)e;
}

extern "C" void s32_fdtd_tables_free(Fdtd32Tables *t)
{
  cudaFree(t->cpd);
  cudaFree(t->cmd);
  cudaFree(t->bzf);
  cudaFree(t->pub);
  cudaFree(t->flag);
  cudaFree(t->arrivals);
  *t = Fdtd32Tables();
}

// Whether this mesh takes the fused TM kernel, and its bands: one block per
// band, as many bands as blocks fit on the device at once (a cooperative
// launch), at least 4 rows each.  Meshes below 2^18 nodes keep the two
// kernels (their launch is not bandwidth-bound); so do rows wider than
// 4096 columns (a block holds four columns per thread).
static int fused_plan(const DevMesh *m, Fdtd32Tables *t)
{
  t->fused = 0;
  const int P = m->pitch;
  if (t->mode == SPIFFE_FDTD_TWO_KERNELS || m->nr < 8 || m->nz < 8 || P > 4096 || P % 32)
    return 0;
  if (t->mode == SPIFFE_FDTD_AUTO && (!FUSED_BY_DEFAULT || (long long)(m->nz + 1) * (m->nr + 1) < (1LL << 18)))
    return 0;
  t->smem = fused_smem(P);
  t->threads = ((P / 4 + 31) / 32) * 32;
  cudaError_t e = cudaFuncSetAttribute(k_tm_fused32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t->smem);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int per = 0, dev = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tm_fused32, t->threads, t->smem) != cudaSuccess ||
      cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || per < 1) {
    cudaGetLastError();
    return 0;
  }
  const int rows = m->nz; // E rows 0..nz-1
  int bands = per * sms;
  if (bands > rows / 4)
    bands = rows / 4;
  t->rows_per = (rows + bands - 1) / bands;
  t->bands = (rows + t->rows_per - 1) / t->rows_per;
  // (a new plan follows a new mesh: the buffers are made again for it; the
  // flags start at 0 below every epoch still to come)
  cudaFree(t->pub);
  cudaFree(t->flag);
  cudaFree(t->arrivals);
  t->pub = nullptr;
  t->flag = t->arrivals = nullptr;
  e = cudaMalloc(&t->pub, sizeof(float) * (size_t)t->bands * P);
  if (e == cudaSuccess) e = cudaMalloc(&t->flag, sizeof(unsigned) * t->bands);
  if (e == cudaSuccess) e = cudaMemset(t->flag, 0, sizeof(unsigned) * t->bands);
  if (e == cudaSuccess) e = cudaMalloc(&t->arrivals, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(t->arrivals, 0, sizeof(unsigned));
  if (e != cudaSuccess)
    return (int)e;
  t->epoch = 0;
  t->fused = 1;
  return 0;
}

extern "C" int s32_fdtd_step(const DevMesh *m, const DevFields32 *f, Fdtd32Tables *t, float kJ, int zero_j,
                             unsigned *err, cudaStream_t s)
{
  const double dt = m->dt;
  Coef32 c{t->cpd, t->cmd, t->bzf, t->fEr, t->topf, (float)(t->fEphi / m->dz), (float)(t->fEphi / m->dr),
           (float)(dt / m->dz), (float)(dt / m->dr), kJ, zero_j};
  const dim3 block(BX, BY), grid = grid_for(m, m->nr + 1);
  if (t->fused < 0) {
    const int rc = fused_plan(m, t);
    if (rc)
      return rc;
  }
  if ((m->modes & SPIFFE_FL_TM_FIELDS) && t->fused == 1) {
    c.reset_box = zero_j && !(m->modes & SPIFFE_FL_TE_FIELDS);
    FusedArgs a{t->pub, t->flag, t->arrivals, err, t->rows_per, t->bands, ++t->epoch};
    DevMesh mm = *m;
    DevFields32 ff = *f;
    void *args[] = {&mm, &ff, &c, &a};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_tm_fused32, dim3(t->bands), dim3(t->threads), args,
                                                t->smem, s);
    if (e != cudaSuccess)
      return (int)e;
    spiffe_note_launches(1);
  } else if (m->modes & SPIFFE_FL_TM_FIELDS) {
    c.reset_box = zero_j && !(m->modes & SPIFFE_FL_TE_FIELDS);
    const TmSplit te = tm_split(m->nz, m->nr, false), tb = tm_split(m->nz, m->nr, true);
    const int per = VX * VY;
    const dim3 vblock(VX, VY);
    k_tm_e32<<<te.tiles + (unsigned)((te.nb + per - 1) / per), vblock, 0, s>>>(*m, *f, c, te);
    k_tm_b32<<<tb.tiles + (unsigned)((tb.nb + per - 1) / per), vblock, 0, s>>>(*m, *f, c, tb);
    spiffe_note_launches(2);
  }
  if (m->modes & SPIFFE_FL_TE_FIELDS) {
    c.reset_box = zero_j;
    k_te_e32<<<grid, block, 0, s>>>(*m, *f, c);
    k_te_b32<<<grid, block, 0, s>>>(*m, *f, c);
    spiffe_note_launches(2);
  }
  return (int)cudaGetLastError();
}

extern "C" int s32_to_f32(const DevMesh *m, const double *d_staging, float *dst, cudaStream_t s)
{
  k_to_f32<<<grid_for(m, m->pitch), dim3(BX, BY), 0, s>>>(m->nz, m->nr, m->pitch, d_staging, dst);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_from_f32(const DevMesh *m, const float *src, double *d_staging, cudaStream_t s)
{
  k_from_f32<<<grid_for(m, m->nr + 1), dim3(BX, BY), 0, s>>>(m->nz, m->nr, m->pitch, src, d_staging);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_to_f64p(const DevMesh *m, const double *d_staging, double *dst, cudaStream_t s)
{
  k_to_f64p<<<grid_for(m, m->pitch), dim3(BX, BY), 0, s>>>(m->nz, m->nr, m->pitch, d_staging, dst);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_from_f64p(const DevMesh *m, const double *src, double *d_staging, cudaStream_t s)
{
  k_from_f64p<<<grid_for(m, m->nr + 1), dim3(BX, BY), 0, s>>>(m->nz, m->nr, m->pitch, src, d_staging);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_to_fixed(const DevMesh *m, const double *d_staging, long long *dst, double quantum, cudaStream_t s)
{
  k_to_fixed<<<grid_for(m, m->pitch), dim3(BX, BY), 0, s>>>(m->nz, m->nr, m->pitch, d_staging, dst, 1 / quantum);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_from_fixed(const DevMesh *m, const long long *src, double *d_staging, double quantum, cudaStream_t s)
{
  k_from_fixed<<<grid_for(m, m->nr + 1), dim3(BX, BY), 0, s>>>(m->nz, m->nr, m->pitch, src, d_staging, quantum);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_antenna(long long *J, int *jbox, int pitch, int direction, long istart, long iend,
                           long iposition, double value, double qJ, cudaStream_t s)
{
  if (iend < istart)
    return 0;
  const long n = iend - istart + 1;
  k_antenna32<<<blocks_for(n, 128), 128, 0, s>>>(J, jbox, pitch, direction, istart, iend, iposition,
                                                  (long long)std::llround(value / qJ));
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_jbox_set(int *jbox, int lo, int hi, cudaStream_t s)
{
  k_jbox_set<<<1, 1, 0, s>>>(jbox, lo, hi);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}

extern "C" int s32_rescale_fixed(long long *a, size_t n, int shift, cudaStream_t s)
{
  if (!a || shift <= 0 || n == 0)
    return 0;
  k_rescale_fixed<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, n, shift);
  spiffe_note_launches(1);
  return (int)cudaGetLastError();
}
