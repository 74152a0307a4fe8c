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
        v += c.kJ * (float)jz + (cp * b1 - cm * b0);
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
        v += c.kJ * (float)jr - c.fEr * (bP - b0);
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
      const float dB = c.dt_dr * (ez - ezm) - c.dt_dz * (er - erm);
      b2 = b + 0.5f * dB;
      b += dB;
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
  if (u.x & S32_U_EZ) ez.x += c.kJ * jz0 + (cp.x * b0.y - cm.x * b0.x);
  if (u.y & S32_U_EZ) ez.y += c.kJ * jz1 + (cp.y * b0.z - cm.y * b0.y);
  if (u.z & S32_U_EZ) ez.z += c.kJ * jz2 + (cp.z * b0.w - cm.z * b0.z);
  if (u.w & S32_U_EZ) ez.w += c.kJ * jz3 + (cp.w * bnext - cm.w * b0.w);
  if (u.x & S32_U_ER) er.x += c.kJ * jr0 - c.fEr * (bP.x - b0.x);
  if (u.y & S32_U_ER) er.y += c.kJ * jr1 - c.fEr * (bP.y - b0.y);
  if (u.z & S32_U_ER) er.z += c.kJ * jr2 - c.fEr * (bP.z - b0.z);
  if (u.w & S32_U_ER) er.w += c.kJ * jr3 - c.fEr * (bP.w - b0.w);
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
  const float dBx = c.dt_dr * (ez.x - eprev) - c.dt_dz * (er.x - erm.x);
  const float dBy = c.dt_dr * (ez.y - ez.x) - c.dt_dz * (er.y - erm.y);
  const float dBz = c.dt_dr * (ez.z - ez.y) - c.dt_dz * (er.z - erm.z);
  const float dBw = c.dt_dr * (ez.w - ez.z) - c.dt_dz * (er.w - erm.w);
  const bool ux = u.x & S32_U_BPHI, uy = u.y & S32_U_BPHI, uz = u.z & S32_U_BPHI, uw = u.w & S32_U_BPHI;
  float4 b2;
  b2.x = b.x + 0.5f * dBx;
  b2.y = b.y + 0.5f * dBy;
  b2.z = b.z + 0.5f * dBz;
  b2.w = b.w + 0.5f * dBw;
  if (ux && uy && uz && uw) {
    b.x += dBx;
    b.y += dBy;
    b.z += dBz;
    b.w += dBw;
    st4(f.Bphi2 + i, b2);
    st4(f.Bphi + i, b);
  } else {
    // a node that is not updated keeps both of its values (next to metal)
    if (ux) { f.Bphi2[i] = b2.x; f.Bphi[i] = b.x + dBx; }
    if (uy) { f.Bphi2[i + 1] = b2.y; f.Bphi[i + 1] = b.y + dBy; }
    if (uz) { f.Bphi2[i + 2] = b2.z; f.Bphi[i + 2] = b.z + dBz; }
    if (uw) { f.Bphi2[i + 3] = b2.w; f.Bphi[i + 3] = b.w + dBw; }
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
  return (int)e;
}

extern "C" void s32_fdtd_tables_free(Fdtd32Tables *t)
{
  cudaFree(t->cpd);
  cudaFree(t->cmd);
  cudaFree(t->bzf);
  *t = Fdtd32Tables();
}

extern "C" int s32_fdtd_step(const DevMesh *m, const DevFields32 *f, const Fdtd32Tables *t, float kJ, int zero_j,
                             cudaStream_t s)
{
  const double dt = m->dt;
  Coef32 c{t->cpd, t->cmd, t->bzf, t->fEr, t->topf, (float)(t->fEphi / m->dz), (float)(t->fEphi / m->dr),
           (float)(dt / m->dz), (float)(dt / m->dr), kJ, zero_j};
  const dim3 block(BX, BY), grid = grid_for(m, m->nr + 1);
  if (m->modes & SPIFFE_FL_TM_FIELDS) {
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
