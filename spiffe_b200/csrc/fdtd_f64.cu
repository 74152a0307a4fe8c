// spiffe_b200/csrc/fdtd_f64.cu -- plain FP64 Yee update (bit-faithful form).
//
// Restates advance_field_solutions (integrate.c:277-541) as data-parallel
// kernels.  The reference updates each field serially and then applies its
// boundary copies; here every mesh node has exactly one writer thread that
// computes the node's final value directly (interior update, or the boundary
// copy of its neighbour's updated value), so no node is read after another
// thread wrote it within a kernel.  The serial "stop the row at the first
// FL_LAST_ACTIVE_PT" rule (integrate.c:345-346) becomes a per-row cut-off
// index computed once on the host.  Built with -fmad=false so every product
// and sum rounds as the reference's does.
#include "modules.cuh"

namespace {

struct Coef64 {
  const double *cpz, *cmz; // Ez metric coefficients per row, integrate.c:327-340
  const double *bzf;       // Bz factor per row, integrate.c:515
  const int *cut0, *cut1;  // last updated iz per row for loops starting at 0 / 1
  double fEr;              // 1/(mu0 eps0 dz), integrate.c:362
  double topf;             // (rmax-dr/2)/(rmax+dr/2), integrate.c:384
  double fEphi;            // 1/(eps0 mu0), integrate.c:450
};

constexpr int BX = 32, BY = 8;

// Ez and Er to their final values for this step (integrate.c:323-380).
__global__ void __launch_bounds__(BX *BY) k_tm_e(DevMesh m, DevFields<double> f, Coef64 c)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (ir > nr || iz > nz)
    return;
  const double eps0 = SPIFFE_EPSILON_O, dti = m.dt;
  const size_t i = node(iz, ir, P);
  const int16_t fl = f.flags[i];
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;

  // Ez: rows ir < nr, interior 1 <= iz <= nz-1; row nr-1 ends at zero
  if (ir < nr && iz >= 1 && iz <= nz - 1) {
    double v;
    if (ir == nr - 1) {
      v = 0.0;
    } else {
      v = f.Ez[i];
      if (iz <= c.cut1[ir] && !(fl & SPIFFE_FL_EZ_ZERO))
        v += dti * (-f.Jz[i] / eps0 + (c.cpz[ir] * f.Bphi[i + 1] - c.cmz[ir] * f.Bphi[i]));
    }
    f.Ez[i] = v;
    if (iz == 1)
      f.Ez[node(0, ir, P)] = ir == nr - 1 ? 0.0 : (leftN ? v : -v);
    if (iz == nz - 1)
      f.Ez[node(nz, ir, P)] = ir == nr - 1 ? 0.0 : (rightN ? v : -v);
  }

  // Er: rows 1 <= ir <= nr-1, 0 <= iz <= nz-1; axis mirror; Neumann end rows
  if (iz <= nz - 1) {
    const bool zero_row = (leftN && iz == 0) || (rightN && iz == nz - 1);
    if (ir >= 1 && ir <= nr - 1) {
      double v = f.Er[i];
      if (iz <= c.cut0[ir] && !(fl & SPIFFE_FL_ER_ZERO))
        v += dti * (-f.Jr[i] / eps0 - c.fEr * (f.Bphi[i + P] - f.Bphi[i]));
      f.Er[i] = zero_row ? 0.0 : v;
      if (ir == 1)
        f.Er[node(iz, 0, P)] = zero_row ? 0.0 : -v;
    } else if (ir == nr && zero_row) {
      f.Er[i] = 0.0;
    }
  }
}

// Bphi and Bphi2 (integrate.c:383-432), reading the final Ez and Er.
__global__ void __launch_bounds__(BX *BY) k_tm_b(DevMesh m, DevFields<double> f, Coef64 c)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (ir > nr || iz < 1 || iz > nz - 1)
    return;
  const double dti = m.dt, dr = m.dr, dz = m.dz;
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;
  const size_t i = node(iz, ir, P);
  if (ir >= 1 && ir <= nr - 2) {
    double b = f.Bphi[i], b2 = f.Bphi2[i];
    if (iz <= c.cut1[ir] && !(f.flags[i] & SPIFFE_FL_BPHI_ZERO)) {
      const double dB = dti * ((f.Ez[i] - f.Ez[i - 1]) / dr - (f.Er[i] - f.Er[i - P]) / dz);
      b2 = b + dB / 2;
      b += dB;
      f.Bphi2[i] = b2;
      f.Bphi[i] = b;
    }
    // axis and top copies of this row
    if (ir == 1) {
      f.Bphi[node(iz, 0, P)] = -b;
      f.Bphi2[node(iz, 0, P)] = -b2;
    }
    if (ir == nr - 2) {
      f.Bphi[node(iz, nr - 1, P)] = b * c.topf;
      f.Bphi2[node(iz, nr - 1, P)] = b2 * c.topf;
    }
    // end rows copy row 1 / row nz-1 after its axis and top copies
    if (iz == 1 || iz == nz - 1) {
      const int row = iz == 1 ? 0 : nz;
      const bool neu = iz == 1 ? leftN : rightN;
      f.Bphi[node(row, ir, P)] = neu ? b : -b;
      f.Bphi2[node(row, ir, P)] = neu ? b2 : -b2;
      if (ir == 1) {
        f.Bphi[node(row, 0, P)] = neu ? -b : b;
        f.Bphi2[node(row, 0, P)] = neu ? -b2 : b2;
      }
      if (ir == nr - 2) {
        const double t = b * c.topf, t2 = b2 * c.topf;
        f.Bphi[node(row, nr - 1, P)] = neu ? t : -t;
        f.Bphi2[node(row, nr - 1, P)] = neu ? t2 : -t2;
      }
      if (iz == 1 && iz == nz - 1) { // nz == 2: row 1 also feeds row nz
        f.Bphi[node(nz, ir, P)] = rightN ? b : -b;
        f.Bphi2[node(nz, ir, P)] = rightN ? b2 : -b2;
      }
    }
  } else if (ir == nr) {
    // column nr is never updated; the end rows still copy it
    if (iz == 1) {
      f.Bphi[node(0, nr, P)] = leftN ? f.Bphi[i] : -f.Bphi[i];
      f.Bphi2[node(0, nr, P)] = leftN ? f.Bphi2[i] : -f.Bphi2[i];
    }
    if (iz == nz - 1) {
      f.Bphi[node(nz, nr, P)] = rightN ? f.Bphi[i] : -f.Bphi[i];
      f.Bphi2[node(nz, nr, P)] = rightN ? f.Bphi2[i] : -f.Bphi2[i];
    }
  }
}

// Ephi (integrate.c:449-471): interior update, then zero on the axis, on
// Neumann end rows and on the Neumann top row.
__global__ void __launch_bounds__(BX *BY) k_te_e(DevMesh m, DevFields<double> f, Coef64 c)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (ir > nr || iz > nz)
    return;
  const double eps0 = SPIFFE_EPSILON_O, dti = m.dt, dz = m.dz, dr = m.dr;
  const size_t i = node(iz, ir, P);
  const bool zero = ir == 0 || (m.right_bc == SPIFFE_NEUMANN && iz == nz - 1) ||
                    (m.left_bc == SPIFFE_NEUMANN && iz == 0) || (m.upper_bc == SPIFFE_NEUMANN && ir == nr - 1);
  if (zero) {
    f.Ephi[i] = 0.0;
    return;
  }
  if (ir >= 1 && ir <= nr - 1 && iz <= nz - 1 && iz <= c.cut0[ir] && !(f.flags[i] & SPIFFE_FL_EPHI_ZERO))
    f.Ephi[i] += dti * (-f.Jphi[i] / eps0 + c.fEphi * ((f.Br[i + P] - f.Br[i]) / dz - (f.Bz[i + 1] - f.Bz[i]) / dr));
}

// Br/Br2 and Bz/Bz2 (integrate.c:473-539), reading the final Ephi.
__global__ void __launch_bounds__(BX *BY) k_te_b(DevMesh m, DevFields<double> f, Coef64 c)
{
  const int ir = blockIdx.x * BX + threadIdx.x, iz = blockIdx.y * BY + threadIdx.y;
  const int nz = m.nz, nr = m.nr, P = m.pitch;
  if (ir > nr || iz > nz)
    return;
  const double dti = m.dt, dz = m.dz;
  const bool leftN = m.left_bc == SPIFFE_NEUMANN, rightN = m.right_bc == SPIFFE_NEUMANN;
  const size_t i = node(iz, ir, P);

  // Br: rows 0 <= ir <= nr-1, interior 1 <= iz <= nz-1; end rows mirror
  if (iz >= 1 && iz <= nz - 1) {
    double b = f.Br[i], b2 = f.Br2[i];
    if (ir <= nr - 1 && iz <= c.cut1[ir] && !(f.flags[i] & SPIFFE_FL_BR_ZERO)) {
      const double dB = dti * (f.Ephi[i] - f.Ephi[i - P]) / dz;
      b2 = b + dB / 2;
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

  // Bz: rows 1 <= ir <= nr-1, 0 <= iz <= nz-1; axis copy; Neumann end rows
  const bool zero_row = (rightN && iz == nz - 1) || (leftN && iz == 0);
  if (ir >= 1 && ir <= nr - 1 && iz <= nz) {
    double b = f.Bz[i], b2 = f.Bz2[i];
    if (iz <= nz - 1 && iz <= c.cut0[ir] && !(f.flags[i] & SPIFFE_FL_BZ_ZERO)) {
      const double dB = c.bzf[ir] * ((ir + 1) * f.Ephi[i] - ir * f.Ephi[i - 1]);
      b2 = b + dB / 2;
      b += dB;
    }
    f.Bz[i] = zero_row ? 0.0 : b;
    f.Bz2[i] = zero_row ? 0.0 : b2;
    if (ir == 1) {
      f.Bz[node(iz, 0, P)] = zero_row ? 0.0 : b;
      f.Bz2[node(iz, 0, P)] = zero_row ? 0.0 : b2;
    }
  } else if (ir == nr && zero_row) {
    f.Bz[i] = 0.0;
    f.Bz2[i] = 0.0;
  }
}

} // namespace

// Host-side coefficient tables, computed with the reference's expressions.

extern "C" int spiffe_fdtd64_tables(const DevMesh *m, const int16_t *host_flags, Fdtd64Tables *t, cudaStream_t s)
{
  const int nz = m->nz, nr = m->nr;
  const double eps0 = SPIFFE_EPSILON_O, mu0 = SPIFFE_MU_O, dr = m->dr, dz = m->dz, dti = m->dt;
  double *cpz = new double[nr + 1], *cmz = new double[nr + 1], *bzf = new double[nr + 1];
  int *cut0 = new int[nr + 1], *cut1 = new int[nr + 1];
  const double factor = 1 / (eps0 * mu0);
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
    cpz[ir] = cp;
    cmz[ir] = cm;
    bzf[ir] = ir >= 1 ? -2 * dti / (dr * (double)((long)(ir + 1) * (ir + 1) - (long)ir * ir)) : 0.0;
    // the serial loops stop after the first node flagged FL_LAST_ACTIVE_PT
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
  t->fEr = 1 / (mu0 * eps0 * dz);
  t->topf = (m->rmax - m->dr / 2) / (m->rmax + m->dr / 2);
  t->fEphi = 1. / (eps0 * mu0);
  cudaError_t e = cudaSuccess;
  if (!t->cpz) {
    e = cudaMalloc(&t->cpz, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&t->cmz, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&t->bzf, sizeof(double) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&t->cut0, sizeof(int) * (nr + 1));
    if (e == cudaSuccess) e = cudaMalloc(&t->cut1, sizeof(int) * (nr + 1));
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->cpz, cpz, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->cmz, cmz, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->bzf, bzf, sizeof(double) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->cut0, cut0, sizeof(int) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(t->cut1, cut1, sizeof(int) * (nr + 1), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  delete[] cpz;
  delete[] cmz;
  delete[] bzf;
  delete[] cut0;
  delete[] cut1;
  return (int)e;
}

extern "C" void spiffe_fdtd64_tables_free(Fdtd64Tables *t)
{
  cudaFree(t->cpz);
  cudaFree(t->cmz);
  cudaFree(t->bzf);
  cudaFree(t->cut0);
  cudaFree(t->cut1);
  *t = Fdtd64Tables();
}

// One advance_field_solutions: TM (E then B), then TE (Ephi then B).
extern "C" int spiffe_fdtd64_step(const DevMesh *m, const DevFields<double> *f, const Fdtd64Tables *t, cudaStream_t s)
{
  Coef64 c{t->cpz, t->cmz, t->bzf, t->cut0, t->cut1, t->fEr, t->topf, t->fEphi};
  dim3 block(BX, BY), grid((m->nr + 1 + BX - 1) / BX, (m->nz + 1 + BY - 1) / BY);
  if (m->modes & SPIFFE_FL_TM_FIELDS) {
    k_tm_e<<<grid, block, 0, s>>>(*m, *f, c);
    spiffe_note_launches(1);
    k_tm_b<<<grid, block, 0, s>>>(*m, *f, c);
    spiffe_note_launches(1);
  }
  if (m->modes & SPIFFE_FL_TE_FIELDS) {
    k_te_e<<<grid, block, 0, s>>>(*m, *f, c);
    spiffe_note_launches(1);
    k_te_b<<<grid, block, 0, s>>>(*m, *f, c);
    spiffe_note_launches(1);
  }
  return (int)cudaGetLastError();
}
