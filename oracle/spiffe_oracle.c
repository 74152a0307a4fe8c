/* oracle/spiffe_oracle.c -- TEST INFRASTRUCTURE: the CPU oracle.
 *
 * A plain-C, FP64 restatement of the reference spiffe per-timestep PIC path,
 * used only by the tests, by the smoke check and by the benchmark's CPU
 * baseline leg as the checker.  It is never linked into, or called by, the
 * product library.  Each function names the reference file:line it restates;
 * arithmetic is written in the reference's expression order and this file is
 * compiled with -ffp-contract=off so results are bit-identical to the
 * reference built the same way (checked against oracle/_ref and the golden
 * fixtures in tests/golden/).
 *
 * Arrays are the contiguous (nz+1) x (nr+1) blocks of spiffe_b200_types.h,
 * indexed [iz*(nr+1)+ir].
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/spiffe_b200_constants.h"
#include "../include/spiffe_b200_types.h"

#define C_MKS SPIFFE_C_MKS
#define EPS0 SPIFFE_EPSILON_O
#define MU0 SPIFFE_MU_O
#define PI SPIFFE_PI
#define PIx2 SPIFFE_PIx2

#define IDX(iz, ir) ((size_t)(iz) * (size_t)(nr + 1) + (size_t)(ir))

static double sq(double x) { return x * x; }

/* ------------------------------------------------------------- currents */

/* zero_current_arrays, integrate.c:210-241 */
void orc_zero_currents(const spiffe_mesh *m, spiffe_field_set *f)
{
  size_t n = (size_t)(m->nz + 1) * (size_t)(m->nr + 1);
  if (m->modes & SPIFFE_FL_TM_FIELDS) {
    memset(f->Jz, 0, n * sizeof(double));
    memset(f->Jr, 0, n * sizeof(double));
  }
  if (m->modes & SPIFFE_FL_TE_FIELDS)
    memset(f->Jphi, 0, n * sizeof(double));
}

/* ----------------------------------------------------------------- FDTD */

/* advance_field_solutions, integrate.c:277-541.  Rows stop at the first node
 * flagged FL_LAST_ACTIVE_PT (:345-346); boundary copies follow each update in
 * the reference's order. */
void orc_advance_fields(const spiffe_mesh *m, spiffe_field_set *f)
{
  const long nz = m->nz, nr = m->nr;
  const double dr = m->dr, dz = m->dz, dti = m->dt;
  const double eps0 = EPS0, mu0 = MU0;
  const int16_t *fl = f->flags;
  long iz, ir;
  double rp, rm, factor, cp, cm, dB;

  if (m->modes & SPIFFE_FL_TM_FIELDS) {
    double *Ez = f->Ez, *Er = f->Er, *Bphi = f->Bphi, *Bphi2 = f->Bphi2, *Jz = f->Jz, *Jr = f->Jr;
    /* Ez, integrate.c:323-359 */
    factor = 1 / (eps0 * mu0);
    for (ir = 0; ir < nr; ir++) {
      rp = (ir + 0.5) * dr;
      rm = (ir - 0.5) * dr;
      if (ir != 0) {
        cp = 2 * factor / (sq(rp) - sq(rm));
        cm = rm * cp;
        cp = rp * cp;
      } else {
        cp = 4 * factor / dr;
        cm = 0;
      }
      for (iz = 1; iz < nz; iz++) {
        if (!(fl[IDX(iz, ir)] & SPIFFE_FL_EZ_ZERO))
          Ez[IDX(iz, ir)] += dti * (-Jz[IDX(iz, ir)] / eps0 + (cp * Bphi[IDX(iz, ir + 1)] - cm * Bphi[IDX(iz, ir)]));
        if (fl[IDX(iz, ir)] & SPIFFE_FL_LAST_ACTIVE_PT)
          break;
      }
      Ez[IDX(0, ir)] = m->left_bc == SPIFFE_NEUMANN ? Ez[IDX(1, ir)] : -Ez[IDX(1, ir)];
      Ez[IDX(nz, ir)] = m->right_bc == SPIFFE_NEUMANN ? Ez[IDX(nz - 1, ir)] : -Ez[IDX(nz - 1, ir)];
    }
    for (iz = 0; iz <= nz; iz++)
      Ez[IDX(iz, nr - 1)] = 0;

    /* Er, integrate.c:361-380 */
    factor = 1 / (mu0 * eps0 * dz);
    for (ir = 1; ir < nr; ir++) {
      for (iz = 0; iz < nz; iz++) {
        if (!(fl[IDX(iz, ir)] & SPIFFE_FL_ER_ZERO))
          Er[IDX(iz, ir)] += dti * (-Jr[IDX(iz, ir)] / eps0 - factor * (Bphi[IDX(iz + 1, ir)] - Bphi[IDX(iz, ir)]));
        if (fl[IDX(iz, ir)] & SPIFFE_FL_LAST_ACTIVE_PT)
          break;
      }
    }
    for (iz = 0; iz < nz; iz++)
      Er[IDX(iz, 0)] = -Er[IDX(iz, 1)];
    if (m->left_bc == SPIFFE_NEUMANN)
      for (ir = 0; ir <= nr; ir++)
        Er[IDX(0, ir)] = 0;
    if (m->right_bc == SPIFFE_NEUMANN)
      for (ir = 0; ir <= nr; ir++)
        Er[IDX(nz - 1, ir)] = 0;

    /* Bphi and Bphi2, integrate.c:383-432 */
    factor = (m->rmax - m->dr / 2) / (m->rmax + m->dr / 2);
    for (ir = 1; ir < nr; ir++) {
      for (iz = 1; iz < nz; iz++) {
        if (!(fl[IDX(iz, ir)] & SPIFFE_FL_BPHI_ZERO)) {
          dB = dti * ((Ez[IDX(iz, ir)] - Ez[IDX(iz, ir - 1)]) / dr - (Er[IDX(iz, ir)] - Er[IDX(iz - 1, ir)]) / dz);
          Bphi2[IDX(iz, ir)] = Bphi[IDX(iz, ir)] + dB / 2;
          Bphi[IDX(iz, ir)] += dB;
        }
        if (fl[IDX(iz, ir)] & SPIFFE_FL_LAST_ACTIVE_PT)
          break;
      }
    }
    for (iz = 1; iz < nz; iz++) {
      Bphi[IDX(iz, 0)] = -Bphi[IDX(iz, 1)];
      Bphi2[IDX(iz, 0)] = -Bphi2[IDX(iz, 1)];
      Bphi[IDX(iz, nr - 1)] = Bphi[IDX(iz, nr - 2)] * factor;
      Bphi2[IDX(iz, nr - 1)] = Bphi2[IDX(iz, nr - 2)] * factor;
    }
    for (ir = 0; ir <= nr; ir++) {
      if (m->left_bc == SPIFFE_NEUMANN) {
        Bphi[IDX(0, ir)] = Bphi[IDX(1, ir)];
        Bphi2[IDX(0, ir)] = Bphi2[IDX(1, ir)];
      } else {
        Bphi[IDX(0, ir)] = -Bphi[IDX(1, ir)];
        Bphi2[IDX(0, ir)] = -Bphi2[IDX(1, ir)];
      }
    }
    for (ir = 0; ir <= nr; ir++) {
      if (m->right_bc == SPIFFE_NEUMANN) {
        Bphi[IDX(nz, ir)] = Bphi[IDX(nz - 1, ir)];
        Bphi2[IDX(nz, ir)] = Bphi2[IDX(nz - 1, ir)];
      } else {
        Bphi[IDX(nz, ir)] = -Bphi[IDX(nz - 1, ir)];
        Bphi2[IDX(nz, ir)] = -Bphi2[IDX(nz - 1, ir)];
      }
    }
  }

  if (m->modes & SPIFFE_FL_TE_FIELDS) {
    double *Ephi = f->Ephi, *Jphi = f->Jphi, *Br = f->Br, *Br2 = f->Br2, *Bz = f->Bz, *Bz2 = f->Bz2;
    /* Ephi, integrate.c:449-471 */
    factor = 1. / (eps0 * mu0);
    for (ir = 1; ir < nr; ir++)
      for (iz = 0; iz < nz; iz++) {
        if (!(fl[IDX(iz, ir)] & SPIFFE_FL_EPHI_ZERO))
          Ephi[IDX(iz, ir)] += dti * (-Jphi[IDX(iz, ir)] / eps0 +
                                      factor * ((Br[IDX(iz + 1, ir)] - Br[IDX(iz, ir)]) / dz - (Bz[IDX(iz, ir + 1)] - Bz[IDX(iz, ir)]) / dr));
        if (fl[IDX(iz, ir)] & SPIFFE_FL_LAST_ACTIVE_PT)
          break;
      }
    for (iz = 0; iz <= nz; iz++)
      Ephi[IDX(iz, 0)] = 0;
    if (m->right_bc == SPIFFE_NEUMANN)
      for (ir = 0; ir <= nr; ir++)
        Ephi[IDX(nz - 1, ir)] = 0;
    if (m->left_bc == SPIFFE_NEUMANN)
      for (ir = 0; ir <= nr; ir++)
        Ephi[IDX(0, ir)] = 0;
    if (m->upper_bc == SPIFFE_NEUMANN)
      for (iz = 0; iz <= nz; iz++)
        Ephi[IDX(iz, nr - 1)] = 0;

    /* Br and Br2, integrate.c:473-509 */
    for (ir = 0; ir < nr; ir++)
      for (iz = 1; iz < nz; iz++) {
        if (!(fl[IDX(iz, ir)] & SPIFFE_FL_BR_ZERO)) {
          dB = dti * (Ephi[IDX(iz, ir)] - Ephi[IDX(iz - 1, ir)]) / dz;
          Br2[IDX(iz, ir)] = Br[IDX(iz, ir)] + dB / 2;
          Br[IDX(iz, ir)] += dB;
        }
        if (fl[IDX(iz, ir)] & SPIFFE_FL_LAST_ACTIVE_PT)
          break;
      }
    for (ir = 0; ir <= nr; ir++) {
      if (m->right_bc == SPIFFE_NEUMANN) {
        Br[IDX(nz, ir)] = Br[IDX(nz - 1, ir)];
        Br2[IDX(nz, ir)] = Br2[IDX(nz - 1, ir)];
      } else {
        Br[IDX(nz, ir)] = -Br[IDX(nz - 1, ir)];
        Br2[IDX(nz, ir)] = -Br2[IDX(nz - 1, ir)];
      }
    }
    for (ir = 0; ir <= nr; ir++) {
      if (m->left_bc == SPIFFE_NEUMANN) {
        Br[IDX(0, ir)] = Br[IDX(1, ir)];
        Br2[IDX(0, ir)] = Br2[IDX(1, ir)];
      } else {
        Br[IDX(0, ir)] = -Br[IDX(1, ir)];
        Br2[IDX(0, ir)] = -Br2[IDX(1, ir)];
      }
    }

    /* Bz and Bz2, integrate.c:511-539 */
    for (ir = 1; ir < nr; ir++) {
      factor = -2 * dti / (dr * ((ir + 1) * (ir + 1) - ir * ir));
      for (iz = 0; iz < nz; iz++) {
        if (!(fl[IDX(iz, ir)] & SPIFFE_FL_BZ_ZERO)) {
          dB = factor * ((ir + 1) * Ephi[IDX(iz, ir)] - ir * Ephi[IDX(iz, ir - 1)]);
          Bz2[IDX(iz, ir)] = Bz[IDX(iz, ir)] + dB / 2;
          Bz[IDX(iz, ir)] += dB;
        }
        if (fl[IDX(iz, ir)] & SPIFFE_FL_LAST_ACTIVE_PT)
          break;
      }
    }
    for (iz = 0; iz <= nz; iz++) {
      Bz[IDX(iz, 0)] = Bz[IDX(iz, 1)];
      Bz2[IDX(iz, 0)] = Bz2[IDX(iz, 1)];
    }
    if (m->right_bc == SPIFFE_NEUMANN)
      for (ir = 0; ir <= nr; ir++)
        Bz[IDX(nz - 1, ir)] = Bz2[IDX(nz - 1, ir)] = 0;
    if (m->left_bc == SPIFFE_NEUMANN)
      for (ir = 0; ir <= nr; ir++)
        Bz[IDX(0, ir)] = Bz2[IDX(0, ir)] = 0;
  }
}

/* ----------------------------------------------------------- deposition */

/* add_particle_currents, space_charge.c:34-295: NGP or area-weighted
 * deposition of Q*v over annulus volume factors, at the particles' current
 * (old) positions and velocities, in particle order. */
void orc_deposit(const spiffe_mesh *m, spiffe_field_set *f, const spiffe_beam_set *b)
{
  const long nz = m->nz, nr = m->nr;
  const double dz = m->dz, dr = m->dr, zmin = m->zmin;
  const double one_over_piDzDr2 = 1 / (PI * dz * sq(dr));
  const int rsm = (m->modes & SPIFFE_FL_RADIAL_SMEAR) != 0, lsm = (m->modes & SPIFFE_FL_LONGIT_SMEAR) != 0;
  long ip, iz, ir;
  double fp, fm, Jm, Jp, QoV, QVG;

  if (m->modes & SPIFFE_FL_TM_FIELDS) {
    double *Jz = f->Jz, *Jr = f->Jr;
    /* Jz, space_charge.c:60-139 */
    for (ip = 0; ip < b->np; ip++) {
      if (!(b->status[ip] & SPIFFE_PART_ACTIVE))
        continue;
      ir = rsm ? (long)(b->r[ip] / dr) : (long)(b->r[ip] / dr + 0.5);
      iz = lsm ? (long)((b->z[ip] - zmin) / dz + 0.5) : (long)((b->z[ip] - zmin) / dz + 1.0);
      if (iz < 0 || iz > nz)
        continue;
      if (ir < 0 || ir > nr)
        continue;
      QoV = b->Q[ip] * one_over_piDzDr2;
      QVG = b->vz[ip] * QoV;
      if (rsm)
        fm = 1 - (fp = b->r[ip] / dr - ir);
      else {
        fm = 1;
        fp = 0;
      }
      if (ir == 0) {
        Jm = 4 * fm * QVG;
        Jp = fp * QVG / (sq(1.5) - sq(0.5));
      } else if (ir < nr - 1) {
        Jm = fm * QVG / (sq(ir + 0.5) - sq(ir - 0.5));
        Jp = fp * QVG / (sq(ir + 1.5) - sq(ir + 0.5));
      } else {
        Jm = 0;
        Jp = fp * QVG / (sq(ir + 0.5) - sq(ir - 0.5));
        ir--;
      }
      if (lsm) {
        if (iz == 0) {
          fp = 1;
          fm = 0;
        } else if (iz == nz) {
          fm = 1;
          fp = 0;
        } else
          fm = 1 - (fp = (b->z[ip] - zmin) / dz + 0.5 - iz);
      } else {
        fm = 1;
        fp = 0;
      }
      Jz[IDX(iz, ir)] += fm * Jm;
      if (lsm)
        Jz[IDX(iz + 1, ir)] += fp * Jm;
      if (rsm) {
        Jz[IDX(iz, ir + 1)] += fm * Jp;
        if (lsm)
          Jz[IDX(iz + 1, ir + 1)] += fp * Jp;
      }
    }
    /* Jr, space_charge.c:141-215 */
    for (ip = 0; ip < b->np; ip++) {
      if (!(b->status[ip] & SPIFFE_PART_ACTIVE))
        continue;
      ir = rsm ? (long)(b->r[ip] / dr + 0.5) : (long)(b->r[ip] / dr + 1.0);
      iz = lsm ? (long)((b->z[ip] - zmin) / dz) : (long)((b->z[ip] - zmin) / dz + 0.5);
      if (iz < 0 || iz > nz)
        continue;
      if (ir < 0 || ir >= nr)
        continue;
      QoV = b->Q[ip] * one_over_piDzDr2;
      if (rsm)
        fm = 1 - (fp = b->r[ip] / dr + 0.5 - ir);
      else {
        fm = 1;
        fp = 0;
      }
      QVG = b->vr[ip] * QoV;
      if (ir == 0) {
        Jm = 0;
        Jp = QVG;
      } else if (ir < nr - 1) {
        Jm = fm * QVG / (sq(ir) - sq(ir - 1));
        Jp = fp * QVG / (sq(ir + 1) - sq(ir));
      } else {
        Jm = 0;
        ir--;
        Jp = QVG / (sq(ir + 1) - sq(ir));
      }
      if (lsm) {
        if (iz == nz) {
          fm = 1;
          fp = 0;
        } else
          fm = 1 - (fp = (b->z[ip] - zmin) / dz - iz);
      } else {
        fm = 1;
        fp = 0;
      }
      Jr[IDX(iz, ir)] += fm * Jm;
      if (lsm)
        Jr[IDX(iz + 1, ir)] += fp * Jm;
      if (rsm) {
        Jr[IDX(iz, ir + 1)] += fm * Jp;
        if (lsm)
          Jr[IDX(iz + 1, ir + 1)] += fp * Jp;
      }
    }
  }
  if (m->modes & SPIFFE_FL_TE_FIELDS) {
    double *Jphi = f->Jphi;
    /* Jphi, space_charge.c:218-294 */
    for (ip = 0; ip < b->np; ip++) {
      if (!(b->status[ip] & SPIFFE_PART_ACTIVE))
        continue;
      ir = rsm ? (long)(b->r[ip] / dr) : (long)(b->r[ip] / dr + 0.5);
      iz = lsm ? (long)((b->z[ip] - zmin) / dz) : (long)((b->z[ip] - zmin) / dz + 0.5);
      if (iz < 0 || iz > nz)
        continue;
      if (ir < 0 || ir > nr)
        continue;
      QoV = b->Q[ip] * one_over_piDzDr2;
      if (rsm)
        fm = 1 - (fp = b->r[ip] / dr - ir);
      else {
        fm = 1;
        fp = 0;
      }
      QVG = b->vphi[ip] * QoV;
      if (ir == 0) {
        Jm = 4 * fm * QVG;
        Jp = fp * QVG / (sq(1.5) - sq(0.5));
      } else if (ir < nr - 1) {
        Jm = fm * QVG / (sq(ir + 0.5) - sq(ir - 0.5));
        Jp = fp * QVG / (sq(ir + 1.5) - sq(ir + 0.5));
      } else {
        Jm = 0;
        Jp = fp * QVG / (sq(ir + 0.5) - sq(ir - 0.5));
        ir--;
      }
      if (lsm) {
        if (iz == nz - 1)
          fm = 1 - (fp = 0);
        else
          fm = 1 - (fp = (b->z[ip] - zmin) / dz - iz);
      } else {
        fm = 1;
        fp = 0;
      }
      Jphi[IDX(iz, ir)] += fm * Jm;
      if (lsm)
        Jphi[IDX(iz + 1, ir)] += fp * Jm;
      if (rsm) {
        Jphi[IDX(iz, ir + 1)] += fm * Jp;
        if (lsm)
          Jphi[IDX(iz + 1, ir + 1)] += fp * Jp;
      }
    }
  }
}

/* ------------------------------------------------------- gather and push */

/* checkLossCode, advance_particles.c:31-65 */
static int loss_code(const spiffe_mesh *m, const int16_t *fl, long iz, long ir)
{
  const long nz = m->nz, nr = m->nr;
  if (fl[IDX(iz, ir)] & SPIFFE_FL_IS_INSIDE)
    return 3;
  if (fl[IDX(iz, ir)] & SPIFFE_FL_IS_SURFACE) {
    if (iz + 1 > nz)
      return 4;
    if (ir + 1 > nr)
      return 5;
    if (fl[IDX(iz + 1, ir + 1)] & SPIFFE_FL_IS_METAL && fl[IDX(iz, ir + 1)] & SPIFFE_FL_IS_METAL &&
        fl[IDX(iz + 1, ir)] & SPIFFE_FL_IS_METAL)
      return 6;
  }
  return 0;
}

/* interpolateFields, advance_particles.c:622-890 (the on-axis expansion of
 * :837-844 contributes nothing unless add_on_axis_fields was given, which this
 * path does not support).  out = Ez, Er, Ephi, Bz, Br, Bphi. */
void orc_gather(const spiffe_mesh *m, const spiffe_field_set *f, double z, double r, double *out)
{
  const long nz = m->nz, nr = m->nr;
  const double dz = m->dz, dr = m->dr, zmin = m->zmin;
  const int longit = (m->modes & SPIFFE_FL_LONGIT_INTERP) != 0, radial = (m->modes & SPIFFE_FL_RADIAL_INTERP) != 0;
  const int16_t *fl = f->flags;
  long iz, ir, iz1, ir1;
  double fr, fl_, fa, fb;
  double Ez = 0, Er = 0, Ephi = 0, Bz = 0, Br = 0, Bphi = 0;

  /* Ez and Br, :649-710 */
  if (longit) {
    iz = (long)(fr = (z - zmin) / dz + 0.5);
    fr -= iz;
    fl_ = 1 - fr;
  } else {
    iz = (long)((z - zmin) / dz + 1);
    fl_ = 1;
    fr = 0;
  }
  if (radial) {
    ir = (long)(fa = r / dr);
    fa -= ir;
    fb = 1 - fa;
  } else {
    ir = (long)(r / dr + 0.5);
    fa = 0;
    fb = 1;
  }
  if (iz >= 0 && iz < nz && ir >= 0 && ir < nr) {
    if ((iz1 = iz + 1) >= nz)
      iz1 = iz;
    if ((ir1 = ir + 1) >= nr)
      ir1 = ir;
    if (fl[IDX(iz, ir + 1)] & SPIFFE_FL_ER_ZERO && fl[IDX(iz, ir)] & SPIFFE_FL_ER_ZERO) {
      if (iz > 0 && (fl[IDX(iz - 1, ir)] || fl[IDX(iz - 1, ir + 1)]))
        iz = iz1;
      else
        iz1 = iz;
    } else if (fl[IDX(iz1, ir + 1)] & SPIFFE_FL_ER_ZERO && fl[IDX(iz1, ir)] & SPIFFE_FL_ER_ZERO) {
      iz1 = iz;
    }
    if (m->modes & SPIFFE_FL_TM_FIELDS)
      Ez = fb * (fl_ * (f->Ez[IDX(iz, ir)] + f->EzImposed[IDX(iz, ir)]) +
                 fr * (f->Ez[IDX(iz1, ir)] + f->EzImposed[IDX(iz1, ir)])) +
           fa * (fl_ * (f->Ez[IDX(iz, ir1)] + f->EzImposed[IDX(iz, ir1)]) +
                 fr * (f->Ez[IDX(iz1, ir1)] + f->EzImposed[IDX(iz1, ir1)]));
    if (r != 0 && m->modes & SPIFFE_FL_TE_FIELDS)
      Br = fb * (fl_ * f->Br2[IDX(iz, ir)] + fr * f->Br2[IDX(iz1, ir)]) +
           fa * (fl_ * f->Br2[IDX(iz, ir1)] + fr * f->Br2[IDX(iz1, ir1)]);
  }

  /* Er and Bz, :713-752 */
  if (longit) {
    iz = (long)(fr = (z - zmin) / dz);
    fr -= iz;
    fl_ = 1 - fr;
  } else {
    iz = (long)((z - zmin) / dz + 0.5);
    fr = 0;
    fl_ = 1;
  }
  if (radial) {
    ir = (long)(fa = r / dr + 0.5);
    fa -= ir;
    fb = 1 - fa;
  } else {
    ir = (long)(r / dr + 1);
    fa = 0;
    fb = 1;
  }
  if (iz >= 0 && iz < nz && ir >= 0) {
    if (ir >= nr)
      ir = nr - 1;
    iz1 = iz + 1;
    ir1 = ir + 1;
    if (fl[IDX(iz + 1, ir)] & SPIFFE_FL_EZ_ZERO && fl[IDX(iz, ir)] & SPIFFE_FL_EZ_ZERO)
      ir = ir1;
    else if (fl[IDX(iz + 1, ir + 1)] & SPIFFE_FL_EZ_ZERO && fl[IDX(iz, ir + 1)] & SPIFFE_FL_EZ_ZERO)
      ir1 = ir;
    if (r != 0 && m->modes & SPIFFE_FL_TM_FIELDS)
      Er = fl_ * (fb * (f->Er[IDX(iz, ir)] + f->ErImposed[IDX(iz, ir)]) + fa * (f->Er[IDX(iz, ir1)] + f->ErImposed[IDX(iz, ir1)])) +
           fr * (fb * (f->Er[IDX(iz1, ir)] + f->ErImposed[IDX(iz1, ir)]) + fa * (f->Er[IDX(iz1, ir1)] + f->ErImposed[IDX(iz1, ir1)]));
    if (m->modes & SPIFFE_FL_TE_FIELDS)
      Bz = fl_ * (fb * f->Bz2[IDX(iz, ir)] + fa * f->Bz2[IDX(iz, ir1)]) + fr * (fb * f->Bz2[IDX(iz1, ir)] + fa * f->Bz2[IDX(iz1, ir1)]);
  }

  /* Ephi, :754-786 */
  if (longit) {
    iz = (long)(fr = (z - zmin) / dz);
    fr -= iz;
    fl_ = 1 - fr;
  } else {
    iz = (long)((z - zmin) / dz + 0.5);
    fr = 0;
    fl_ = 1;
  }
  if (radial) {
    ir = (long)(fa = r / dr);
    fa -= ir;
    fb = 1 - fa;
  } else {
    ir = (long)(r / dr + 0.5);
    fa = 0;
    fb = 1;
  }
  if (r != 0 && m->modes & SPIFFE_FL_TE_FIELDS && iz >= 0 && iz < nz && ir >= 0 && ir < nr) {
    if ((iz1 = iz + 1) >= nz)
      iz1 = iz;
    if ((ir1 = ir + 1) >= nr)
      ir1 = ir;
    Ephi = fl_ * fb * f->Ephi[IDX(iz, ir)] + fr * fb * f->Ephi[IDX(iz1, ir)] + fl_ * fa * f->Ephi[IDX(iz, ir1)] +
           fr * fa * f->Ephi[IDX(iz1, ir1)];
  }

  /* Bphi at the E-field time level (Bphi2), :788-825 */
  if (m->modes & SPIFFE_FL_TM_FIELDS) {
    if (longit) {
      iz = (long)(fr = (z - zmin) / dz + 0.5);
      fr -= iz;
      fl_ = 1 - fr;
    } else {
      iz = (long)((z - zmin) / dz + 1);
      fr = 0;
      fl_ = 1;
    }
    if (radial) {
      ir = (long)(fa = r / dr + 0.5);
      fa -= ir;
      fb = 1 - fa;
    } else {
      ir = (long)(r / dr + 1);
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
      Bphi = fl_ * fb * f->Bphi2[IDX(iz, ir)] + fr * fb * f->Bphi2[IDX(iz1, ir)] + fa * fl_ * f->Bphi2[IDX(iz, ir1)] +
             fr * fa * f->Bphi2[IDX(iz1, ir1)];
    }
  }

  /* uniform fields and switches, :828-857 */
  Ez += m->constant_E[0];
  Er += m->constant_E[1];
  Ephi += m->constant_E[2];
  Bz += m->constant_B[0];
  Br += m->constant_B[1];
  Bphi += m->constant_B[2];
  if (m->turn_off[0])
    Ez = 0;
  if (m->turn_off[1])
    Er = 0;
  if (m->turn_off[2])
    Ephi = 0;
  if (m->turn_off[3])
    Bz = 0;
  if (m->turn_off[4])
    Br = 0;
  if (m->turn_off[5])
    Bphi = 0;

  /* solenoid fields on nodes, :859-875 */
  if (m->has_solenoid) {
    iz = (long)(fr = (z - zmin) / dz);
    ir = (long)(fa = r / dr);
    if (ir >= 0 && iz >= 0 && ir < nr && iz < nz) {
      fa -= ir;
      fb = 1 - fa;
      fr -= iz;
      fl_ = 1 - fr;
      Bz += fl_ * (fb * f->BzImposed[IDX(iz, ir)] + fa * f->BzImposed[IDX(iz, ir + 1)]) +
            fr * (fb * f->BzImposed[IDX(iz + 1, ir)] + fa * f->BzImposed[IDX(iz + 1, ir + 1)]);
      Br += fl_ * (fb * f->BrImposed[IDX(iz, ir)] + fa * f->BrImposed[IDX(iz, ir + 1)]) +
            fr * (fb * f->BrImposed[IDX(iz + 1, ir)] + fa * f->BrImposed[IDX(iz + 1, ir + 1)]);
    }
  }
  out[0] = Ez;
  out[1] = Er;
  out[2] = Ephi;
  out[3] = Bz;
  out[4] = Br;
  out[5] = Bphi;
}

/* setParticleVelocities, advance_particles.c:605-620 */
static void set_velocities(double *vz, double *vr, double *vphi, double *gamma, double pz, double pr, double r_pphi,
                           double r)
{
  if (r) {
    *gamma = sqrt(sq(pz) + sq(pr) + sq(r_pphi / r) + 1);
    *vphi = C_MKS * r_pphi / r / (*gamma);
  } else {
    *gamma = sqrt(sq(pz) + sq(pr) + 1);
    *vphi = 0;
  }
  *vz = C_MKS * pz / (*gamma);
  *vr = C_MKS * pr / (*gamma);
}

static void screen_record(spiffe_screen_set *s, const spiffe_beam_set *b, long ip, const double *q)
{
  int k;
  if (s->nb >= s->capacity)
    return;
  for (k = 0; k < SPIFFE_SCREEN_QUANS; k++)
    s->col[k][s->nb] = q[k];
  s->rmin[s->nb] = b->rmin[ip];
  s->rmax[s->nb] = b->rmax[ip];
  s->zmin[s->nb] = b->zmin[ip];
  s->zmax[s->nb] = b->zmax[ip];
  s->generation[s->nb] = b->generation[ip];
  s->particleID[s->nb] = b->particleID[ip];
  s->nb++;
}

/* advance_particles, advance_particles.c:67-575: drift with the old velocity,
 * activation and loss tests, gather, momentum kick with the stored (old)
 * velocities, new velocities, screen crossings, then removal of lost
 * particles under the chosen compaction policy.  Screen records are appended
 * after s->nb (callers reset nb per step as the reference does, :347). */
long orc_advance_particles(const spiffe_mesh *m, const spiffe_field_set *f, spiffe_beam_set *b, spiffe_screen_set *screens,
                           int n_screens, const spiffe_push_options *opt)
{
  const long nz = m->nz, nr = m->nr;
  const double dt = m->dt, dz = m->dz, dr = m->dr, zmin = m->zmin, zmax = m->zmax, rmax = m->rmax;
  const int16_t *fl = f->flags;
  const long np = b->np;
  const int forced = opt->tb_electrons_per_macroparticle && (opt->tb_z_force || opt->tb_r_force);
  double *z0 = malloc(sizeof(double) * (size_t)(np + 1)), *r0s = malloc(sizeof(double) * (size_t)(np + 1));
  double *vzz = malloc(sizeof(double) * (size_t)(np + 1)), *vra = malloc(sizeof(double) * (size_t)(np + 1));
  double *pz0a = malloc(sizeof(double) * (size_t)(np + 1)), *pr0a = malloc(sizeof(double) * (size_t)(np + 1));
  double *rp0a = malloc(sizeof(double) * (size_t)(np + 1));
  char *lost = calloc((size_t)(np + 1), 1);
  long ip, is, newActive = 0, nlost = 0;
  double pz0_last = 0, pr0_last = 0, r_pphi0_last = 0;

  for (ip = 0; ip < np; ip++) {
    double z, r, vz, vr, pz, pr, r_pphi, vphi, gamma, pphi, adjust = 1, E[6];
    long iz, ir;
    int r_was_negative = 0;
    z = z0[ip] = b->z[ip];
    r = r0s[ip] = b->r[ip];
    if (z > b->zmax[ip])
      b->zmax[ip] = z;
    if (z < b->zmin[ip])
      b->zmin[ip] = z;
    if (r > b->rmax[ip])
      b->rmax[ip] = r;
    if (r < b->rmin[ip])
      b->rmin[ip] = r;
    vz = b->vz[ip];
    vr = b->vr[ip];
    z += vz * dt;
    r += vr * dt;
    if (!(b->status[ip] & SPIFFE_PART_ACTIVE)) {
      /* activation on entering the mesh, :167-189 */
      iz = (long)((z - zmin) / dz);
      ir = (long)(fabs(r) / dr);
      if ((z >= zmin && z <= zmax && r <= rmax) && ir <= nr && !loss_code(m, fl, iz, ir)) {
        b->status[ip] |= SPIFFE_PART_ACTIVE;
        newActive++;
        b->t0[ip] = m->time;
        b->r0[ip] = b->r[ip];
        b->z0[ip] = b->z[ip];
        if (iz > 0 && loss_code(m, fl, iz - 1, ir))
          adjust = (z - (iz * dz + zmin)) / (z - z0[ip]);
        else
          adjust = (z - zmin) / (z - z0[ip]);
        if (adjust > 1)
          adjust = 1;
      }
    }
    if (opt->z_forces_start > zmin && opt->z_forces_start < zmax) {
      if (z0[ip] < opt->z_forces_start) {
        if (z < opt->z_forces_start)
          adjust = 0;
        else
          adjust = (z - opt->z_forces_start) / (z - z0[ip]);
      }
    }
    pz = pz0a[ip] = b->pz[ip];
    pr = pr0a[ip] = b->pr[ip];
    r_pphi = rp0a[ip] = b->r_pphi[ip];
    pz0_last = pz;
    pr0_last = pr;
    r_pphi0_last = r_pphi;
    vphi = b->vphi[ip];

    /* loss tests, :211-236 */
    if ((b->status[ip] & SPIFFE_PART_ACTIVE) && (z < zmin || z > zmax || r > rmax))
      lost[ip] = 1;
    if (!lost[ip] && (b->status[ip] & SPIFFE_PART_ACTIVE)) {
      iz = (long)((z - zmin) / dz);
      ir = (long)(fabs(r) / dr);
      if (iz > nz || ir > nr || iz < 0 || ir < 0)
        lost[ip] = 1;
      else if (loss_code(m, fl, iz, ir))
        lost[ip] = 1;
    }
    /* reflection through the axis, :242-248 */
    if (r < 0) {
      r *= -1;
      pr *= -1;
      r_was_negative = 1;
    }
    if (!lost[ip] && (b->status[ip] & SPIFFE_PART_ACTIVE)) {
      if (z > b->zmax[ip])
        b->zmax[ip] = z;
      if (z < b->zmin[ip])
        b->zmin[ip] = z;
      if (r > b->rmax[ip])
        b->rmax[ip] = r;
      if (r < b->rmin[ip])
        b->rmin[ip] = r;
    }

    if (!forced) {
      /* kick, :270-287 */
      if (b->status[ip] & SPIFFE_PART_ACTIVE)
        orc_gather(m, f, z, r, E);
      else
        E[0] = E[1] = E[2] = E[3] = E[4] = E[5] = 0;
      if (opt->tb_electrons_per_macroparticle)
        b->stiffness = 1;
      pphi = (r ? r_pphi / r : 0);
      gamma = sqrt(sq(pr) + sq(pz) + sq(pphi) + 1);
      pr += adjust * dt * ((r ? sq(pphi) * C_MKS / gamma / r : 0) + b->QoMC * (E[1] + vphi * E[3] - vz * E[5])) / b->stiffness;
      pz += adjust * dt * b->QoMC * (E[0] + vr * E[5] - vphi * E[4]) / b->stiffness;
      r_pphi += adjust * dt * b->QoMC * r * (E[2] + vz * E[4] - vr * E[3]) / b->stiffness;
    } else {
      /* forced test-beam acceleration, :289-311 */
      pphi = (r ? r_pphi / r : 0);
      gamma = sqrt(sq(pr) + sq(pz) + sq(pphi) + 1);
      pr += dt * ((r ? sq(pphi) * C_MKS / gamma / r : 0));
      if (z <= opt->tb_z_start_deceleration)
        pz += dt * opt->tb_z_force;
      else {
        pz -= dt * opt->tb_z_force;
        if (pz < 0)
          pz = 0;
      }
      if (r_was_negative)
        pr = 0;
      else if (r <= opt->tb_r_start_deceleration)
        pr += dt * opt->tb_r_force;
      else
        pr -= dt * opt->tb_r_force;
    }
    b->z[ip] = z;
    b->r[ip] = r;
    b->pz[ip] = pz;
    b->pr[ip] = pr;
    b->r_pphi[ip] = r_pphi;
    set_velocities(&b->vz[ip], &b->vr[ip], &b->vphi[ip], &gamma, pz, pr, r_pphi, r);
    if (lost[ip]) {
      b->status[ip] &= ~SPIFFE_PART_ACTIVE;
      b->status[ip] |= SPIFFE_PART_LOST;
      nlost++;
    }
    vzz[ip] = vz;
    vra[ip] = vr;
  }
  b->npActive += newActive;

  /* screen crossings, :362-434 */
  for (ip = 0; ip < np; ip++) {
    double dtp, r0 = r0s[ip], pphi0, pphi_new, q[SPIFFE_SCREEN_QUANS];
    const int ref = opt->screen_momentum == SPIFFE_SCREEN_REFERENCE;
    const double pz0 = ref ? pz0_last : pz0a[ip], pr0 = ref ? pr0_last : pr0a[ip];
    const double r_pphi0 = ref ? r_pphi0_last : rp0a[ip];
    for (is = 0; is < n_screens; is++) {
      spiffe_screen_set *s = screens + is;
      if (s->z_position <= b->z[ip] && s->z_position > z0[ip] && s->direction == 1) {
        dtp = (s->z_position - z0[ip]) / vzz[ip];
        pphi_new = b->r[ip] ? b->r_pphi[ip] / b->r[ip] : 0;
        pphi0 = r0 ? r_pphi0 / r0 : 0;
        q[0] = r0 + vra[ip] * dtp;
        q[1] = pz0 + (b->pz[ip] - pz0) / dt * dtp;
        q[2] = pr0 + (b->pr[ip] - pr0) / dt * dtp;
        q[3] = pphi0 + (pphi_new - pphi0) / dt * dtp;
        q[4] = (m->time - dt + dtp);
        q[5] = b->Q[ip];
        q[6] = b->r0[ip];
        q[7] = b->t0[ip];
        screen_record(s, b, ip, q);
      } else if (s->z_position >= b->z[ip] && s->z_position < z0[ip] && s->direction == -1) {
        dtp = (s->z_position - z0[ip]) / vzz[ip];
        r0 += vra[ip] * dtp;
        q[0] = r0;
        q[1] = b->pz[ip];
        q[2] = b->pr[ip];
        q[3] = r0 ? b->r_pphi[ip] / r0 : 0;
        q[4] = (m->time - dt + dtp);
        q[5] = b->Q[ip];
        q[6] = b->r0[ip];
        q[7] = b->t0[ip];
        screen_record(s, b, ip, q);
      }
    }
  }

  /* removal of lost particles, :490-518 */
  if (nlost) {
#define MOVE(dst, src)                       \
  do {                                       \
    b->Q[dst] = b->Q[src];                   \
    b->z[dst] = b->z[src];                   \
    b->r[dst] = b->r[src];                   \
    b->pz[dst] = b->pz[src];                 \
    b->pr[dst] = b->pr[src];                 \
    b->vz[dst] = b->vz[src];                 \
    b->vr[dst] = b->vr[src];                 \
    b->r_pphi[dst] = b->r_pphi[src];         \
    b->vphi[dst] = b->vphi[src];             \
    b->t0[dst] = b->t0[src];                 \
    b->r0[dst] = b->r0[src];                 \
    b->z0[dst] = b->z0[src];                 \
    b->rmin[dst] = b->rmin[src];             \
    b->zmin[dst] = b->zmin[src];             \
    b->rmax[dst] = b->rmax[src];             \
    b->zmax[dst] = b->zmax[src];             \
    b->generation[dst] = b->generation[src]; \
    b->particleID[dst] = b->particleID[src]; \
    b->status[dst] = b->status[src];         \
  } while (0)
    if (opt->compaction == SPIFFE_COMPACT_REFERENCE) {
      /* as the reference behaves: the first lost index ends the beam */
      for (ip = 0; ip < b->np; ip++)
        if (lost[ip]) {
          b->npActive -= b->np - ip;
          b->np = ip;
          break;
        }
    } else {
      for (ip = 0; ip < b->np; ip++) {
        while (ip < b->np && lost[ip]) {
          b->np -= 1;
          b->npActive -= 1;
          MOVE(ip, b->np);
          lost[ip] = lost[b->np];
        }
      }
    }
#undef MOVE
  }
  free(z0);
  free(r0s);
  free(vzz);
  free(vra);
  free(pz0a);
  free(pr0a);
  free(rp0a);
  free(lost);
  return nlost;
}

/* --------------------------------------------------------------- Poisson */

/* Chebyshev over-relaxation factor sequence of solve_poisson_cyl,
 * poisson.c:342-344, :416-419: omega[n] is used on half-sweep n. */
static double jacobi_radius(long nz, long nr, double dz, double dr)
{
  return (cos(PI / nz) + sq(dz / dr) * cos(PI / nr)) / (1 + sq(dz / dr));
}

/* solve_poisson_cyl, poisson.c:17-130: red-black SOR, one colour per
 * iteration, stopping when sum|residual| < accuracy*sum|rhs| (n > 0). */
long orc_solve_poisson(const spiffe_mesh *m, const int16_t *fl, double *Psi, const double *rhs, double accuracy,
                       long iteration_limit, double *residual_out, double *driving_out)
{
  const long nz = m->nz, nr = m->nr;
  const double dz = m->dz, dr = m->dr;
  long iz, ir, n;
  double residual, omega, r_jacobi, total_rhs = 0, total_res = 0, a, c, d, e;
  if (rhs)
    for (iz = 0; iz < nz; iz++)
      for (ir = 0; ir < nr - 1; ir++)
        total_rhs += fabs(rhs[IDX(iz, ir)]);
  if (driving_out)
    *driving_out = total_rhs;
  r_jacobi = jacobi_radius(nz, nr, dz, dr);
  omega = 1.0;
  a = 1 / sq(dz);
  e = -2 * (1 / sq(dz) + 1 / sq(dr));
  for (n = 0; n < iteration_limit; n++) {
    total_res = 0;
    for (ir = 0; ir < nr - 1; ir++) {
      long lo = m->left_bc == SPIFFE_DIRICHLET ? 0 : 1;
      long hi = m->right_bc == SPIFFE_DIRICHLET ? nz - 1 : nz - 2;
      if (ir != 0) {
        c = 1 / sq(dr) * (1 + 1. / (2 * ir));
        d = 1 / sq(dr) * (1 - 1. / (2 * ir));
      } else
        c = d = 1 / sq(dr);
      /* the reference visits the left row, the interior, then the right row */
      for (iz = lo; iz <= hi; iz++) {
        double left, right;
        if ((ir + iz) % 2 != n % 2 || (fl[IDX(iz, ir)] & SPIFFE_FL_IS_METAL))
          continue;
        if (iz == 0 && lo == 0) {
          left = Psi[IDX(iz + 1, ir)];
          right = Psi[IDX(iz + 1, ir)];
        } else if (iz == nz - 1 && hi == nz - 1) {
          left = Psi[IDX(iz - 1, ir)];
          right = Psi[IDX(iz - 1, ir)];
        } else {
          left = Psi[IDX(iz + 1, ir)];
          right = Psi[IDX(iz - 1, ir)];
        }
        if (ir == 0) {
          residual = a * (left + right) + 4 * c * Psi[IDX(iz, ir + 1)] + (e - 2 * c) * Psi[IDX(iz, ir)] -
                     (rhs ? rhs[IDX(iz, ir)] : 0);
          Psi[IDX(iz, ir)] -= omega * residual / (e - 2 * c);
        } else {
          residual = a * (left + right) + c * Psi[IDX(iz, ir + 1)] + d * Psi[IDX(iz, ir - 1)] + e * Psi[IDX(iz, ir)] -
                     (rhs ? rhs[IDX(iz, ir)] : 0);
          Psi[IDX(iz, ir)] -= omega * residual / e;
        }
        total_res += fabs(residual);
      }
    }
    if (n == 0)
      omega = 1.0 / (1 - sq(r_jacobi) / 2);
    else
      omega = 1.0 / (1 - sq(r_jacobi) * omega / 4);
    if (n > 0 && (total_res < accuracy * total_rhs || total_res == 0)) {
      if (residual_out)
        *residual_out = total_res;
      return n;
    }
  }
  if (residual_out)
    *residual_out = total_res;
  return -1;
}

/* cells that carry surface rather than volume charge, poisson_correction.c:166 */
static int surface_cell(const spiffe_mesh *m, const int16_t *fl, long iz, long ir)
{
  const long nr = m->nr;
  return (fl[IDX(iz, ir)] & SPIFFE_FL_IS_METAL) || (iz == 0 && m->left_bc == SPIFFE_NEUMANN) ||
         (iz == m->nz - 1 && m->right_bc == SPIFFE_NEUMANN) || (ir == m->nr - 1 && m->upper_bc == SPIFFE_NEUMANN);
}

/* apparent charge from the flux of E through each cell, poisson_correction.c:
 * 141-182 (first pass: top-row surface term added, :173) and :335-375 (second
 * pass: subtracted, :367).  Returns the centroid numerator in *centroid. */
static void apparent_charge(const spiffe_mesh *m, spiffe_field_set *f, double *volume, int second_pass, double *Qsurface,
                            double *centroid)
{
  const long nz = m->nz, nr = m->nr;
  const double dr = m->dr, dz = m->dz, dr2 = sq(dr), drdz = dr * dz;
  const double eps = EPS0;
  long iz, ir;
  double Az, Ar_inner, Ar_outer, dQ;
  for (ir = 0; ir < nr; ir++) {
    if (ir == 0) {
      Ar_inner = Ar_outer = PI * drdz;
      Az = dr2 / 4 * PI;
    } else {
      Ar_inner = PI * (2 * ir - 1) * drdz;
      Ar_outer = PI * (2 * ir + 1) * drdz;
      Az = PI * dr2 / 4 * ((2 * ir + 1) * (2 * ir + 1) - (2 * ir - 1) * (2 * ir - 1));
    }
    volume[ir] = Az * dz;
    for (iz = 0; iz < nz; iz++) {
      f->Q[IDX(iz, ir)] = 0;
      if (ir == 0)
        dQ = (f->Er[IDX(iz, ir + 1)] * Ar_outer + (f->Ez[IDX(iz + 1, ir)] - f->Ez[IDX(iz, ir)]) * Az) * eps;
      else
        dQ = (f->Er[IDX(iz, ir + 1)] * Ar_outer - f->Er[IDX(iz, ir)] * Ar_inner +
              (f->Ez[IDX(iz + 1, ir)] - f->Ez[IDX(iz, ir)]) * Az) *
             eps;
      if (surface_cell(m, f->flags, iz, ir)) {
        if (iz == 0)
          dQ += f->Ez[IDX(iz, ir)] * Az * eps;
        if (iz == nz - 1)
          dQ -= f->Ez[IDX(iz + 1, ir)] * Az * eps;
        if (ir == nr - 1) {
          if (second_pass)
            dQ -= f->Ez[IDX(iz, ir + 1)] * Ar_outer * eps;
          else
            dQ += f->Ez[IDX(iz, ir + 1)] * Ar_outer * eps;
        }
        *Qsurface += dQ;
      } else {
        f->Q[IDX(iz, ir)] = dQ;
        if (centroid)
          *centroid += dQ * (iz * dz + m->zmin);
      }
    }
  }
}

/* removal of the particles' own charge, poisson_correction.c:190-242 */
static double remove_particle_charge(const spiffe_mesh *m, spiffe_field_set *f, const spiffe_beam_set *b)
{
  const long nz = m->nz, nr = m->nr;
  const double dz = m->dz, dr = m->dr;
  const int lsm = (m->modes & SPIFFE_FL_LONGIT_SMEAR) != 0, rsm = (m->modes & SPIFFE_FL_RADIAL_SMEAR) != 0;
  const int ln = m->left_bc == SPIFFE_NEUMANN, rn = m->right_bc == SPIFFE_NEUMANN, un = m->upper_bc == SPIFFE_NEUMANN;
  const int16_t *fl = f->flags;
  double Qreal = 0, fa, fb, fr, fl_;
  long ip, iz, ir;
  for (ip = 0; ip < b->np; ip++) {
    if (!(b->status[ip] & SPIFFE_PART_ACTIVE))
      continue;
    iz = lsm ? (long)((b->z[ip] - m->zmin) / dz) : (long)((b->z[ip] - m->zmin) / dz + 0.5);
    ir = rsm ? (long)(b->r[ip] / dr) : (long)(b->r[ip] / dr + 0.5);
    if (iz < 0 || iz >= nz)
      continue;
    if (ir < 0 || ir >= nr)
      continue;
    if (rsm && ir != nr - 1)
      fb = 1 - (fa = b->r[ip] / dr - ir);
    else {
      fb = 1;
      fa = 0;
    }
    if (lsm && iz != nz - 1)
      fl_ = 1 - (fr = (b->z[ip] - m->zmin) / dz - iz);
    else {
      fl_ = 1;
      fr = 0;
    }
    if (!((fl[IDX(iz, ir)] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz - 1 && rn) || (ir >= nr - 1 && un))) {
      f->Q[IDX(iz, ir)] -= b->Q[ip] * fb * fl_;
      Qreal += b->Q[ip] * fb * fl_;
    }
    if (!((fl[IDX(iz + 1, ir)] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz && rn) || (ir >= nr - 1 && un))) {
      f->Q[IDX(iz + 1, ir)] -= b->Q[ip] * fb * fr;
      Qreal += b->Q[ip] * fb * fr;
    }
    if (!((fl[IDX(iz, ir + 1)] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz - 1 && rn) || (ir >= nr && un))) {
      f->Q[IDX(iz, ir + 1)] -= b->Q[ip] * fa * fl_;
      Qreal += b->Q[ip] * fa * fl_;
    }
    if (!((fl[IDX(iz + 1, ir + 1)] & SPIFFE_FL_IS_METAL) || (iz == 0 && ln) || (iz >= nz && rn) || (ir >= nr && un))) {
      f->Q[IDX(iz + 1, ir + 1)] -= b->Q[ip] * fa * fr;
      Qreal += b->Q[ip] * fa * fr;
    }
  }
  return Qreal;
}

/* poisson_guess, poisson_correction.c:564-615 */
static void poisson_guess(const spiffe_mesh *m, double *Psi, double charge, double centroid, int code)
{
  const long nz = m->nz, nr = m->nr;
  long iz, ir;
  double guess, dist;
  switch (code) {
  case 1:
    for (ir = 0; ir < nr; ir++) {
      guess = charge / (PIx2 * EPS0) * log((ir ? ir : 0.5) * m->dr);
      for (iz = 0; iz < nz; iz++)
        Psi[IDX(iz, ir)] = guess;
    }
    break;
  case 2:
    for (ir = 0; ir < nr; ir++)
      for (iz = 0; iz < nz; iz++) {
        dist = sqrt(sq((iz * m->dz + m->zmin) - centroid) + sq(m->dr * (ir + 0.5)));
        Psi[IDX(iz, ir)] = charge / (4 * PI * EPS0 * dist);
      }
    break;
  case 3:
    for (iz = 0; iz < nz; iz++)
      for (ir = 0; ir < nr; ir++)
        Psi[IDX(iz, ir)] = 0;
    break;
  default:
    break;
  }
}

/* Ez, Er -= grad(Psi) and their boundary copies, poisson_correction.c:288-326 */
static void subtract_gradient(const spiffe_mesh *m, spiffe_field_set *f)
{
  const long nz = m->nz, nr = m->nr;
  const double dz = m->dz, dr = m->dr;
  const int16_t *fl = f->flags;
  long iz, ir;
  for (ir = 0; ir < nr; ir++) {
    for (iz = 1; iz < nz; iz++)
      if (!(fl[IDX(iz, ir)] & SPIFFE_FL_EZ_ZERO))
        f->Ez[IDX(iz, ir)] -= -(f->Psi[IDX(iz, ir)] - f->Psi[IDX(iz - 1, ir)]) / dz;
    f->Ez[IDX(0, ir)] = m->left_bc == SPIFFE_NEUMANN ? f->Ez[IDX(1, ir)] : -f->Ez[IDX(1, ir)];
    f->Ez[IDX(nz, ir)] = m->right_bc == SPIFFE_NEUMANN ? f->Ez[IDX(nz - 1, ir)] : -f->Ez[IDX(nz - 1, ir)];
  }
  for (iz = 0; iz <= nz; iz++)
    f->Ez[IDX(iz, nr - 1)] = 0;
  for (ir = 1; ir <= nr; ir++)
    for (iz = 0; iz < nz; iz++)
      if (!(fl[IDX(iz, ir)] & SPIFFE_FL_ER_ZERO))
        f->Er[IDX(iz, ir)] -= -(f->Psi[IDX(iz, ir)] - f->Psi[IDX(iz, ir - 1)]) / dr;
  for (iz = 0; iz < nz; iz++)
    f->Er[IDX(iz, 0)] = -f->Er[IDX(iz, 1)];
  if (m->left_bc == SPIFFE_NEUMANN)
    for (ir = 0; ir <= nr; ir++)
      f->Er[IDX(0, ir)] = 0;
  if (m->right_bc == SPIFFE_NEUMANN)
    for (ir = 0; ir <= nr; ir++)
      f->Er[IDX(nz - 1, ir)] = 0;
}

/* add_poisson_correction, poisson_correction.c:73-454.  *pc_start_step holds
 * the reference's static (-1 before the first call, :87-92). */
int orc_poisson_correction(const spiffe_mesh *m, spiffe_field_set *f, const spiffe_beam_set *b, int space_charge,
                           const spiffe_poisson_options *o, int64_t *pc_start_step, spiffe_poisson_report *rep)
{
  const long nz = m->nz, nr = m->nr;
  double *volume, Qreal = 0, Qerror = 0, Qsurface = 0, centroid = 0;
  long iz, ir;
  memset(rep, 0, sizeof(*rep));
  if (o->maximum_iterations <= 0)
    return 0;
  if (*pc_start_step == -1)
    *pc_start_step = (int64_t)((o->start_time - m->start_time) / m->dt);
  if (o->step_interval <= 0 || m->time_step % o->step_interval != 0 || *pc_start_step > m->time_step)
    return 0;
  volume = calloc((size_t)nr + 1, sizeof(double));
  apparent_charge(m, f, volume, 0, &Qsurface, &centroid);
  if (space_charge)
    Qreal = remove_particle_charge(m, f, b);
  for (iz = 0; iz < nz; iz++)
    for (ir = 0; ir < nr; ir++)
      Qerror += f->Q[IDX(iz, ir)];
  rep->Qreal = Qreal;
  rep->Qerror = Qerror;
  rep->Qsurface = Qsurface;
  if ((o->error_charge_threshold > 0 && fabs(Qerror) < o->error_charge_threshold) ||
      (o->error_charge_threshold < 0 && (Qreal == 0 || fabs(Qerror / Qreal) < fabs(o->error_charge_threshold)))) {
    free(volume);
    return 0;
  }
  for (ir = 0; ir < nr; ir++)
    for (iz = 0; iz < nz; iz++)
      f->Q[IDX(iz, ir)] = -f->Q[IDX(iz, ir)] / (volume[ir] * EPS0);
  poisson_guess(m, f->Psi, Qerror, centroid, o->guess_code);
  rep->iterations = orc_solve_poisson(m, f->flags, f->Psi, f->Q, o->accuracy, (long)o->maximum_iterations,
                                      &rep->residual, &rep->driving);
  rep->ran = 1;
  subtract_gradient(m, f);
  /* the reference recomputes Q after the correction, :333-439 */
  Qsurface = 0;
  apparent_charge(m, f, volume, 1, &Qsurface, NULL);
  if (space_charge)
    remove_particle_charge(m, f, b);
  free(volume);
  return 1;
}

/* compute_imposed_Efield, poisson_correction.c:456-562; *last_factor holds
 * the reference's static (-1 initially, :463). */
void orc_imposed_efield(const spiffe_mesh *m, spiffe_field_set *f, const spiffe_poisson_options *o, int initialize,
                        double *last_factor, int64_t *iterations)
{
  const long nz = m->nz, nr = m->nr;
  const double dz = m->dz, dr = m->dr, T = m->imposed_ramp_time, F = m->imposed_flat_top_time, t = m->time;
  double ff = 1;
  long iz, ir;
  if (o->maximum_iterations <= 0)
    return;
  if (initialize) {
    long n = orc_solve_poisson(m, f->flags, f->PsiImposed, NULL, o->accuracy, (long)o->maximum_iterations, NULL, NULL);
    if (iterations)
      *iterations = n;
  }
  if (T) {
    if (t < T)
      ff = t / T;
    else if (t < (T + F))
      ff = 1;
    else if (t < (2 * T + F))
      ff = ((2 * T + F) - t) / T;
    else
      ff = 0;
    if (ff < 0)
      ff = 0;
  }
  if (ff == *last_factor)
    return;
  *last_factor = ff;
  for (ir = 0; ir < nr; ir++) {
    for (iz = 1; iz < nz; iz++)
      if (!(f->flags[IDX(iz, ir)] & SPIFFE_FL_EZ_ZERO))
        f->EzImposed[IDX(iz, ir)] = -ff * (f->PsiImposed[IDX(iz, ir)] - f->PsiImposed[IDX(iz - 1, ir)]) / dz;
    f->EzImposed[IDX(0, ir)] = m->left_bc == SPIFFE_NEUMANN ? f->EzImposed[IDX(1, ir)] : -f->EzImposed[IDX(1, ir)];
    f->EzImposed[IDX(nz, ir)] = m->right_bc == SPIFFE_NEUMANN ? f->EzImposed[IDX(nz - 1, ir)] : -f->EzImposed[IDX(nz - 1, ir)];
  }
  for (iz = 0; iz <= nz; iz++)
    f->EzImposed[IDX(iz, nr - 1)] = 0;
  for (ir = 1; ir <= nr; ir++)
    for (iz = 0; iz < nz; iz++)
      if (!(f->flags[IDX(iz, ir)] & SPIFFE_FL_ER_ZERO))
        f->ErImposed[IDX(iz, ir)] = -ff * (f->PsiImposed[IDX(iz, ir)] - f->PsiImposed[IDX(iz, ir - 1)]) / dr;
  for (iz = 0; iz < nz; iz++)
    f->ErImposed[IDX(iz, 0)] = -f->ErImposed[IDX(iz, 1)];
  if (m->left_bc == SPIFFE_NEUMANN)
    for (ir = 0; ir <= nr; ir++)
      f->ErImposed[IDX(0, ir)] = 0;
  if (m->right_bc == SPIFFE_NEUMANN)
    for (ir = 0; ir <= nr; ir++)
      f->ErImposed[IDX(nz - 1, ir)] = 0;
}

/* -------------------------------------------------------------- emission */

/* The project's counter-based generator (SplitMix64 finaliser; see
 * include/spiffe_b200_rng.h) as the stream random_1 draws from. */
static uint64_t orc_mix64(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

typedef struct {
  uint64_t key, counter;
} orc_rng;

static void orc_rng_seed(orc_rng *g, long seed)
{
  g->key = orc_mix64((uint64_t)seed * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL);
  g->counter = 0;
}

static double orc_rng_next(orc_rng *g)
{
  g->counter++;
  return (double)(orc_mix64(g->key + g->counter * 0x9E3779B97F4A7C15ULL) >> 11) * 0x1.0p-53;
}

/* Derived state of one cathode (CATHODE, spiffe.h:236-262). */
typedef struct orc_cathode {
  spiffe_cathode_options o;
  double initial_vz, QoMC, Q, inner_r2, outer_r2, ref_current_density, current_density, totalArea;
  double start_time, stop_time, number_per_step, electrons_per_macroparticle;
  int64_t start_step, stop_step, step_emission_started, n_bins, correction_interval, zoned_emission;
  long *distribution, *deficit;
  double *area, *rmin;
} orc_cathode;

typedef struct orc_emitter {
  orc_rng rng;
  int n;
  orc_cathode c[64];
} orc_emitter;

/* process_cathode_definition, cathode.c:21-237 (field emission splits the
 * cathode into one sub-cathode per radial cell, :93-99, :168-186).  Returns
 * the number of cathodes, or -1 for an input the reference rejects. */
int orc_cathode_define(orc_emitter *E, const spiffe_mesh *m, const spiffe_cathode_options *o)
{
  long n = 1, i;
  if (o->z_position < m->zmin || o->z_position > m->zmax || o->inner_radius > o->outer_radius ||
      o->inner_radius < 0 || o->outer_radius > m->rmax || o->stiffness <= 0)
    return -1;
  if (o->field_emission) {
    if (o->inner_radius != 0)
      n = (long)((o->outer_radius - o->inner_radius) / m->dr);
    else
      n = (long)((o->outer_radius - o->inner_radius + m->dr / 2) / m->dr);
  }
  orc_rng_seed(&E->rng, labs((long)o->random_number_seed));
  for (i = 0; i < n && E->n < 64; i++) {
    orc_cathode *c = &E->c[E->n++];
    memset(c, 0, sizeof(*c));
    c->o = *o;
    if (o->field_emission) {
      c->o.outer_radius = (i + 0.5) * m->dr;
      if ((c->o.inner_radius = c->o.outer_radius - m->dr) < 0)
        c->o.inner_radius = 0;
      if (i == n - 1)
        c->o.outer_radius = o->outer_radius;
      if (c->o.outer_radius > o->outer_radius)
        c->o.outer_radius = o->outer_radius;
      if (c->o.inner_radius < o->inner_radius)
        c->o.inner_radius = o->inner_radius;
    }
    c->initial_vz = o->initial_pz / sqrt(1 + sq(o->initial_pz)) * C_MKS;
    c->current_density = o->current_density;
    c->start_time = o->start_time;
    c->stop_time = o->stop_time;
    c->number_per_step = o->number_per_step;
    c->QoMC = -SPIFFE_E_MKS / (SPIFFE_ME_MKS * C_MKS);
    c->correction_interval = o->distribution_correction_interval;
    c->start_step = -1;
    c->step_emission_started = -1;
    c->electrons_per_macroparticle = o->electrons_per_macroparticle;
    c->zoned_emission = o->zoned_emission;
    if (o->discretize_radii)
      c->correction_interval = 0;
    if (o->field_emission)
      c->zoned_emission = 0;
    if (!c->zoned_emission)
      c->correction_interval = 0;
  }
  return (int)n;
}

/* fieldEmissionCurrentDensity, cathode.c:799-810 */
static double field_emission_J(double E, double beta, double wf)
{
  double y, t, v;
  E = fabs(E) * beta;
  y = 3.79e-5 * sqrt(E) / wf;
  t = ((-0.0020 * y + 0.0131) * y + 0.1091) * y + 0.9899;
  v = ((0.0445 * y - 0.6782) * y - 0.4091) * y + 1.0437;
  return 1.54e-6 * sq(E) / (wf * sq(t)) * exp(-6.83e9 * v * pow(wf, 1.5) / E);
}

/* set_current_density, cathode.c:673-715 */
void orc_set_current_density(orc_emitter *E, const spiffe_mesh *m, const spiffe_field_set *f)
{
  const long nr = m->nr;
  int k;
  for (k = 0; k < E->n; k++) {
    orc_cathode *c = &E->c[k];
    long iz = (long)((c->o.z_position - m->zmin) / m->dz + 1.5), ir = (long)((c->o.inner_radius + c->o.outer_radius) / 2 / m->dr);
    double Ez, wf;
    if (iz <= 0)
      iz = 1;
    Ez = m->constant_E[0];
    if (m->modes & SPIFFE_FL_TM_FIELDS)
      Ez += f->Ez[IDX(iz, ir)] + f->EzImposed[IDX(iz, ir)];
    if (Ez >= 0 && c->initial_vz <= 0)
      continue;
    if (c->o.temperature > 0 && c->o.work_function) {
      wf = 0.012 * sqrt(fabs(Ez * 1e-5));
      if (wf > c->o.work_function)
        wf = c->o.work_function;
      c->current_density = 60e4 * sq(c->o.temperature) *
                           exp(-(c->o.work_function - wf) / (c->o.temperature * SPIFFE_KB_MKS / SPIFFE_E_MKS));
    } else if (c->o.field_emission)
      c->current_density = field_emission_J(Ez, c->o.field_emission_beta, c->o.work_function);
  }
}

static double profile_value(const spiffe_cathode_options *o, double t)
{
  long lo = 0, hi = o->n_profile - 1, mid;
  if (t <= o->profile_t[0])
    return o->profile_A[0];
  if (t >= o->profile_t[hi])
    return o->profile_A[hi];
  while (hi - lo > 1) {
    mid = (lo + hi) / 2;
    if (o->profile_t[mid] <= t)
      lo = mid;
    else
      hi = mid;
  }
  return o->profile_A[lo] + (o->profile_A[hi] - o->profile_A[lo]) / (o->profile_t[hi] - o->profile_t[lo]) * (t - o->profile_t[lo]);
}

static void birth_common(spiffe_beam_set *b, long ip, const orc_cathode *c, double r, double time)
{
  double gamma;
  b->particleID[ip] = b->nextParticleID++;
  b->rmin[ip] = b->zmin[ip] = DBL_MAX;
  b->rmax[ip] = b->zmax[ip] = -DBL_MAX;
  b->z[ip] = b->z0[ip] = c->o.z_position;
  b->r[ip] = b->r0[ip] = r;
  b->t0[ip] = time;
  b->generation[ip] = 0;
  b->Q[ip] = c->Q;
  b->vz[ip] = c->initial_vz;
  b->vr[ip] = 0;
  b->vphi[ip] = c->o.initial_omega * b->r[ip];
  gamma = 1 / sqrt(1 - sq(b->vz[ip] / C_MKS) - sq(b->vr[ip] / C_MKS) - sq(b->vphi[ip] / C_MKS));
  b->pz[ip] = b->vz[ip] / C_MKS * gamma;
  b->pr[ip] = b->vr[ip] / C_MKS * gamma;
  b->r_pphi[ip] = b->r[ip] * b->vphi[ip] / C_MKS * gamma;
  b->status[ip] = SPIFFE_PART_ACTIVE;
  b->npActive++;
}

/* spread of births over the step, cathode.c:490-518 (and :561-592, :627-657) */
static void spread_over_dt(spiffe_beam_set *b, long ip, const orc_cathode *c, const spiffe_mesh *m,
                           const spiffe_field_set *f, double dte)
{
  const long nr = m->nr;
  long iz, ir;
  double Ez, Er, pphi, gamma;
  iz = (long)((c->o.z_position - m->zmin) / m->dz);
  if (iz <= 0)
    iz = 1;
  if (iz > m->nz)
    iz = m->nz;
  ir = (long)(b->r[ip] / m->dr);
  Ez = m->constant_E[0];
  if (m->modes & SPIFFE_FL_TM_FIELDS)
    Ez = f->Ez[IDX(iz, ir)] + f->EzImposed[IDX(iz, ir)];
  ir += 1;
  iz -= 1;
  Er = m->constant_E[1];
  if (m->modes & SPIFFE_FL_TM_FIELDS)
    Er = f->Er[IDX(iz, ir)] + f->ErImposed[IDX(iz, ir)];
  b->t0[ip] -= dte;
  pphi = (b->r[ip] ? b->r_pphi[ip] / b->r[ip] : 0);
  b->z[ip] += b->vz[ip] * dte;
  b->z0[ip] = b->z[ip];
  b->r[ip] += b->vr[ip] * dte;
  b->r0[ip] = b->r[ip];
  b->pr[ip] += dte * c->QoMC * Er / c->o.stiffness;
  b->pz[ip] += dte * c->QoMC * Ez / c->o.stiffness;
  gamma = sqrt(sq(b->pz[ip]) + sq(b->pr[ip]) + sq(pphi) + 1);
  b->vz[ip] = C_MKS * b->pz[ip] / gamma;
  b->vr[ip] = C_MKS * b->pr[ip] / gamma;
}

/* emit_electrons_from_cathode, cathode.c:239-671.  Returns the number of
 * births, or -1 when the particle arrays would overflow. */
long orc_emit(orc_emitter *E, const spiffe_mesh *m, const spiffe_field_set *f, spiffe_beam_set *b)
{
  long born = 0;
  int k;
  for (k = 0; k < E->n; k++) {
    orc_cathode *c = &E->c[k];
    long ib, ip, np_new, total, ir;
    double area, r_min, r_max, profile_factor, fnumber, dr2, totalNominal, total_area, totalf;
    if (c->number_per_step == 0 && c->electrons_per_macroparticle == 0)
      continue;
    if (c->start_step == -1) {
      /* first call: macroparticle charge and annulus bins, :271-347 */
      if (c->current_density <= 1. / sqrt(DBL_MAX))
        continue;
      c->ref_current_density = c->current_density;
      if (c->o.autophase) {
        c->stop_time = (c->stop_time - c->start_time) + m->time + c->o.time_offset;
        c->start_time = m->time + c->o.time_offset;
      }
      c->inner_r2 = sq(c->o.inner_radius);
      c->outer_r2 = sq(c->o.outer_radius);
      if ((area = PI * (c->outer_r2 - c->inner_r2)) != 0) {
        if (c->electrons_per_macroparticle) {
          c->number_per_step = area * m->dt * c->current_density / (SPIFFE_E_MKS * c->electrons_per_macroparticle);
          if (c->number_per_step == 0)
            continue;
        } else
          c->electrons_per_macroparticle = area * m->dt * c->current_density / (SPIFFE_E_MKS * c->number_per_step);
      } else {
        c->correction_interval = 0;
        c->n_bins = 1;
      }
      c->start_step = (int64_t)((c->start_time - m->start_time) / m->dt);
      if (c->stop_time && c->stop_time > m->start_time)
        c->stop_step = (int64_t)((c->stop_time - m->start_time) / m->dt);
      else
        c->stop_step = LONG_MAX;
      c->Q = -SPIFFE_E_MKS * c->electrons_per_macroparticle;
      c->n_bins = (long)((c->o.outer_radius - c->o.inner_radius) / m->dr + 1);
      c->distribution = calloc((size_t)c->n_bins, sizeof(long));
      c->deficit = calloc((size_t)c->n_bins, sizeof(long));
      c->area = calloc((size_t)c->n_bins, sizeof(double));
      c->rmin = calloc((size_t)c->n_bins, sizeof(double));
      c->totalArea = 0;
      for (ib = 0; ib < c->n_bins; ib++) {
        ir = (long)(c->o.inner_radius / m->dr + ib);
        if (ir == 0) {
          r_max = m->dr / 2;
          c->area[ib] = sq(r_max) * PI;
          c->rmin[ib] = 0;
        } else {
          r_min = m->dr * (ir - 0.5);
          r_max = m->dr * (ir + 0.5);
          c->area[ib] = PI * (sq(r_max) - sq(r_min));
          c->rmin[ib] = r_min;
          c->totalArea += c->area[ib];
        }
      }
    }
    profile_factor = 1;
    if (c->o.n_profile) {
      if (m->time >= c->o.profile_t[0] && m->time <= c->o.profile_t[c->o.n_profile - 1])
        profile_factor = profile_value(&c->o, m->time);
      else
        profile_factor = 0;
    }
    if (c->start_step > m->time_step || c->stop_step < m->time_step)
      continue;
    if (c->step_emission_started < 0)
      c->step_emission_started = m->time_step;

    /* birth count, :370-422 */
    dr2 = (c->outer_r2 - c->inner_r2) / c->number_per_step;
    total_area = c->totalArea;
    totalf = totalNominal = c->number_per_step * (c->current_density / c->ref_current_density);
    total = (long)totalf; /* overwritten below in every branch */
    np_new = b->np;
    if (c->correction_interval && m->time_step % c->correction_interval == 0) {
      total = 0;
      for (ib = 0; ib < c->n_bins; ib++) {
        if ((c->deficit[ib] = (long)((m->time_step - c->step_emission_started + 1) * (c->area[ib] / total_area) *
                                         totalNominal +
                                     0.5) -
                              c->distribution[ib]) <= 0)
          c->deficit[ib] = 0;
        total += c->deficit[ib];
      }
    } else if (c->zoned_emission) {
      total = 0;
      for (ib = 0; ib < c->n_bins; ib++) {
        if (total_area) {
          fnumber = profile_factor * (c->area[ib] / total_area) * totalNominal;
          if (fnumber > 1) {
            c->deficit[ib] = (long)fnumber;
            fnumber -= c->deficit[ib];
          } else
            c->deficit[ib] = 0;
          if (fnumber && fnumber > orc_rng_next(&E->rng))
            c->deficit[ib] += 1;
          total += c->deficit[ib];
        }
      }
    } else {
      fnumber = totalf * profile_factor;
      total = (long)fnumber;
      fnumber -= (long)fnumber;
      if (fnumber && fnumber > orc_rng_next(&E->rng))
        total += 1;
    }
    if ((np_new += total) < 0)
      return -1;
    if (np_new > b->capacity)
      return -1;
    if (total) {
      if (c->correction_interval) {
        /* zone by zone, :460-527 */
        for (ib = 0; ib < c->n_bins; ib++) {
          for (ip = b->np; ip < b->np + c->deficit[ib]; ip++) {
            double r = sqrt(orc_rng_next(&E->rng) * c->area[ib] / PI + sq(c->rmin[ib]));
            birth_common(b, ip, c, r, m->time);
            if (c->o.spread_over_dt)
              spread_over_dt(b, ip, c, m, f, m->dt * (ip - b->np) / (1.0 * c->deficit[ib]));
          }
          c->distribution[ib] += c->deficit[ib];
          b->np = ip;
        }
      } else if (!c->o.discretize_radii) {
        /* uniform in r^2 over the annulus, :528-599 */
        for (ip = b->np; ip < b->np + total; ip++) {
          double rn = orc_rng_next(&E->rng);
          double r = sqrt(rn * (sq(c->o.outer_radius) - sq(c->o.inner_radius)) + sq(c->o.inner_radius));
          birth_common(b, ip, c, r, m->time);
          if (c->o.spread_over_dt)
            spread_over_dt(b, ip, c, m, f, m->dt * (ip - b->np) / (1.0 * total));
        }
        b->np = ip;
      } else {
        /* discrete radii, :600-659 */
        for (ip = b->np; ip < np_new; ip++) {
          double r = sqrt(c->inner_r2 + (ip - b->np + 1) * dr2);
          birth_common(b, ip, c, r, m->time);
          if (c->o.spread_over_dt)
            spread_over_dt(b, ip, c, m, f, m->dt * (ip - b->np) / (1.0 * (np_new - b->np)));
        }
      }
      b->QoMC = c->QoMC;
      b->np = np_new;
      b->stiffness = c->o.stiffness;
      born += total;
    }
  }
  return born;
}

/* ---------------------------------------------------------------- antenna */

/* add_antenna_excitation, antenna.c:113-157, for one antenna whose waveform
 * times already include time_offset.  *last_index is the reference's
 * per-antenna search cursor. */
void orc_antenna(const spiffe_mesh *m, spiffe_field_set *f, int direction, long istart, long iend, long iposition,
                 double current, double frequency, double phase, const double *t, const double *W, long n_pts,
                 long *last_index, double time)
{
  const long nr = m->nr;
  double J;
  long i;
  if (time <= t[0])
    J = W[0];
  else if (time > t[n_pts - 1] || *last_index >= (n_pts - 1))
    J = W[n_pts - 1];
  else {
    i = *last_index;
    while (i < n_pts - 2 && time >= t[i + 1])
      i++;
    *last_index = i;
    J = (W[i + 1] - W[i]) / (t[i + 1] - t[i]) * (time - t[i]) + W[i];
  }
  J *= current * sin(PIx2 * frequency * time + phase);
  if (direction == 0)
    for (i = istart; i <= iend; i++)
      f->Jz[IDX(i, iposition)] += J;
  else if (direction == 1)
    for (i = istart; i <= iend; i++)
      f->Jr[IDX(iposition, i)] += J;
  else
    for (i = istart; i <= iend; i++)
      f->Jphi[IDX(i, iposition)] += J;
}

/* -------------------------------------------------------- diagnostics */

/* kinetic_energy, status_pr.c:342-359 */
double orc_kinetic_energy(const spiffe_beam_set *b)
{
  long ip;
  double sum = 0;
  if (!b->np)
    return 0.0;
  for (ip = 0; ip < b->np; ip++)
    sum += sqrt(1 + sq(b->pz[ip]) + sq(b->pr[ip]) + sq(b->r[ip] ? b->r_pphi[ip] / b->r[ip] : 0));
  return b->stiffness * SPIFFE_ME_MKS * sq(C_MKS) * (sum - b->np);
}

/* field_energy (TM part), status_pr.c:361-452, with the annulus areas of
 * calculate_areas, integrate.c:689-706 */
void orc_field_energy(const spiffe_mesh *m, const spiffe_field_set *f, double *out)
{
  const long nz = m->nz, nr = m->nr;
  const double dz = m->dz, dr2 = sq(m->dr);
  long iz, ir;
  double sum, area_c, area_o;
  out[0] = out[1] = 0;
  if (!(m->modes & SPIFFE_FL_TM_FIELDS))
    return;
  for (ir = 0; ir < nr; ir++) {
    sum = 0;
    area_c = ir ? PIx2 * ir * dr2 : PI * dr2 / 4;
    for (iz = 1; iz < nz; iz++)
      if (!(f->flags[IDX(iz, ir)] & SPIFFE_FL_EZ_ZERO))
        sum += sq(f->Ez[IDX(iz, ir)]);
    out[0] += sum * area_c * dz * EPS0 / 2;
  }
  for (ir = 1; ir < nr; ir++) {
    sum = 0;
    area_o = PI * (2 * ir - 1) * dr2;
    for (iz = 0; iz < nz; iz++)
      if (!(f->flags[IDX(iz, ir)] & SPIFFE_FL_ER_ZERO))
        sum += sq(f->Er[IDX(iz, ir)]);
    out[0] += sum * area_o * dz * EPS0 / 2;
  }
  for (ir = 1; ir < nr; ir++) {
    sum = 0;
    area_o = PI * (2 * ir - 1) * dr2;
    for (iz = 1; iz < nz; iz++)
      if (!(f->flags[IDX(iz, ir)] & SPIFFE_FL_BPHI_ZERO))
        sum += sq(f->Bphi2[IDX(iz, ir)]);
    out[1] += sum * area_o * dz / (2 * MU0);
  }
}

/* ----------------------------------------------------------- full steps */

/* One run of the perform_integration loop (integrate.c:134-194) on the
 * checked commands: emission, J zero and deposit, antenna, Poisson
 * correction, FDTD, push, current-density update.  The caller owns the
 * emitter, antenna and Poisson state across calls. */
typedef struct orc_run_state {
  orc_emitter emitter;
  int32_t space_charge;
  spiffe_push_options push;
  spiffe_poisson_options poisson;
  int64_t pc_start_step;
  double last_imposed_factor;
  /* one antenna */
  int32_t has_antenna, antenna_direction;
  long antenna_istart, antenna_iend, antenna_iposition, antenna_npts, antenna_last;
  double antenna_current, antenna_frequency, antenna_phase;
  const double *antenna_t, *antenna_W;
} orc_run_state;

orc_run_state *orc_run_new(void)
{
  orc_run_state *s = calloc(1, sizeof(orc_run_state));
  s->pc_start_step = -1;
  s->last_imposed_factor = -1;
  s->push.z_forces_start = -1;
  return s;
}

void orc_run_free(orc_run_state *s) { free(s); }
orc_emitter *orc_run_emitter(orc_run_state *s) { return &s->emitter; }

void orc_run_configure(orc_run_state *s, int32_t space_charge, const spiffe_push_options *push,
                       const spiffe_poisson_options *poisson)
{
  s->space_charge = space_charge;
  s->push = *push;
  if (poisson)
    s->poisson = *poisson;
}

void orc_run_antenna(orc_run_state *s, int32_t direction, long istart, long iend, long iposition, double current,
                     double frequency, double phase, const double *t, const double *W, long n_pts)
{
  s->has_antenna = 1;
  s->antenna_direction = direction;
  s->antenna_istart = istart;
  s->antenna_iend = iend;
  s->antenna_iposition = iposition;
  s->antenna_current = current;
  s->antenna_frequency = frequency;
  s->antenna_phase = phase;
  s->antenna_t = t;
  s->antenna_W = W;
  s->antenna_npts = n_pts;
  s->antenna_last = 0;
}

/* setup before the loop, integrate.c:125-133 */
void orc_run_begin(orc_run_state *s, const spiffe_mesh *m, spiffe_field_set *f, const spiffe_beam_set *b,
                   spiffe_poisson_report *rep)
{
  orc_imposed_efield(m, f, &s->poisson, 1, &s->last_imposed_factor, NULL);
  orc_poisson_correction(m, f, b, s->space_charge, &s->poisson, &s->pc_start_step, rep);
  orc_set_current_density(&s->emitter, m, f);
}

long orc_run_step(orc_run_state *s, spiffe_mesh *m, spiffe_field_set *f, spiffe_beam_set *b, spiffe_screen_set *screens,
                  int n_screens, spiffe_poisson_report *rep)
{
  long lost;
  if (m->imposed_ramp_time > 0)
    orc_imposed_efield(m, f, &s->poisson, 0, &s->last_imposed_factor, NULL);
  m->time = m->time_step * m->dt + m->start_time;
  if (orc_emit(&s->emitter, m, f, b) < 0)
    return -1;
  orc_zero_currents(m, f);
  if (s->space_charge)
    orc_deposit(m, f, b);
  if (s->has_antenna)
    orc_antenna(m, f, s->antenna_direction, s->antenna_istart, s->antenna_iend, s->antenna_iposition,
                s->antenna_current, s->antenna_frequency, s->antenna_phase, s->antenna_t, s->antenna_W,
                s->antenna_npts, &s->antenna_last, m->time + m->dt / 2);
  orc_poisson_correction(m, f, b, s->space_charge, &s->poisson, &s->pc_start_step, rep);
  orc_advance_fields(m, f);
  lost = orc_advance_particles(m, f, b, screens, n_screens, &s->push);
  orc_set_current_density(&s->emitter, m, f);
  m->time_step++;
  return lost;
}
