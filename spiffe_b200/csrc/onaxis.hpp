// spiffe_b200/csrc/onaxis.hpp -- add_on_axis_fields on the host.
//
// An on-axis RF field is an Ez(z) table that the push expands off axis to
// third order (addOffAxisExpansionFields, onAxisFields.c:208-268, restated
// as onaxis_expand in common.cuh).  This header holds the set-up the
// reference does once per definition (process_on_axis_field_definition,
// onAxisFields.c:18-172): the z offset, the monotonic check, the scaling to
// the requested peak and three central-difference derivatives
// (take_derivative, onAxisFields.c:174-204), plus the per-step sine and
// cosine terms, which the host computes once per push so the device never
// evaluates them.  The runtime and the command session both use it.
#pragma once

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/spiffe_b200_constants.h"
#include "common.cuh"

struct OnAxisProfile {
  std::vector<double> z, Ez, D1, D2, D3;
  double frequency = 0, phase = 0; // phase in radians
  int order = 3;

  double omega() const { return frequency * SPIFFE_PIx2; }
  OnAxisField view() const
  {
    return {z.data(), Ez.data(), D1.data(), D2.data(), D3.data(), (int)z.size(), order, omega() / SPIFFE_C_MKS};
  }
  // sin(omega t + phase) and omega / c^2 cos(omega t + phase); both cosine
  // and sine are 1 for the profile written to fields_used
  // (onAxisFields.c:229-238)
  void terms(double t, bool profile, double &sin_wt, double &bf) const
  {
    const double w = omega();
    double cos_wt;
    if (profile) {
      sin_wt = cos_wt = 1;
    } else {
      sin_wt = std::sin(w * t + phase);
      cos_wt = std::cos(w * t + phase);
    }
    bf = w / (SPIFFE_C_MKS * SPIFFE_C_MKS) * cos_wt;
  }
};

// take_derivative (onAxisFields.c:174-204): central differences inside,
// two-point differences at the ends.  The equispacing test is the caller's.
inline void onaxis_derivative(std::vector<double> &dF, const std::vector<double> &F, const std::vector<double> &z)
{
  const size_t n = z.size();
  dF.assign(n, 0.0);
  for (size_t i = 1; i + 1 < n; i++)
    dF[i] = (F[i + 1] - F[i - 1]) / (z[i + 1] - z[i - 1]);
  dF[0] = (F[1] - F[0]) / (z[1] - z[0]);
  dF[n - 1] = (F[n - 1] - F[n - 2]) / (z[n - 1] - z[n - 2]);
}

// The set-up of one definition (onAxisFields.c:49-128).  Returns "" on
// success, else the reference's message for the error.  Ez_peak = 0 is the
// caller's case (the reference ignores such a field with a warning).
inline std::string onaxis_prepare(OnAxisProfile &p, const double *z, const double *Ez, int64_t n, double z_offset,
                                  double Ez_peak, double frequency, double phase_rad, int64_t order)
{
  if (frequency < 0)
    return "frequency is negative";
  if (order < 0 || order > 3)
    return "expansion_order must by on [0, 3]";
  if (n <= 4)
    return "Too few points in file (need at least 4)";
  p.frequency = frequency;
  p.order = (int)order;
  p.phase = phase_rad;
  p.z.assign(z, z + n);
  p.Ez.assign(Ez, Ez + n);
  for (double &v : p.z)
    v += z_offset;
  for (int64_t i = 0; i + 1 < n; i++)
    if (p.z[i + 1] <= p.z[i])
      return "Data points are not monotonically increasing in z.";
  // scale to the requested peak |Ez| (:94-102)
  double Emin = p.Ez[0], Emax = p.Ez[0];
  for (double v : p.Ez) {
    if (v < Emin)
      Emin = v;
    if (v > Emax)
      Emax = v;
  }
  Emin = std::fabs(Emin);
  Emax = std::fabs(Emax);
  if (Emax < Emin)
    Emax = Emin;
  if (Emax > 0)
    for (double &v : p.Ez)
      v *= Ez_peak / Emax;
  // equispacing, checked to 1e-4 of the mean spacing (:180-195)
  double dz_min = p.z[1] - p.z[0], dz_max = dz_min;
  for (int64_t i = 2; i < n; i++) {
    const double dz = p.z[i] - p.z[i - 1];
    if (dz < dz_min)
      dz_min = dz;
    if (dz > dz_max)
      dz_max = dz;
  }
  if ((dz_max - dz_min) / ((dz_max + dz_min) / 2) > 1e-4)
    return "points are not equispaced with sufficient accuracy";
  onaxis_derivative(p.D1, p.Ez, p.z);
  onaxis_derivative(p.D2, p.D1, p.z);
  onaxis_derivative(p.D3, p.D2, p.z);
  return "";
}

// Every profile's contribution at (z, r, t), added into Ez, Er, Bphi as the
// reference adds it (straight into the caller's values).
inline void onaxis_eval(const std::vector<OnAxisProfile> &ps, double z, double r, double t, bool profile, double &Ez,
                        double &Er, double &Bphi)
{
  std::vector<OnAxisField> v;
  std::vector<double> s(ps.size()), bf(ps.size());
  for (size_t i = 0; i < ps.size(); i++) {
    v.push_back(ps[i].view());
    ps[i].terms(t, profile, s[i], bf[i]);
  }
  onaxis_expand(v.data(), (int)v.size(), s.data(), bf.data(), z, r, Ez, Er, Bphi);
}
