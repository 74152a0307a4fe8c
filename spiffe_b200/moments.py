"""Exit-plane beam moments from screen records.

The reference writes screen crossings (r, pz, pr, pphi, t, q, ...;
screens.c:18-21) and leaves moments to external SDDS tools, so their
definitions are fixed here and shared by every comparison:

* transmitted charge: sum of q;
* mean kinetic energy: m c^2 <gamma - 1>, gamma = sqrt(1 + pz^2 + pr^2 + pphi^2);
* rms energy spread: the rms of m c^2 (gamma - 1);
* rms bunch length: sigma_t <beta_z> c;
* normalized rms emittance of the x projection of the axisymmetric beam:
  <x^2> = <r^2>/2, <px^2> = (<pr^2> + <pphi^2>)/2, <x px> = <r pr>/2,
  eps = sqrt(<x^2><px^2> - <x px>^2)  (momenta in units of m c).

All averages weight each record by |q| and are accumulated in float64.
"""
from __future__ import annotations

import numpy as np

MC2_EV = 0.51099895000e6
C_MKS = 2.99792458e8


def exit_moments(rec):
    q = np.abs(np.asarray(rec["q"], np.float64))
    n = len(q)
    if n == 0 or q.sum() == 0:
        return {"count": 0, "charge": 0.0, "mean_ke_ev": 0.0, "rms_energy_ev": 0.0, "bunch_length_m": 0.0,
                "emittance_m": 0.0}
    w = q / q.sum()
    pz, pr, pphi = (np.asarray(rec[k], np.float64) for k in ("pz", "pr", "pphi"))
    r, t = np.asarray(rec["r"], np.float64), np.asarray(rec["t"], np.float64)
    gamma = np.sqrt(1 + pz ** 2 + pr ** 2 + pphi ** 2)
    ke = MC2_EV * (gamma - 1)
    mean_ke = float(np.sum(w * ke))
    rms_e = float(np.sqrt(np.sum(w * (ke - mean_ke) ** 2)))
    tm = np.sum(w * t)
    sig_t = float(np.sqrt(np.sum(w * (t - tm) ** 2)))
    beta_z = float(np.sum(w * pz / gamma))
    x2 = np.sum(w * r ** 2) / 2
    px2 = (np.sum(w * pr ** 2) + np.sum(w * pphi ** 2)) / 2
    xpx = np.sum(w * r * pr) / 2
    eps = float(np.sqrt(max(x2 * px2 - xpx ** 2, 0.0)))
    return {"count": int(n), "charge": float(np.sum(np.asarray(rec["q"], np.float64))), "mean_ke_ev": mean_ke,
            "rms_energy_ev": rms_e, "bunch_length_m": sig_t * beta_z * C_MKS, "emittance_m": eps}


def relative_errors(a, b, keys=("charge", "mean_ke_ev", "rms_energy_ev", "bunch_length_m", "emittance_m")):
    out = {}
    for k in keys:
        den = abs(b[k])
        out[k] = abs(a[k] - b[k]) / den if den else abs(a[k] - b[k])
    return out
