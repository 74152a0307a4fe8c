"""Synthetic workloads of the benchmark configurations, as spiffe input.

Each builder returns spiffe namelist commands (the reference's command
surface: define_geometry with a boundary file of &po points, define_cathode,
define_screen, poisson_correction, integrate) plus any analytic initial field,
with the sizes, seeds and parameters of the configuration it names.  No
dataset is involved; every value is derived from the numbers below.
"""
from __future__ import annotations

import math

import numpy as np

C_MKS = 2.99792458e8
E_MKS = 1.602176634e-19


def po_lines(points):
    """&po boundary points: list of dicts of &po variables (geometry.nl:40-55)."""
    out = []
    for p in points:
        body = ", ".join(f"{k}={v!r}" if not isinstance(v, str) else f'{k}="{v}"' for k, v in p.items())
        out.append(f"&po {body} &end")
    return "\n".join(out) + "\n"


def pillbox_geo(R, L):
    """Closed PEC pillbox of radius R and length L with its axis on r=0."""
    return po_lines([dict(x=0.0, y=0.0), dict(x=0.0, y=R), dict(x=L, y=R), dict(x=L, y=0.0), dict(x=0.0, y=0.0)])


def dc_gun_geo(cathode_radius=5e-3, gap=10e-3, hole=3e-3, plate=0.2e-3, wall=20e-3, length=30e-3, voltage=300e3):
    """Axisymmetric DC gun: cathode plane at z=0 (0 V), anode plate at z=gap
    with a hole of radius `hole` at `voltage`, outer PEC wall of radius `wall`
    whose potential ramps linearly from 0 to `voltage` between cathode and
    anode (ramp_potential, grid_drawing.c draw_line startPotential), drift
    region to z=length.  The emitting disk (cathode_radius) is the cathode
    command's business, not the boundary's."""
    v = float(voltage)
    return po_lines([
        dict(x=0.0, y=0.0, potential=0.0),
        dict(x=0.0, y=wall, potential=0.0),
        dict(x=gap, y=wall, potential=v, ramp_potential=1),
        dict(x=gap, y=hole, potential=v),
        dict(x=gap + plate, y=hole, potential=v),
        dict(x=gap + plate, y=wall, potential=v),
        dict(x=length, y=wall, potential=v),
        dict(x=length, y=0.0, potential=v),
        dict(x=0.0, y=0.0, potential=0.0),
    ])


def gun16_geo(half_cell=17.5e-3, full_cell=52.5e-3, cavity_r=41e-3, iris_r=10e-3, iris_t=5e-3,
              pipe_r=10e-3, length=150e-3):
    """1.6-cell RF gun: a half cell (length `half_cell`) and a full cell (length
    `full_cell`), both of radius `cavity_r`, separated by an iris of radius
    `iris_r` and thickness `iris_t`, an exit iris of the same size, then a beam
    pipe of radius `pipe_r` out to z=`length`.  Cell lengths are measured
    between iris faces."""
    z1 = half_cell
    z2 = z1 + iris_t
    z3 = z2 + full_cell
    z4 = z3 + iris_t
    return po_lines([
        dict(x=0.0, y=0.0), dict(x=0.0, y=cavity_r),
        dict(x=z1, y=cavity_r), dict(x=z1, y=iris_r), dict(x=z2, y=iris_r), dict(x=z2, y=cavity_r),
        dict(x=z3, y=cavity_r), dict(x=z3, y=iris_r), dict(x=z4, y=iris_r), dict(x=z4, y=pipe_r),
        dict(x=length, y=pipe_r), dict(x=length, y=0.0), dict(x=0.0, y=0.0),
    ])


def geometry_command(nz, nr, zmin, zmax, rmax, boundary, **extra):
    args = dict(nz=nz, nr=nr, zmin=zmin, zmax=zmax, rmax=rmax)
    args.update(extra)
    body = ", ".join(f"{k}={v}" for k, v in args.items())
    return f'&define_geometry {body}, boundary="{boundary}" &end'


def namelist(group, **kw):
    parts = []
    for k, v in kw.items():
        parts.append(f'{k}="{v}"' if isinstance(v, str) else f"{k}={v!r}")
    return f"&{group} " + ", ".join(parts) + " &end"


def tm010_ez(nz, nr, dr, R, E0):
    """Ez = E0 J0(2.405 r/R) on the Ez nodes (r = ir*dr), uniform in z."""
    from scipy.special import j0, jn_zeros

    x01 = float(jn_zeros(0, 1)[0])
    r = np.arange(nr + 1) * dr
    prof = E0 * j0(x01 * r / R)
    prof[r > R] = 0.0
    return np.repeat(prof[None, :], nz + 1, axis=0)


class PillboxConfig:
    """Closed PEC pillbox: radius 40 mm (the 40.1 mm of the specification
    snapped to the 0.25 mm mesh), length 26 mm (26.2 mm snapped), 161 x 105
    nodes, TM010 standing wave of 80 MV/m at t=0, a 1 mm cathode on the z=0
    wall emitting 1 nC as 20,000 macroparticles with a Gaussian 3 ps rms time
    profile centred at RF phase 30 degrees, dt = 0.5 x Courant."""

    def __init__(self, nz=105, nr=161, R=0.040, L=0.026, E0=-80e6, charge=1e-9, n_macro=20000,
                 sigma_t=3e-12, cathode_radius=1e-3, seed=987654321, dt_factor=0.5, space_charge=1):
        self.nz, self.nr, self.R, self.L = nz, nr, R, L
        self.zmin, self.zmax, self.rmax = 0.0, L, R
        self.dz = L / (nz - 1)
        self.dr = R / (nr - 1)
        self.E0 = E0
        self.charge, self.n_macro, self.sigma_t = charge, n_macro, sigma_t
        self.cathode_radius, self.seed = cathode_radius, seed
        self.dt = dt_factor * min(self.dz, self.dr) / C_MKS / math.sqrt(2.0)
        self.space_charge = space_charge
        f = 2.405 * C_MKS / (2 * math.pi * R)
        self.t_centre = (30.0 / 360.0) / f
        self.epm = charge / E_MKS / n_macro

    def geo_text(self):
        return pillbox_geo(self.R, self.L)

    def geometry(self, boundary="pillbox.geo"):
        return geometry_command(self.nz, self.nr, self.zmin, self.zmax, self.rmax, boundary)

    def initial_ez(self):
        return tm010_ez(self.nz, self.nr, self.dr, self.R, self.E0)

    def profile(self, n=161, nsig=4.0):
        t = self.t_centre + np.linspace(-nsig, nsig, n) * self.sigma_t
        return t, np.exp(-0.5 * ((t - self.t_centre) / self.sigma_t) ** 2)

    def peak_current_density(self):
        return self.charge / (math.sqrt(2 * math.pi) * self.sigma_t * math.pi * self.cathode_radius ** 2)

    def cathode_options(self):
        from . import abi

        t, A = self.profile()
        self._profile = (np.ascontiguousarray(t), np.ascontiguousarray(A))
        o = abi.CathodeOptions()
        o.z_position = 0.0
        o.outer_radius = self.cathode_radius
        o.current_density = self.peak_current_density()
        o.electrons_per_macroparticle = self.epm
        o.stiffness = 1.0
        o.zoned_emission = 1
        o.random_number_seed = self.seed
        o.field_emission_beta = 1.0
        o.n_profile = len(t)
        o.profile_t = self._profile[0].ctypes.data_as(abi.D)
        o.profile_A = self._profile[1].ctypes.data_as(abi.D)
        return o

    def screen_z(self):
        return self.L - self.dz


class Gun16Config:
    """The 1.6-cell RF gun workload: half cell 17.5 mm and full cell 52.5 mm
    of radius 41 mm, 10 mm irises 5 mm thick, a 10 mm beam pipe to z=150 mm,
    mesh dr=dz=50 um (3001 x 821 nodes), dt = 0.5 x Courant.  Field: a
    pi-mode standing wave (TM010 profile in each cell, opposite signs) with
    100 MV/m on the cathode at t=0 and B=0.  Solenoid: Gaussian on-axis Bz,
    0.25 T peak at z=100 mm, sigma 20 mm, extended off axis to first order
    (Br = -r/2 dBz/dz).  Beam: 1 nC as 1,000,000 macroparticles from a 1 mm
    disk with a 2 ps rms Gaussian emission time, already emitted: a particle
    emitted tau before t=0 sits where uniform acceleration by the cathode
    field carries it.  Poisson correction every 20 steps (accuracy 1e-6, at
    most 1000 iterations)."""

    def __init__(self, nz=3001, nr=821, length=0.150, radius=0.041, n_macro=1_000_000, charge=1e-9,
                 sigma_t=2e-12, cathode_radius=1e-3, E_cathode=100e6, B_peak=0.25, B_z=0.100, B_sigma=0.020,
                 step_interval=20, seed=1234):
        self.nz, self.nr, self.length, self.radius = nz, nr, length, radius
        self.zmin, self.zmax, self.rmax = 0.0, length, radius
        self.dz = length / (nz - 1)
        self.dr = radius / (nr - 1)
        self.dt = 0.5 * min(self.dz, self.dr) / C_MKS / math.sqrt(2.0)
        self.n_macro, self.charge, self.sigma_t = n_macro, charge, sigma_t
        self.cathode_radius, self.E_cathode = cathode_radius, E_cathode
        self.B_peak, self.B_z, self.B_sigma = B_peak, B_z, B_sigma
        self.step_interval, self.seed = step_interval, seed

    def geo_text(self):
        return gun16_geo(pipe_r=10e-3, length=self.length, cavity_r=self.radius)

    def cell_spans(self):
        return [(0.0, 17.5e-3, -1.0), (22.5e-3, 75e-3, 1.0)]

    def initial_ez(self, flags):
        from scipy.special import j0, jn_zeros

        x01 = float(jn_zeros(0, 1)[0])
        nz, nr = self.nz, self.nr
        z = (np.arange(nz + 1) - 0.5) * self.dz + self.zmin  # Ez nodes, spiffe.h:60
        r = np.arange(nr + 1) * self.dr
        ez = np.zeros((nz + 1, nr + 1))
        prof = j0(x01 * r / self.radius)
        prof[r > self.radius] = 0
        for z0, z1, sign in self.cell_spans():
            sel = (z > z0) & (z < z1)
            ez[sel, :] = sign * prof[None, :]
        ez[(flags & 4) != 0] = 0.0  # FL_EZ_ZERO
        ez *= self.E_cathode / abs(ez[1, 0])
        return ez

    def solenoid(self):
        z = np.arange(self.nz + 1) * self.dz + self.zmin  # BzImposed nodes, spiffe.h:114
        r = np.arange(self.nr + 1) * self.dr
        bz0 = self.B_peak * np.exp(-0.5 * ((z - self.B_z) / self.B_sigma) ** 2)
        dbz = -bz0 * (z - self.B_z) / self.B_sigma ** 2
        bz = np.repeat(bz0[:, None], self.nr + 1, axis=1)
        br = -0.5 * r[None, :] * dbz[:, None]
        return bz, br

    def beam_arrays(self):
        rng = np.random.default_rng(self.seed)
        n = self.n_macro
        te = rng.normal(0.0, self.sigma_t, n)
        te = np.clip(te, -4 * self.sigma_t, 4 * self.sigma_t)
        tau = 4 * self.sigma_t - te
        kappa = E_MKS * self.E_cathode / (9.1093837015e-31 * C_MKS)
        pz = kappa * tau
        gamma = np.sqrt(1 + pz ** 2)
        z = C_MKS / kappa * (gamma - 1) + 1e-9
        r = self.cathode_radius * np.sqrt(rng.uniform(0, 1, n))
        vz = C_MKS * pz / gamma
        zeros = np.zeros(n)
        return dict(z=z, r=r, pz=pz, pr=zeros, r_pphi=zeros, vz=vz, vr=zeros, vphi=zeros,
                    Q=np.full(n, -self.charge / n), r0=r.copy(), z0=np.zeros(n), t0=-tau, rmin=r.copy(),
                    rmax=r.copy(), zmin=np.zeros(n), zmax=z.copy(), particleID=np.arange(1, n + 1, dtype=np.int32),
                    generation=np.zeros(n, np.int16), status=np.ones(n, np.uint64))

    def screen_z(self):
        return self.length - self.dz

    def state(self, capacity_factor=1.25):
        """Fields (flags and PsiImposed from the product's define_geometry,
        the analytic field, the solenoid) and the beam, as abi containers."""
        from . import abi, geometry

        modes = abi.FL_TM_FIELDS | abi.FL_RADIAL_INTERP | abi.FL_LONGIT_INTERP | abi.FL_SPACE_CHARGE
        f = geometry.fields_for(self.nz, self.nr, self.zmin, self.zmax, self.rmax, self.geo_text(), modes=modes)
        f.mesh.dt = self.dt
        f["Ez"] = self.initial_ez(f.flags)
        bz, br = self.solenoid()
        f["BzImposed"] = bz
        f["BrImposed"] = br
        arrays = self.beam_arrays()
        n = len(arrays["z"])
        b = abi.Beam(int(n * capacity_factor))
        b.set(n, **arrays)
        b.npActive, b.nextParticleID, b.QoMC, b.stiffness = n, n + 1, -E_MKS / (9.1093837015e-31 * C_MKS), 1.0
        return f, b

    def poisson(self):
        from . import abi

        return abi.poisson_options(step_interval=self.step_interval, accuracy=1e-6, maximum_iterations=1000)


class DcGunConfig:
    """The DC gun workload: cathode plane at z=0 (0 V), anode plate at z=10 mm
    with a 3 mm hole at 300 kV, an outer wall of radius 20 mm whose potential
    ramps between them, drift to z=30 mm (dc_gun_geo); mesh dr=dz=20 um (1501
    x 1001 nodes), dt = 0.5 x Courant.  Field: the imposed field of the
    electrodes' Laplace solve, which the integration's start computes
    (compute_imposed_Efield).  Beam: 0.5 nC as 4,000,000 macroparticles from a
    2 mm disk (inside the anode hole), emitted from rest uniformly over a
    100 ps flat top and already emitted: a particle emitted tau before t=0
    sits where uniform acceleration by the gap field (V/gap) carries it, or,
    past the anode, drifts with the gap's full energy.  Poisson correction
    every step (accuracy 1e-6, at most 1000 iterations)."""

    def __init__(self, nz=1501, nr=1001, length=0.030, radius=0.020, gap=0.010, voltage=300e3,
                 n_macro=4_000_000, charge=0.5e-9, flat_top=100e-12, cathode_radius=2e-3, seed=2024):
        self.nz, self.nr, self.length, self.radius = nz, nr, length, radius
        self.zmin, self.zmax, self.rmax = 0.0, length, radius
        self.dz = length / (nz - 1)
        self.dr = radius / (nr - 1)
        self.dt = 0.5 * min(self.dz, self.dr) / C_MKS / math.sqrt(2.0)
        self.gap, self.voltage = gap, voltage
        self.n_macro, self.charge, self.flat_top = n_macro, charge, flat_top
        self.cathode_radius, self.seed = cathode_radius, seed

    def geo_text(self):
        return dc_gun_geo(cathode_radius=self.cathode_radius, gap=self.gap, wall=self.radius, length=self.length,
                          voltage=self.voltage)

    def beam_arrays(self):
        rng = np.random.default_rng(self.seed)
        n = self.n_macro
        tau = rng.uniform(0.0, self.flat_top, n)
        kappa = E_MKS * (self.voltage / self.gap) / (9.1093837015e-31 * C_MKS)
        g_gap = 1 + E_MKS * self.voltage / (9.1093837015e-31 * C_MKS ** 2)  # gamma at the anode
        p_gap = math.sqrt(g_gap ** 2 - 1)
        tau_gap = p_gap / kappa  # time to cross the gap
        pz = np.minimum(kappa * tau, p_gap)
        gamma = np.sqrt(1 + pz ** 2)
        z = np.where(tau < tau_gap, C_MKS / kappa * (gamma - 1),
                     self.gap + C_MKS * p_gap / g_gap * (tau - tau_gap)) + 1e-9
        r = self.cathode_radius * np.sqrt(rng.uniform(0, 1, n))
        vz = C_MKS * pz / gamma
        zeros = np.zeros(n)
        return dict(z=z, r=r, pz=pz, pr=zeros, r_pphi=zeros, vz=vz, vr=zeros, vphi=zeros,
                    Q=np.full(n, -self.charge / n), r0=r.copy(), z0=np.zeros(n), t0=-tau, rmin=r.copy(),
                    rmax=r.copy(), zmin=np.zeros(n), zmax=z.copy(), particleID=np.arange(1, n + 1, dtype=np.int32),
                    generation=np.zeros(n, np.int16), status=np.ones(n, np.uint64))

    def screen_z(self):
        return self.length - self.dz

    def state(self, capacity_factor=1.25):
        """Fields (flags and electrode potentials from the product's
        define_geometry, no initial field) and the beam, as abi containers."""
        from . import abi, geometry

        modes = abi.FL_TM_FIELDS | abi.FL_RADIAL_INTERP | abi.FL_LONGIT_INTERP | abi.FL_SPACE_CHARGE
        f = geometry.fields_for(self.nz, self.nr, self.zmin, self.zmax, self.rmax, self.geo_text(), modes=modes)
        f.mesh.dt = self.dt
        arrays = self.beam_arrays()
        n = len(arrays["z"])
        b = abi.Beam(int(n * capacity_factor))
        b.set(n, **arrays)
        b.npActive, b.nextParticleID, b.QoMC, b.stiffness = n, n + 1, -E_MKS / (9.1093837015e-31 * C_MKS), 1.0
        return f, b

    def poisson(self):
        from . import abi

        return abi.poisson_options(step_interval=1, accuracy=1e-6, maximum_iterations=1000)

