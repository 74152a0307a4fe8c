"""ctypes mirror of include/spiffe_b200_types.h and numpy-backed containers.

The C-ABI of libspiffe_b200 takes plain structs of scalars and pointers.  This
module defines the matching ctypes Structures and small containers that own
the numpy arrays a struct points into, so the same state can be handed to the
CUDA library (which copies it to the device) or to any other C routine that
speaks this ABI.  Arrays are contiguous (nz+1) x (nr+1) float64 blocks indexed
[iz, ir], the layout of the reference's zarray_2d rows (spiffe.h:60-71).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

# mode bits (spiffe.h:50-56)
FL_TM_FIELDS = 1
FL_TE_FIELDS = 2
FL_SPACE_CHARGE = 4
FL_RADIAL_INTERP = 8
FL_LONGIT_INTERP = 16
FL_RADIAL_SMEAR = 32
FL_LONGIT_SMEAR = 64

# metal flags (spiffe.h:90-100)
FL_IS_SURFACE = 1
FL_IS_INSIDE = 2
FL_EZ_ZERO = 4
FL_ER_ZERO = 8
FL_IS_VACUUM = 16
FL_BPHI_ZERO = 32
FL_EPHI_ZERO = 64
FL_BZ_ZERO = 128
FL_BR_ZERO = 256
FL_IS_METAL = FL_IS_SURFACE | FL_IS_INSIDE
FL_LAST_ACTIVE_PT = 512

DIRICHLET, NEUMANN = 0, 1
PART_ACTIVE, PART_LOST = 1, 2

COMPACT_REFERENCE, COMPACT_SWAP, COMPACT_ANY = 0, 1, 2
SCREEN_REFERENCE, SCREEN_PARTICLE = 0, 1

D = C.POINTER(C.c_double)
I16 = C.POINTER(C.c_int16)
I32 = C.POINTER(C.c_int32)
U64 = C.POINTER(C.c_uint64)


class Mesh(C.Structure):
    _fields_ = [
        ("nz", C.c_int32), ("nr", C.c_int32),
        ("zmin", C.c_double), ("zmax", C.c_double), ("rmax", C.c_double),
        ("dz", C.c_double), ("dr", C.c_double),
        ("lower_bc", C.c_int32), ("upper_bc", C.c_int32),
        ("right_bc", C.c_int32), ("left_bc", C.c_int32),
        ("modes", C.c_uint32),
        ("dt", C.c_double), ("start_time", C.c_double), ("time", C.c_double),
        ("time_step", C.c_int64),
        ("constant_E", C.c_double * 3), ("constant_B", C.c_double * 3),
        ("turn_off", C.c_int16 * 6),
        ("has_solenoid", C.c_int32),
        ("imposed_ramp_time", C.c_double), ("imposed_flat_top_time", C.c_double),
    ]


FIELD_NAMES = ["Ez", "Er", "Bphi", "Bphi2", "Jz", "Jr", "Ephi", "Jphi", "Br", "Br2",
               "Bz", "Bz2", "EzImposed", "ErImposed", "PsiImposed", "BzImposed",
               "BrImposed", "Psi", "Q"]


class FieldSet(C.Structure):
    _fields_ = [("flags", I16)] + [(n, D) for n in FIELD_NAMES]


BEAM_DOUBLES = ["z", "r", "pz", "pr", "r_pphi", "vz", "vr", "vphi", "Q",
                "r0", "z0", "t0", "rmin", "rmax", "zmin", "zmax"]


class BeamSet(C.Structure):
    _fields_ = [
        ("np", C.c_int64), ("npActive", C.c_int64), ("capacity", C.c_int64),
        ("nextParticleID", C.c_int32),
        ("QoMC", C.c_double), ("stiffness", C.c_double),
    ] + [(n, D) for n in BEAM_DOUBLES] + [
        ("particleID", I32), ("generation", I16), ("status", U64)]


SCREEN_COLUMNS = ["r", "pz", "pr", "pphi", "t", "q", "r0", "t0"]


class ScreenSet(C.Structure):
    _fields_ = [
        ("z_position", C.c_double), ("direction", C.c_int32),
        ("nb", C.c_int64), ("capacity", C.c_int64),
        ("col", D * 8),
        ("rmin", D), ("rmax", D), ("zmin", D), ("zmax", D),
        ("generation", I16), ("particleID", I32)]


class PushOptions(C.Structure):
    _fields_ = [
        ("z_forces_start", C.c_double),
        ("tb_electrons_per_macroparticle", C.c_double),
        ("tb_z_force", C.c_double), ("tb_r_force", C.c_double),
        ("tb_z_start_deceleration", C.c_double), ("tb_r_start_deceleration", C.c_double),
        ("compaction", C.c_int32), ("screen_momentum", C.c_int32)]


class PoissonOptions(C.Structure):
    _fields_ = [
        ("start_time", C.c_double), ("step_interval", C.c_int64),
        ("accuracy", C.c_double), ("error_charge_threshold", C.c_double),
        ("maximum_iterations", C.c_int64), ("verbosity", C.c_int32),
        ("guess_code", C.c_int32)]


class PoissonReport(C.Structure):
    _fields_ = [
        ("ran", C.c_int32), ("iterations", C.c_int64),
        ("Qreal", C.c_double), ("Qerror", C.c_double), ("Qsurface", C.c_double),
        ("residual", C.c_double), ("driving", C.c_double)]


class CathodeOptions(C.Structure):
    _fields_ = [
        ("z_position", C.c_double), ("inner_radius", C.c_double), ("outer_radius", C.c_double),
        ("current_density", C.c_double), ("temperature", C.c_double), ("work_function", C.c_double),
        ("field_emission", C.c_int32), ("field_emission_beta", C.c_double),
        ("electrons_per_macroparticle", C.c_double),
        ("start_time", C.c_double), ("stop_time", C.c_double), ("time_offset", C.c_double),
        ("autophase", C.c_int32),
        ("number_per_step", C.c_double), ("initial_pz", C.c_double),
        ("initial_omega", C.c_double), ("stiffness", C.c_double),
        ("discretize_radii", C.c_int32), ("random_number_seed", C.c_int32),
        ("distribution_correction_interval", C.c_int32), ("spread_over_dt", C.c_int32),
        ("zoned_emission", C.c_int32), ("n_profile", C.c_int32),
        ("profile_t", D), ("profile_A", D)]


class TestBeamOptions(C.Structure):
    _fields_ = [
        ("start_time", C.c_double), ("stop_time", C.c_double),
        ("initial_z", C.c_double), ("initial_r", C.c_double),
        ("initial_pz", C.c_double), ("initial_pr", C.c_double), ("initial_rpphi", C.c_double),
        ("electrons_per_macroparticle", C.c_double)]


class SolenoidOptions(C.Structure):
    _fields_ = [
        ("radius", C.c_double), ("evaluation_radius_limit", C.c_double), ("z_start", C.c_double),
        ("z_end", C.c_double), ("current", C.c_double), ("Bz_peak", C.c_double),
        ("turns", C.c_int64), ("symmetry", C.c_int32), ("bucking", C.c_int32), ("z_buck", C.c_double)]


def _dptr(a):
    return a.ctypes.data_as(D) if a is not None else None


def push_options(compaction=COMPACT_REFERENCE, screen_momentum=SCREEN_REFERENCE,
                 z_forces_start=-1.0, **test_beam):
    o = PushOptions()
    o.z_forces_start = z_forces_start
    o.tb_electrons_per_macroparticle = test_beam.get("electrons_per_macroparticle", 0.0)
    o.tb_z_force = test_beam.get("z_force", 0.0)
    o.tb_r_force = test_beam.get("r_force", 0.0)
    o.tb_z_start_deceleration = test_beam.get("z_start_deceleration", 1.7976931348623157e308)
    o.tb_r_start_deceleration = test_beam.get("r_start_deceleration", 1.7976931348623157e308)
    o.compaction = compaction
    o.screen_momentum = screen_momentum
    return o


def poisson_options(step_interval=0, accuracy=1e-6, maximum_iterations=1000,
                    error_charge_threshold=0.0, start_time=0.0, guess_code=0, verbosity=0):
    o = PoissonOptions()
    o.start_time = start_time
    o.step_interval = step_interval
    o.accuracy = accuracy
    o.error_charge_threshold = error_charge_threshold
    o.maximum_iterations = maximum_iterations
    o.verbosity = verbosity
    o.guess_code = guess_code
    return o


class Fields:
    """Mesh description plus the numpy arrays of one problem."""

    def __init__(self, nz, nr, zmin, zmax, rmax, modes=FL_TM_FIELDS | FL_RADIAL_INTERP | FL_LONGIT_INTERP,
                 left_bc=NEUMANN, right_bc=NEUMANN, lower_bc=DIRICHLET, upper_bc=NEUMANN, flags=None):
        self.mesh = Mesh()
        m = self.mesh
        m.nz, m.nr = nz, nr
        m.zmin, m.zmax, m.rmax = zmin, zmax, rmax
        m.dz = (zmax - zmin) / (nz - 1)
        m.dr = rmax / (nr - 1)
        m.lower_bc, m.upper_bc, m.right_bc, m.left_bc = lower_bc, upper_bc, right_bc, left_bc
        m.modes = modes
        m.imposed_flat_top_time = 1.0
        self.shape = (nz + 1, nr + 1)
        self.flags = np.zeros(self.shape, np.int16) if flags is None else np.ascontiguousarray(flags, np.int16)
        self.a = {}
        te = bool(modes & FL_TE_FIELDS)
        for n in FIELD_NAMES:
            if n in ("Ephi", "Jphi", "Br", "Br2", "Bz", "Bz2") and not te:
                continue
            if n in ("BzImposed", "BrImposed"):
                continue
            self.a[n] = np.zeros(self.shape)

    def __getitem__(self, k):
        return self.a[k]

    def __setitem__(self, k, v):
        arr = np.ascontiguousarray(v, dtype=np.float64)
        assert arr.shape == self.shape, (k, arr.shape, self.shape)
        self.a[k] = arr.copy()
        if k == "BzImposed":
            self.mesh.has_solenoid = 1

    def copy(self):
        f = Fields.__new__(Fields)
        f.mesh = Mesh.from_buffer_copy(self.mesh)
        f.shape = self.shape
        f.flags = self.flags.copy()
        f.a = {k: v.copy() for k, v in self.a.items()}
        return f

    def c(self):
        s = FieldSet()
        s.flags = self.flags.ctypes.data_as(I16)
        for n in FIELD_NAMES:
            setattr(s, n, _dptr(self.a.get(n)))
        return s


class Beam:
    """Structure-of-arrays beam with a fixed capacity."""

    def __init__(self, capacity):
        self.capacity = int(capacity)
        self.np = 0
        self.npActive = 0
        self.nextParticleID = 1
        self.QoMC = 0.0
        self.stiffness = 1.0
        self.a = {n: np.zeros(self.capacity) for n in BEAM_DOUBLES}
        self.particleID = np.zeros(self.capacity, np.int32)
        self.generation = np.zeros(self.capacity, np.int16)
        self.status = np.zeros(self.capacity, np.uint64)

    def __getitem__(self, k):
        if k == "particleID":
            return self.particleID[: self.np]
        if k == "generation":
            return self.generation[: self.np]
        if k == "status":
            return self.status[: self.np]
        return self.a[k][: self.np]

    def set(self, n, **arrays):
        assert n <= self.capacity
        self.np = n
        for k, v in arrays.items():
            if k == "particleID":
                self.particleID[:n] = v
            elif k == "generation":
                self.generation[:n] = v
            elif k == "status":
                self.status[:n] = v
            else:
                self.a[k][:n] = v

    def copy(self):
        b = Beam.__new__(Beam)
        b.capacity, b.np, b.npActive, b.nextParticleID = self.capacity, self.np, self.npActive, self.nextParticleID
        b.QoMC, b.stiffness = self.QoMC, self.stiffness
        b.a = {k: v.copy() for k, v in self.a.items()}
        b.particleID, b.generation, b.status = self.particleID.copy(), self.generation.copy(), self.status.copy()
        return b

    def c(self):
        s = BeamSet()
        s.np, s.npActive, s.capacity = self.np, self.npActive, self.capacity
        s.nextParticleID = self.nextParticleID
        s.QoMC, s.stiffness = self.QoMC, self.stiffness
        for n in BEAM_DOUBLES:
            setattr(s, n, _dptr(self.a[n]))
        s.particleID = self.particleID.ctypes.data_as(I32)
        s.generation = self.generation.ctypes.data_as(I16)
        s.status = self.status.ctypes.data_as(U64)
        return s

    def take(self, s):
        """Adopt the counters a C routine wrote back into BeamSet `s`."""
        self.np, self.npActive, self.nextParticleID = s.np, s.npActive, s.nextParticleID
        self.QoMC, self.stiffness = s.QoMC, s.stiffness


class Screen:
    """Append buffer of screen-crossing records."""

    def __init__(self, z_position, direction=1, capacity=1 << 16):
        self.z_position, self.direction, self.capacity = z_position, direction, int(capacity)
        self.nb = 0
        self.cols = {n: np.zeros(self.capacity) for n in SCREEN_COLUMNS + ["rmin", "rmax", "zmin", "zmax"]}
        self.generation = np.zeros(self.capacity, np.int16)
        self.particleID = np.zeros(self.capacity, np.int32)

    def c(self):
        s = ScreenSet()
        s.z_position, s.direction, s.nb, s.capacity = self.z_position, self.direction, self.nb, self.capacity
        for i, n in enumerate(SCREEN_COLUMNS):
            s.col[i] = _dptr(self.cols[n])
        for n in ("rmin", "rmax", "zmin", "zmax"):
            setattr(s, n, _dptr(self.cols[n]))
        s.generation = self.generation.ctypes.data_as(I16)
        s.particleID = self.particleID.ctypes.data_as(I32)
        return s

    def records(self):
        out = {n: v[: self.nb].copy() for n, v in self.cols.items()}
        out["particleID"] = self.particleID[: self.nb].copy()
        out["generation"] = self.generation[: self.nb].copy()
        return out


def screens_c(screens):
    arr = (ScreenSet * max(1, len(screens)))()
    for i, s in enumerate(screens):
        arr[i] = s.c()
    return arr


def screens_take(screens, arr):
    for i, s in enumerate(screens):
        s.nb = arr[i].nb
