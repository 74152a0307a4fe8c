"""Python binding of libspiffe_b200 (the CUDA implementation, C ABI).

`GpuInstance` mirrors the reference's per-step functions on one device-
resident problem: advance_field_solutions, add_particle_currents,
advance_particles, solve_poisson_cyl, add_poisson_correction and the whole
perform_integration loop.  State moves through abi.Fields / abi.Beam /
abi.Screen.  There is no fallback: if the shared library or a GPU is
missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspiffe_b200.so")

PRECISION_F64 = 0
PRECISION_SPLIT32 = 1
POISSON_SOR = 0
POISSON_MULTIGRID = 1
FDTD_AUTO = 0
FDTD_TWO_KERNELS = 1
FDTD_FUSED = 2

_lib = None
P = C.POINTER
H = C.c_void_p


class SpiffeGpuError(RuntimeError):
    pass


def load():
    """Loads libspiffe_b200.so (raises when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SpiffeGpuError(f"{LIB_PATH} is missing: build it with `make -C spiffe_b200/csrc`")
    lib = C.CDLL(LIB_PATH)
    M, F, B, S = P(abi.Mesh), P(abi.FieldSet), P(abi.BeamSet), P(abi.ScreenSet)
    sig = {
        "spiffe_gpu_last_error": ([], C.c_char_p),
        "spiffe_gpu_version": ([], C.c_char_p),
        "spiffe_gpu_create": ([M, P(C.c_int16), C.c_int32, C.c_int64, P(H)], C.c_int),
        "spiffe_gpu_destroy": ([H], C.c_int),
        "spiffe_gpu_set_mesh": ([H, M], C.c_int),
        "spiffe_gpu_get_mesh": ([H, M], C.c_int),
        "spiffe_gpu_upload_fields": ([H, F], C.c_int),
        "spiffe_gpu_download_fields": ([H, F], C.c_int),
        "spiffe_gpu_upload_beam": ([H, B], C.c_int),
        "spiffe_gpu_download_beam": ([H, B], C.c_int),
        "spiffe_gpu_set_deposit_order": ([H, C.c_int32], C.c_int),
        "spiffe_gpu_zero_current_arrays": ([H], C.c_int),
        "spiffe_gpu_advance_field_solutions": ([H], C.c_int),
        "spiffe_gpu_add_particle_currents": ([H], C.c_int),
        "spiffe_gpu_advance_particles": ([H, P(abi.PushOptions)], C.c_int),
        "spiffe_gpu_solve_poisson_cyl": ([H, C.c_int32, C.c_double, C.c_int64, P(C.c_int64)], C.c_int),
        "spiffe_gpu_add_poisson_correction": ([H, C.c_int32, P(abi.PoissonOptions), P(abi.PoissonReport)], C.c_int),
        "spiffe_gpu_compute_imposed_efield": ([H, P(abi.PoissonOptions), C.c_int32], C.c_int),
        "spiffe_gpu_add_screen": ([H, C.c_double, C.c_int32, C.c_int64], C.c_int),
        "spiffe_gpu_screen_count": ([H, C.c_int32, P(C.c_int64)], C.c_int),
        "spiffe_gpu_download_screen": ([H, C.c_int32, S], C.c_int),
        "spiffe_gpu_clear_screens": ([H], C.c_int),
        "spiffe_gpu_add_cathode": ([H, P(abi.CathodeOptions)], C.c_int),
        "spiffe_gpu_add_antenna": ([H, C.c_int32, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                    C.c_double, P(C.c_double), P(C.c_double), C.c_int64], C.c_int),
        "spiffe_gpu_configure_run": ([H, C.c_int32, P(abi.PushOptions), P(abi.PoissonOptions)], C.c_int),
        "spiffe_gpu_run_begin": ([H, P(abi.PoissonReport)], C.c_int),
        "spiffe_gpu_run_steps": ([H, C.c_int64], C.c_int),
        "spiffe_gpu_synchronize": ([H], C.c_int),
        "spiffe_gpu_counts": ([H, P(C.c_int64), P(C.c_int64)], C.c_int),
        "spiffe_gpu_counts_async": ([H, C.c_void_p], C.c_int),
        "spiffe_gpu_select_device": ([C.c_int32], C.c_int),
        "spiffe_gpu_stream": ([H, P(C.c_void_p)], C.c_int),
        "spiffe_gpu_set_profiling": ([H, C.c_int32], C.c_int),
        "spiffe_gpu_phase_times": ([H, P(C.c_double), P(C.c_int64)], C.c_int),
        "spiffe_gpu_launch_count": ([], C.c_int64),
        "spiffe_gpu_work_counters": ([H, P(C.c_int64)], C.c_int),
        "spiffe_gpu_set_sort_interval": ([H, C.c_int64], C.c_int),
        "spiffe_gpu_set_poisson_solver": ([H, C.c_int32], C.c_int),
        "spiffe_gpu_poisson_log": ([H, C.c_int64, P(C.c_double), P(C.c_int64)], C.c_int),
        "spiffe_gpu_screen_moments": ([H, C.c_int32, P(C.c_double)], C.c_int),
        "spiffe_gpu_batch_run": ([P(H), C.c_int32, P(C.c_int64), C.c_int32, C.c_int64, P(C.c_double)], C.c_int),
        "spiffe_gpu_set_test_beam": ([H, P(abi.TestBeamOptions)], C.c_int),
        "spiffe_gpu_add_on_axis_field": ([H, P(C.c_double), P(C.c_double), C.c_int64, C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_int32], C.c_int),
        "spiffe_gpu_on_axis_fields_at": ([H, C.c_double, C.c_double, C.c_double, C.c_int32, P(C.c_double)], C.c_int),
        "spiffe_gpu_set_translation": ([H, C.c_int32, C.c_double], C.c_int),
        "spiffe_gpu_translate_problem": ([H, P(C.c_int32), P(C.c_double)], C.c_int),
        "spiffe_session_create": ([C.c_int32, C.c_char_p, P(H)], C.c_int),
        "spiffe_session_destroy": ([H], C.c_int),
        "spiffe_session_execute": ([H, C.c_char_p], C.c_int),
        "spiffe_session_run_file": ([H, C.c_char_p], C.c_int),
        "spiffe_session_set": ([H, C.c_char_p, C.c_double], C.c_int),
        "spiffe_session_mesh": ([H, M], C.c_int),
        "spiffe_session_fields": ([H, F], C.c_int),
        "spiffe_session_instance": ([H, P(H)], C.c_int),
        "spiffe_session_steps": ([H], C.c_int64),
        "spiffe_solenoid_add": ([M, P(abi.SolenoidOptions), P(C.c_double), P(C.c_double), P(C.c_double)], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def select_device(device):
    """Device used by instances created afterwards on this thread."""
    _check(load().spiffe_gpu_select_device(int(device)))


def launch_count():
    return load().spiffe_gpu_launch_count()


def batch_run(instances, steps, workers=8, chunk=20):
    """Advances the instances concurrently (spiffe_gpu_batch_run): instance i
    by steps[i] integration steps, on `workers` host threads, `chunk` steps
    at a time.  Returns the milliseconds from the call to each instance's
    completion."""
    n = len(instances)
    hs = (H * max(n, 1))(*[g.h for g in instances])
    st = (C.c_int64 * max(n, 1))(*[int(k) for k in steps])
    done = (C.c_double * max(n, 1))()
    _check(load().spiffe_gpu_batch_run(hs, n, st, int(workers), int(chunk), done))
    return [done[i] for i in range(n)]


def _check(rc):
    if rc != 0:
        raise SpiffeGpuError(f"spiffe_b200 error {rc}: {load().spiffe_gpu_last_error().decode()}")


class GpuInstance:
    """One spiffe problem resident on the GPU."""

    def __init__(self, fields, capacity=1 << 16, precision=PRECISION_F64):
        lib = load()
        self.lib = lib
        self.precision = precision
        self.shape = fields.shape
        self.mesh = abi.Mesh.from_buffer_copy(fields.mesh)
        h = H()
        flags = np.ascontiguousarray(fields.flags, np.int16)
        _check(lib.spiffe_gpu_create(C.byref(self.mesh), flags.ctypes.data_as(P(C.c_int16)), precision,
                                     int(capacity), C.byref(h)))
        self.h = h
        self.upload_fields(fields)

    @classmethod
    def attach(cls, handle, precision):
        """A view of an instance another owner (a session) created and destroys."""
        g = cls.__new__(cls)
        g.lib = load()
        g.precision = precision
        g.h = handle
        g.borrowed = True
        g.mesh = g.get_mesh()
        g.shape = (g.mesh.nz + 1, g.mesh.nr + 1)
        return g

    def close(self):
        if getattr(self, "h", None) and not getattr(self, "borrowed", False):
            self.lib.spiffe_gpu_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_mesh(self, mesh=None):
        if mesh is not None:
            self.mesh = abi.Mesh.from_buffer_copy(mesh)
        _check(self.lib.spiffe_gpu_set_mesh(self.h, C.byref(self.mesh)))

    def get_mesh(self):
        m = abi.Mesh()
        _check(self.lib.spiffe_gpu_get_mesh(self.h, C.byref(m)))
        return m

    def upload_fields(self, fields):
        _check(self.lib.spiffe_gpu_upload_fields(self.h, C.byref(fields.c())))

    def download_fields(self, fields):
        _check(self.lib.spiffe_gpu_download_fields(self.h, C.byref(fields.c())))
        return fields

    def fields(self, like):
        out = like.copy()
        return self.download_fields(out)

    def upload_beam(self, beam):
        _check(self.lib.spiffe_gpu_upload_beam(self.h, C.byref(beam.c())))

    def download_beam(self, beam):
        bs = beam.c()
        _check(self.lib.spiffe_gpu_download_beam(self.h, C.byref(bs)))
        beam.take(bs)
        return beam

    def set_deposit_order(self, ordered):
        _check(self.lib.spiffe_gpu_set_deposit_order(self.h, int(ordered)))

    def set_sort_interval(self, n):
        _check(self.lib.spiffe_gpu_set_sort_interval(self.h, C.c_int64(int(n))))

    def zero_currents(self):
        _check(self.lib.spiffe_gpu_zero_current_arrays(self.h))

    def advance_fields(self):
        _check(self.lib.spiffe_gpu_advance_field_solutions(self.h))

    def deposit(self):
        _check(self.lib.spiffe_gpu_add_particle_currents(self.h))

    def advance_particles(self, opts=None):
        opts = opts or abi.push_options()
        _check(self.lib.spiffe_gpu_advance_particles(self.h, C.byref(opts)))

    def solve_poisson(self, target, accuracy, limit):
        n = C.c_int64()
        _check(self.lib.spiffe_gpu_solve_poisson_cyl(self.h, target, accuracy, limit, C.byref(n)))
        return n.value

    def poisson_correction(self, space_charge, opts):
        rep = abi.PoissonReport()
        _check(self.lib.spiffe_gpu_add_poisson_correction(self.h, space_charge, C.byref(opts), C.byref(rep)))
        return rep

    def imposed_efield(self, opts, initialize):
        _check(self.lib.spiffe_gpu_compute_imposed_efield(self.h, C.byref(opts), int(initialize)))

    def add_screen(self, z_position, direction=1, capacity=1 << 16):
        _check(self.lib.spiffe_gpu_add_screen(self.h, z_position, direction, int(capacity)))

    def screen(self, index, capacity=None):
        n = C.c_int64()
        _check(self.lib.spiffe_gpu_screen_count(self.h, index, C.byref(n)))
        sc = abi.Screen(0.0, 1, capacity=max(1, n.value if capacity is None else capacity))
        ss = sc.c()
        _check(self.lib.spiffe_gpu_download_screen(self.h, index, C.byref(ss)))
        sc.nb, sc.z_position, sc.direction = ss.nb, ss.z_position, ss.direction
        return sc

    def clear_screens(self):
        _check(self.lib.spiffe_gpu_clear_screens(self.h))

    def add_cathode(self, opts):
        _check(self.lib.spiffe_gpu_add_cathode(self.h, C.byref(opts)))

    def set_test_beam(self, opts):
        """define_test_beam's emission (abi.TestBeamOptions, or None to remove it)."""
        _check(self.lib.spiffe_gpu_set_test_beam(self.h, C.byref(opts) if opts is not None else None))

    def add_antenna(self, direction, istart, iend, iposition, current, frequency, phase, t, W):
        t = np.ascontiguousarray(t, np.float64)
        W = np.ascontiguousarray(W, np.float64)
        _check(self.lib.spiffe_gpu_add_antenna(self.h, direction, istart, iend, iposition, current, frequency, phase,
                                               t.ctypes.data_as(P(C.c_double)), W.ctypes.data_as(P(C.c_double)),
                                               len(t)))

    def add_on_axis_field(self, z, Ez, Ez_peak, frequency, phase_rad, z_offset=0.0, expansion_order=3):
        """add_on_axis_fields on an Ez(z) table (phase in radians)."""
        z = np.ascontiguousarray(z, np.float64)
        Ez = np.ascontiguousarray(Ez, np.float64)
        _check(self.lib.spiffe_gpu_add_on_axis_field(self.h, z.ctypes.data_as(P(C.c_double)),
                                                     Ez.ctypes.data_as(P(C.c_double)), len(z), z_offset, Ez_peak,
                                                     frequency, phase_rad, expansion_order))

    def on_axis_fields_at(self, z, r, t, profile=False):
        """(Ez, Er, Bphi) of the on-axis fields at (z, r) and time t."""
        out = (C.c_double * 3)()
        _check(self.lib.spiffe_gpu_on_axis_fields_at(self.h, z, r, t, int(profile), out))
        return tuple(out)

    def set_translation(self, enable, z_trigger):
        """translate's moving window (z_trigger in [zmin+dz, zmax-dz])."""
        _check(self.lib.spiffe_gpu_set_translation(self.h, int(enable), z_trigger))

    def translate_problem(self):
        """translate_problem: (moved this call, total translation)."""
        moved, total = C.c_int32(), C.c_double()
        _check(self.lib.spiffe_gpu_translate_problem(self.h, C.byref(moved), C.byref(total)))
        return bool(moved.value), total.value

    def configure_run(self, space_charge=1, push=None, poisson=None):
        self._push = push or abi.push_options()
        self._pc = poisson
        _check(self.lib.spiffe_gpu_configure_run(self.h, space_charge, C.byref(self._push),
                                                 C.byref(poisson) if poisson is not None else None))

    def run_begin(self):
        rep = abi.PoissonReport()
        _check(self.lib.spiffe_gpu_run_begin(self.h, C.byref(rep)))
        return rep

    def run_steps(self, n):
        _check(self.lib.spiffe_gpu_run_steps(self.h, int(n)))

    def synchronize(self):
        _check(self.lib.spiffe_gpu_synchronize(self.h))

    PHASES = ("emission", "deposit", "poisson", "fdtd", "push")

    def stream_handle(self):
        p = C.c_void_p()
        _check(self.lib.spiffe_gpu_stream(self.h, C.byref(p)))
        return p.value or 0

    def set_profiling(self, on):
        _check(self.lib.spiffe_gpu_set_profiling(self.h, int(on)))

    def phase_times(self):
        ms = (C.c_double * 5)()
        cnt = (C.c_int64 * 5)()
        _check(self.lib.spiffe_gpu_phase_times(self.h, ms, cnt))
        return {n: (ms[i], cnt[i]) for i, n in enumerate(self.PHASES)}

    def work_counters(self):
        """particle-steps, SOR half-sweeps, Poisson solves, FDTD steps and
        multigrid V-cycles so far."""
        out = (C.c_int64 * 5)()
        _check(self.lib.spiffe_gpu_work_counters(self.h, out))
        return dict(particle_steps=out[0], sor_halfsweeps=out[1], sor_solves=out[2], fdtd_steps=out[3],
                    mg_cycles=out[4])

    def screen_moments(self, screen=0):
        """Exit-plane moments of a screen's records, reduced on the device
        (the keys of spiffe_b200.moments.exit_moments)."""
        out = (C.c_double * 6)()
        _check(self.lib.spiffe_gpu_screen_moments(self.h, int(screen), out))
        return {"count": int(out[0]), "charge": out[1], "mean_ke_ev": out[2], "rms_energy_ev": out[3],
                "bunch_length_m": out[4], "emittance_m": out[5]}

    def poisson_log(self, max_rows=1 << 16):
        """The Poisson corrections run so far: an (n, 4) array of time step,
        iterations, final sum|residual| and sum|rhs|."""
        rows = np.zeros((max_rows, 4))
        n = C.c_int64()
        _check(self.lib.spiffe_gpu_poisson_log(self.h, max_rows, rows.ctypes.data_as(P(C.c_double)), C.byref(n)))
        return rows[: min(n.value, max_rows)].copy()

    def set_fdtd_kernel(self, kernel):
        """FDTD_AUTO, FDTD_TWO_KERNELS or FDTD_FUSED (split form)."""
        _check(self.lib.spiffe_gpu_set_fdtd_kernel(self.h, int(kernel)))

    def set_poisson_solver(self, solver):
        """POISSON_MULTIGRID (split form default) or POISSON_SOR."""
        _check(self.lib.spiffe_gpu_set_poisson_solver(self.h, int(solver)))

    def counts_async(self, out):
        """Enqueues a copy of (np, npActive) into out[0:2] (an int64 numpy
        array, best page-locked) without waiting; valid after synchronize()."""
        assert out.dtype == np.int64 and out.size >= 2 and out.flags["C_CONTIGUOUS"]
        _check(self.lib.spiffe_gpu_counts_async(self.h, out.ctypes.data))

    def counts(self):
        a, b = C.c_int64(), C.c_int64()
        _check(self.lib.spiffe_gpu_counts(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value
