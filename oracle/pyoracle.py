"""TEST INFRASTRUCTURE: Python bindings for the two CPU checkers.

* ``Oracle`` wraps build/liboracle.so, the project's C restatement of the
  reference's per-step path (spiffe_oracle.c), over the numpy containers of
  spiffe_b200.abi.
* ``run_reference(program)`` executes a list of operations against the
  reference spiffe itself, compiled in place into _ref/libspiffe_ref.so, in a
  fresh ``spawn`` process (the reference keeps state in function statics, so
  every case needs its own process).

Only tests, the smoke check and the benchmark's CPU-baseline leg use this
module, and only as a checker.
"""
from __future__ import annotations

import ctypes as C
import os
import pickle
import subprocess
import sys

import numpy as np

from spiffe_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libspiffe_ref.so")
DROPIN_SO = os.path.join(HERE, "_ref", "libspiffe_dropin.so")

P = C.POINTER


def _load_oracle():
    lib = C.CDLL(ORACLE_SO)
    M, F, B, S = P(abi.Mesh), P(abi.FieldSet), P(abi.BeamSet), P(abi.ScreenSet)
    lib.orc_zero_currents.argtypes = [M, F]
    lib.orc_advance_fields.argtypes = [M, F]
    lib.orc_deposit.argtypes = [M, F, B]
    lib.orc_gather.argtypes = [M, F, C.c_double, C.c_double, P(C.c_double)]
    lib.orc_advance_particles.argtypes = [M, F, B, S, C.c_int, P(abi.PushOptions)]
    lib.orc_advance_particles.restype = C.c_long
    lib.orc_solve_poisson.argtypes = [M, P(C.c_int16), P(C.c_double), P(C.c_double), C.c_double, C.c_long,
                                      P(C.c_double), P(C.c_double)]
    lib.orc_solve_poisson.restype = C.c_long
    lib.orc_poisson_correction.argtypes = [M, F, B, C.c_int, P(abi.PoissonOptions), P(C.c_int64),
                                           P(abi.PoissonReport)]
    lib.orc_poisson_correction.restype = C.c_int
    lib.orc_imposed_efield.argtypes = [M, F, P(abi.PoissonOptions), C.c_int, P(C.c_double), P(C.c_int64)]
    lib.orc_kinetic_energy.argtypes = [B]
    lib.orc_kinetic_energy.restype = C.c_double
    lib.orc_field_energy.argtypes = [M, F, P(C.c_double)]
    lib.orc_run_new.restype = C.c_void_p
    lib.orc_run_free.argtypes = [C.c_void_p]
    lib.orc_run_emitter.argtypes = [C.c_void_p]
    lib.orc_run_emitter.restype = C.c_void_p
    lib.orc_cathode_define.argtypes = [C.c_void_p, M, P(abi.CathodeOptions)]
    lib.orc_cathode_define.restype = C.c_int
    lib.orc_emit.argtypes = [C.c_void_p, M, F, B]
    lib.orc_emit.restype = C.c_long
    lib.orc_set_current_density.argtypes = [C.c_void_p, M, F]
    lib.orc_run_configure.argtypes = [C.c_void_p, C.c_int32, P(abi.PushOptions), P(abi.PoissonOptions)]
    lib.orc_run_antenna.argtypes = [C.c_void_p, C.c_int32, C.c_long, C.c_long, C.c_long, C.c_double, C.c_double,
                                    C.c_double, P(C.c_double), P(C.c_double), C.c_long]
    lib.orc_run_begin.argtypes = [C.c_void_p, M, F, B, P(abi.PoissonReport)]
    lib.orc_run_step.argtypes = [C.c_void_p, M, F, B, S, C.c_int, P(abi.PoissonReport)]
    lib.orc_run_step.restype = C.c_long
    return lib


class Oracle:
    """The C restatement, operating in place on abi.Fields / abi.Beam."""

    def __init__(self):
        self.lib = _load_oracle()

    def zero_currents(self, f):
        self.lib.orc_zero_currents(C.byref(f.mesh), C.byref(f.c()))

    def advance_fields(self, f):
        self.lib.orc_advance_fields(C.byref(f.mesh), C.byref(f.c()))

    def deposit(self, f, b):
        self.lib.orc_deposit(C.byref(f.mesh), C.byref(f.c()), C.byref(b.c()))

    def gather(self, f, z, r):
        out = (C.c_double * 6)()
        self.lib.orc_gather(C.byref(f.mesh), C.byref(f.c()), z, r, out)
        return np.array(out[:])

    def advance_particles(self, f, b, screens=(), opts=None):
        opts = opts or abi.push_options()
        bs = b.c()
        sc = abi.screens_c(screens)
        lost = self.lib.orc_advance_particles(C.byref(f.mesh), C.byref(f.c()), C.byref(bs), sc, len(screens),
                                              C.byref(opts))
        b.take(bs)
        abi.screens_take(screens, sc)
        return lost

    def solve_poisson(self, f, psi, rhs, accuracy, limit):
        res, drv = C.c_double(), C.c_double()
        n = self.lib.orc_solve_poisson(C.byref(f.mesh), f.flags.ctypes.data_as(P(C.c_int16)),
                                       psi.ctypes.data_as(P(C.c_double)),
                                       rhs.ctypes.data_as(P(C.c_double)) if rhs is not None else None,
                                       accuracy, limit, C.byref(res), C.byref(drv))
        return n, res.value, drv.value

    def poisson_correction(self, f, b, space_charge, opts, start_step=None):
        st = C.c_int64(-1 if start_step is None else start_step)
        rep = abi.PoissonReport()
        self.lib.orc_poisson_correction(C.byref(f.mesh), C.byref(f.c()), C.byref(b.c()), space_charge,
                                        C.byref(opts), C.byref(st), C.byref(rep))
        return rep

    def kinetic_energy(self, b):
        return self.lib.orc_kinetic_energy(C.byref(b.c()))

    def field_energy(self, f):
        out = (C.c_double * 2)()
        self.lib.orc_field_energy(C.byref(f.mesh), C.byref(f.c()), out)
        return out[0], out[1]


class OracleRun:
    """The oracle's perform_integration loop (integrate.c:134-194)."""

    def __init__(self, oracle, fields, beam, space_charge=1, push=None, poisson=None, screens=()):
        self.o, self.f, self.b = oracle, fields, beam
        self.lib = oracle.lib
        self.h = self.lib.orc_run_new()
        self.push = push or abi.push_options()
        self.poisson = poisson or abi.PoissonOptions()
        self.lib.orc_run_configure(self.h, space_charge, C.byref(self.push), C.byref(self.poisson))
        self.screens = list(screens)
        self._keep = []

    def add_cathode(self, opts):
        self._keep.append(opts)
        n = self.lib.orc_cathode_define(self.lib.orc_run_emitter(self.h), C.byref(self.f.mesh), C.byref(opts))
        if n < 0:
            raise ValueError("cathode rejected")
        return n

    def add_antenna(self, direction, istart, iend, iposition, current, frequency, phase, t, W):
        t = np.ascontiguousarray(t, np.float64)
        W = np.ascontiguousarray(W, np.float64)
        self._keep += [t, W]
        self.lib.orc_run_antenna(self.h, direction, istart, iend, iposition, current, frequency, phase,
                                 t.ctypes.data_as(P(C.c_double)), W.ctypes.data_as(P(C.c_double)), len(t))

    def begin(self):
        rep = abi.PoissonReport()
        bs = self.b.c()
        self.lib.orc_run_begin(self.h, C.byref(self.f.mesh), C.byref(self.f.c()), C.byref(bs), C.byref(rep))
        return rep

    def step(self):
        rep = abi.PoissonReport()
        bs = self.b.c()
        sc = abi.screens_c(self.screens)
        lost = self.lib.orc_run_step(self.h, C.byref(self.f.mesh), C.byref(self.f.c()), C.byref(bs), sc,
                                     len(self.screens), C.byref(rep))
        if lost < 0:
            raise RuntimeError("oracle: particle capacity exceeded")
        self.b.take(bs)
        abi.screens_take(self.screens, sc)
        return rep

    def __del__(self):
        try:
            self.lib.orc_run_free(self.h)
        except Exception:
            pass


# ------------------------------------------------------------- the reference

def _ref_lib():
    lib = C.CDLL(REF_SO)
    lib.ref_session_init.argtypes = [C.c_long]
    lib.ref_command.argtypes = [C.c_char_p]
    lib.ref_get_mesh.argtypes = [P(C.c_int32), P(C.c_int32), P(C.c_double), P(C.c_int32), P(C.c_uint32)]
    lib.ref_set_time.argtypes = [C.c_double, C.c_double, C.c_int64, C.c_uint32]
    lib.ref_set_constant_fields.argtypes = [P(C.c_double), P(C.c_int16)]
    lib.ref_get_field.argtypes = [C.c_char_p, P(C.c_double)]
    lib.ref_set_field.argtypes = [C.c_char_p, P(C.c_double)]
    lib.ref_get_flags.argtypes = [P(C.c_int16)]
    lib.ref_set_flags.argtypes = [P(C.c_int16)]
    lib.ref_get_beam_counts.argtypes = [P(C.c_int64), P(C.c_double)]
    lib.ref_set_beam_counts.argtypes = [P(C.c_int64), P(C.c_double)]
    lib.ref_get_beam.argtypes = [C.c_char_p, C.c_void_p]
    lib.ref_set_beam.argtypes = [C.c_char_p, C.c_void_p, C.c_int64]
    lib.ref_add_poisson_correction.argtypes = [C.c_long]
    lib.ref_compute_imposed_Efield.argtypes = [C.c_long]
    lib.ref_add_antenna_excitation.argtypes = [C.c_double]
    lib.ref_advance_particles.argtypes = [C.c_double]
    lib.ref_solve_poisson_cyl.argtypes = [P(C.c_double), P(C.c_double), C.c_int, C.c_double, C.c_long]
    lib.ref_solve_poisson_cyl.restype = C.c_long
    lib.ref_step.argtypes = [C.c_long, C.c_double]
    lib.ref_screen_count.argtypes = [C.c_long]
    lib.ref_screen_count.restype = C.c_int64
    lib.ref_screen_column.argtypes = [C.c_long, C.c_char_p, P(C.c_double)]
    lib.ref_screen_column.restype = C.c_int64
    lib.ref_table_column.argtypes = [C.c_long, C.c_char_p, P(C.c_double)]
    lib.ref_table_column.restype = C.c_int64
    lib.ref_table_pages.argtypes = [C.c_long]
    lib.ref_table_pages.restype = C.c_int64
    lib.ref_kinetic_energy.restype = C.c_double
    lib.ref_field_energy.argtypes = [P(C.c_double)]
    lib.ref_time_step.restype = C.c_int64
    lib.ref_rng_counter.restype = C.c_uint64
    lib.ref_boundary_points.argtypes = [C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long]
    lib.ref_boundary_points.restype = C.c_long
    return lib


def _mesh(lib):
    nz, nr, mo = C.c_int32(), C.c_int32(), C.c_uint32()
    g = (C.c_double * 8)()
    bc = (C.c_int32 * 4)()
    lib.ref_get_mesh(C.byref(nz), C.byref(nr), g, bc, C.byref(mo))
    return dict(nz=nz.value, nr=nr.value, zmin=g[0], zmax=g[1], rmax=g[2], dz=g[3], dr=g[4], dt=g[5], time=g[6],
                start_time=g[7], lower_bc=bc[0], upper_bc=bc[1], right_bc=bc[2], left_bc=bc[3], modes=mo.value)


_BEAM_INT = {"particleID": np.int32, "generation": np.int16, "status": np.uint64}


def _child(program, capacity, cwd, preload=()):
    """Runs in a spawned process: executes `program` against the reference.
    Libraries in `preload` are loaded first into the global symbol scope, so
    their definitions take the place of the reference's own (a link-time
    drop-in)."""
    if cwd:
        os.chdir(cwd)
    for path in preload:
        C.CDLL(path, mode=C.RTLD_GLOBAL)
    lib = _ref_lib()
    lib.ref_session_init(capacity)
    out = []
    shape = None
    for op in program:
        kind, args = op[0], op[1:]
        if kind == "command":
            rc = lib.ref_command(args[0].encode())
            if rc != 0:
                raise RuntimeError(f"reference rejected command ({rc}): {args[0][:60]}")
            m = _mesh(lib)
            shape = (m["nz"] + 1, m["nr"] + 1)
        elif kind == "mesh":
            m = _mesh(lib)
            shape = (m["nz"] + 1, m["nr"] + 1)
            out.append(m)
        elif kind == "set_time":
            lib.ref_set_time(*args)
        elif kind == "set_constant_fields":
            c = (C.c_double * 6)(*args[0])
            t = (C.c_int16 * 6)(*args[1])
            lib.ref_set_constant_fields(c, t)
        elif kind == "set_field":
            a = np.ascontiguousarray(args[1], np.float64)
            assert a.shape == shape, (args[0], a.shape, shape)
            lib.ref_set_field(args[0].encode(), a.ctypes.data_as(P(C.c_double)))
        elif kind == "get_field":
            a = np.zeros(shape)
            if lib.ref_get_field(args[0].encode(), a.ctypes.data_as(P(C.c_double))) != 0:
                a = None
            out.append(a)
        elif kind == "set_flags":
            a = np.ascontiguousarray(args[0], np.int16)
            lib.ref_set_flags(a.ctypes.data_as(P(C.c_int16)))
        elif kind == "get_flags":
            a = np.zeros(shape, np.int16)
            lib.ref_get_flags(a.ctypes.data_as(P(C.c_int16)))
            out.append(a)
        elif kind == "set_beam":
            counts = (C.c_int64 * 4)(*args[0])
            sc = (C.c_double * 2)(*args[1])
            for name, arr in args[2].items():
                a = np.ascontiguousarray(arr, _BEAM_INT.get(name, np.float64))
                lib.ref_set_beam(name.encode(), a.ctypes.data, len(a))
            lib.ref_set_beam_counts(counts, sc)
        elif kind == "get_beam":
            counts = (C.c_int64 * 4)()
            sc = (C.c_double * 2)()
            lib.ref_get_beam_counts(counts, sc)
            n = counts[0]
            d = {"np": n, "npActive": counts[1], "max_np": counts[2], "nextParticleID": counts[3],
                 "QoMC": sc[0], "stiffness": sc[1]}
            for name in abi.BEAM_DOUBLES + list(_BEAM_INT):
                a = np.zeros(n, _BEAM_INT.get(name, np.float64))
                lib.ref_get_beam(name.encode(), a.ctypes.data)
                d[name] = a
            out.append(d)
        elif kind == "call":
            fn = getattr(lib, args[0])
            r = fn(*args[1:])
            out.append(r)
        elif kind == "solve_poisson":
            psi = np.ascontiguousarray(args[0], np.float64).copy()
            rhs = None if args[1] is None else np.ascontiguousarray(args[1], np.float64)
            n = lib.ref_solve_poisson_cyl(psi.ctypes.data_as(P(C.c_double)),
                                          rhs.ctypes.data_as(P(C.c_double)) if rhs is not None else None,
                                          1 if rhs is not None else 0, args[2], args[3])
            out.append((n, psi))
        elif kind == "screen":
            n = lib.ref_screen_count(args[0])
            d = {}
            for col in abi.SCREEN_COLUMNS + ["rMin", "rMax", "zMin", "zMax", "generation", "particleID"]:
                a = np.zeros(max(n, 0))
                lib.ref_screen_column(args[0], col.encode(), a.ctypes.data_as(P(C.c_double)))
                d[col] = a
            out.append(d)
        elif kind == "table":
            # ("table", which, [columns]): which 0 beam snapshots, 1 field output,
            # 2 + k the k-th table closed inside a command, 100 + k the k-th
            # table written row by row (the status file)
            which, cols = args
            d = {"pages": lib.ref_table_pages(which)}
            for col in cols:
                n = lib.ref_table_column(which, col.encode(), None)
                a = np.zeros(max(n, 0))
                if n > 0:
                    lib.ref_table_column(which, col.encode(), a.ctypes.data_as(P(C.c_double)))
                d[col] = a if n >= 0 else None
            out.append(d)
        elif kind == "kinetic_energy":
            out.append(lib.ref_kinetic_energy())
        elif kind == "field_energy":
            e = (C.c_double * 2)()
            lib.ref_field_energy(e)
            out.append((e[0], e[1]))
        elif kind == "boundary_points":
            mx = 1 << 16
            iz, ir, d = np.zeros(mx, np.int32), np.zeros(mx, np.int32), np.zeros(mx, np.int16)
            n = lib.ref_boundary_points(args[0], iz.ctypes.data, ir.ctypes.data, d.ctypes.data, mx)
            out.append((iz[:n].copy(), ir[:n].copy(), d[:n].copy()))
        elif kind == "rng_counter":
            out.append(lib.ref_rng_counter())
        elif kind == "time_steps":
            # (seconds, active particles) of each perform_integration loop step
            import time

            n, space_charge, zfs = args
            res = []
            for _ in range(n):
                counts = (C.c_int64 * 4)()
                sc = (C.c_double * 2)()
                lib.ref_get_beam_counts(counts, sc)
                t0 = time.perf_counter()
                lib.ref_step(space_charge, zfs)
                res.append((time.perf_counter() - t0, counts[1]))
            out.append(res)
        else:
            raise ValueError(kind)
    return out


def run_reference(program, capacity=1 << 16, cwd=None, timeout=900, threads=1, preload=()):
    """Runs `program` (a list of tuples) against the compiled reference in a
    fresh Python process (pickles over stdin/stdout) and returns the list of
    requested outputs.  `threads` sets OMP_NUM_THREADS: the reference's push
    loop shares pz0/pr0/r_pphi0 between OpenMP threads
    (advance_particles.c:79, :131, :202-204), so only a one-thread run is
    deterministic."""
    if not os.path.exists(REF_SO):
        raise FileNotFoundError(REF_SO)
    repo = os.path.dirname(HERE)
    env = dict(os.environ)
    env["PYTHONPATH"] = repo + os.pathsep + env.get("PYTHONPATH", "")
    env["OMP_NUM_THREADS"] = str(threads)
    proc = subprocess.run([sys.executable, "-m", "oracle.pyoracle"],
                          input=pickle.dumps((program, capacity, cwd, tuple(preload))),
                          capture_output=True, timeout=timeout, env=env, cwd=repo)
    if proc.returncode != 0:
        raise RuntimeError("reference run failed (%d): %s" % (proc.returncode, proc.stderr.decode()[-2000:]))
    return pickle.loads(proc.stdout)


def reference_available():
    return os.path.exists(REF_SO)


if __name__ == "__main__":
    _program, _capacity, _cwd, _preload = pickle.loads(sys.stdin.buffer.read())
    # the reference prints progress on stdout; keep the pickle channel clean
    _real = os.dup(1)
    os.dup2(2, 1)
    _out = _child(_program, _capacity, _cwd, _preload)
    sys.stdout.flush()
    os.dup2(_real, 1)
    with os.fdopen(_real, "wb") as _f:
        _f.write(pickle.dumps(_out))
