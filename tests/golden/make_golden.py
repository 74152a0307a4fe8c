"""Generates the golden fixtures in this directory from the reference itself.

Each fixture is produced by the reference spiffe's own code, compiled in
place from its sources by oracle/Makefile into oracle/_ref/libspiffe_ref.so
(one thread, so the OpenMP push loop is deterministic), on the project's
synthetic inputs (spiffe_b200.workloads).  Inputs and outputs are stored
together so the oracle and the CUDA path can be checked without the
reference present.  Run from the repository root:

    python tests/golden/make_golden.py          # every fixture
    python tests/golden/make_golden.py decks    # the input-deck fixtures only
    python tests/golden/make_golden.py onaxis   # one deck fixture (also: translate)
    python tests/golden/make_golden.py te       # the TE-field fixture
    python tests/golden/make_golden.py lost     # the lost-particle deck
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle  # noqa: E402
from spiffe_b200 import abi, workloads  # noqa: E402

MODES = abi.FL_TM_FIELDS | abi.FL_RADIAL_INTERP | abi.FL_LONGIT_INTERP
QoMC = -1.602176634e-19 / (9.1093837015e-31 * 2.99792458e8)


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print("wrote", name, sum(np.asarray(v).nbytes for v in arrays.values()), "bytes raw")


def geometry(cmd, geo_name, geo_text):
    d = tempfile.mkdtemp()
    with open(os.path.join(d, geo_name), "w") as f:
        f.write(geo_text)
    mesh, flags, psi = pyoracle.run_reference([("command", cmd), ("mesh",), ("get_flags",), ("get_field", "PsiImposed")],
                                              cwd=d)
    return d, mesh, flags, psi


def mesh_arrays(mesh):
    return dict(nz=mesh["nz"], nr=mesh["nr"], zmin=mesh["zmin"], zmax=mesh["zmax"], rmax=mesh["rmax"],
                dz=mesh["dz"], dr=mesh["dr"], bcs=np.array([mesh["lower_bc"], mesh["upper_bc"], mesh["right_bc"],
                                                             mesh["left_bc"]]))


def random_beam(rng, n, zlo, zhi, rhi, active_frac=0.9):
    z = rng.uniform(zlo, zhi, n)
    r = rng.uniform(-0.05 * rhi, 1.02 * rhi, n)
    pz = rng.normal(size=n)
    pr = rng.normal(size=n) * 0.1
    rpp = rng.normal(size=n) * 1e-5
    rs = np.where(r != 0, r, 1.0)
    g = np.sqrt(1 + pz ** 2 + pr ** 2 + (rpp / rs) ** 2)
    c = 2.99792458e8
    status = np.where(rng.uniform(size=n) < active_frac, 1, 0).astype(np.uint64)
    return dict(z=z, r=r, pz=pz, pr=pr, r_pphi=rpp, vz=c * pz / g, vr=c * pr / g, vphi=c * rpp / rs / g,
                Q=np.full(n, -1e-14), r0=r.copy(), z0=z.copy(), t0=np.zeros(n), rmin=r - 1e-4, rmax=r + 1e-4,
                zmin=z - 1e-4, zmax=z + 1e-4, particleID=np.arange(1, n + 1, dtype=np.int32),
                generation=np.zeros(n, np.int16), status=status)


def beam_out(rb):
    return {"out_" + k: rb[k] for k in abi.BEAM_DOUBLES + ["particleID", "status"]} | {
        "out_np": rb["np"], "out_npActive": rb["npActive"]}


def main():
    rng = np.random.default_rng(20261203)

    # --- config-1 pillbox: geometry, and the cavity ringing 400 steps
    cfg = workloads.PillboxConfig()
    d, mesh, flags, _ = geometry(cfg.geometry(), "pillbox.geo", cfg.geo_text())
    ez0 = cfg.initial_ez()
    steps = 400
    prog = [("command", cfg.geometry()), ("set_time", cfg.dt, 0.0, 0, MODES), ("set_field", "Ez", ez0)]
    prog += [("call", "ref_advance_field_solutions")] * steps
    prog += [("get_field", n) for n in ("Ez", "Er", "Bphi", "Bphi2")]
    out = pyoracle.run_reference(prog, cwd=d)[-4:]
    save("pillbox_fdtd", flags=flags, geo=np.array(cfg.geo_text()), dt=cfg.dt, steps=steps, Ez0=ez0,
         Ez=out[0], Er=out[1], Bphi=out[2], Bphi2=out[3], **mesh_arrays(mesh))

    # --- one push + deposition on disturbed fields with a solenoid and a screen
    shape = flags.shape
    fields = {n: rng.normal(size=shape) * (1e7 if n[0] == "E" else 0.05) for n in ("Ez", "Er", "Bphi", "Bphi2")}
    fields["EzImposed"] = rng.normal(size=shape) * 1e6
    fields["ErImposed"] = rng.normal(size=shape) * 1e6
    fields["BzImposed"] = rng.normal(size=shape) * 0.1
    fields["BrImposed"] = rng.normal(size=shape) * 0.1
    N = 1500
    beam = random_beam(rng, N, -0.0003, cfg.L + 0.0003, cfg.R)
    tstep = 37
    modes = MODES | abi.FL_SPACE_CHARGE
    zs = cfg.L / 2
    for comp, tag in ((0, "ref"), (1, "swap")):
        prog = [("command", cfg.geometry()), ("command", workloads.namelist("define_screen", filename="s", z_position=zs)),
                ("set_time", cfg.dt, 0.0, tstep, modes)]
        prog += [("set_field", n, a) for n, a in fields.items()]
        prog += [("set_beam", (N, int(beam["status"].sum()), 0, N + 1), (QoMC, 1.0), beam),
                 ("call", "ref_zero_current_arrays"), ("call", "ref_add_particle_currents"), ("get_field", "Jz"),
                 ("get_field", "Jr"), ("call", "ref_advance_particles", -1.0), ("get_beam",), ("screen", 0)]
        if tag == "swap":
            continue  # the reference has one compaction behaviour; "swap" is checked against the oracle
        res = pyoracle.run_reference(prog, cwd=d)
        Jz, Jr, rb, rs = res[-5], res[-4], res[-2], res[-1]
        save("pillbox_push", flags=flags, dt=cfg.dt, time_step=tstep, modes=modes, screen_z=zs, QoMC=QoMC,
             **{"f_" + k: v for k, v in fields.items()}, **{"in_" + k: v for k, v in beam.items()},
             Jz=Jz, Jr=Jr, **beam_out(rb), **{"screen_" + k: v for k, v in rs.items()}, **mesh_arrays(mesh))

    # --- DC gun (coarse): imposed Laplace solve and a Poisson correction
    geo = workloads.dc_gun_geo()
    cmd = workloads.geometry_command(151, 101, 0.0, 0.030, 0.020, "dc.geo")
    d2, mesh2, flags2, psi_imp0 = geometry(cmd, "dc.geo", geo)
    pc = workloads.namelist("poisson_correction", step_interval=1, accuracy=1e-6, maximum_iterations=1000)
    shape2 = flags2.shape
    Ez = rng.normal(size=shape2) * 1e5
    Er = rng.normal(size=shape2) * 1e5
    N2 = 1200
    beam2 = dict(z=rng.uniform(0, 0.03, N2), r=rng.uniform(0, 0.02, N2), Q=np.full(N2, -1e-13),
                 status=np.ones(N2, np.uint64))
    dt2 = 1e-13
    prog = [("command", cmd), ("command", pc), ("set_time", dt2, 0.0, 0, modes), ("call", "ref_compute_imposed_Efield", 1),
            ("get_field", "PsiImposed"), ("get_field", "EzImposed"), ("get_field", "ErImposed"),
            ("set_field", "Ez", Ez), ("set_field", "Er", Er), ("set_beam", (N2, N2, 0, 1), (0.0, 1.0), beam2),
            ("call", "ref_add_poisson_correction", 1), ("get_field", "Ez"), ("get_field", "Er"), ("get_field", "Psi"),
            ("get_field", "Q")]
    res = pyoracle.run_reference(prog, cwd=d2)
    save("dcgun_poisson", flags=flags2, dt=dt2, PsiImposed0=psi_imp0, PsiImposed=res[1], EzImposed=res[2],
         ErImposed=res[3], Ez0=Ez, Er0=Er, **{"in_" + k: v for k, v in beam2.items()}, Ez=res[-4], Er=res[-3],
         Psi=res[-2], Q=res[-1], **mesh_arrays(mesh2))

    # --- config-1 loop with emission through perform_integration, 220 steps
    t, A = cfg.profile()
    with open(os.path.join(d, "prof.sdds"), "w") as f:
        f.write("SDDS1\n&column name=t type=double &end\n&column name=A type=double &end\n"
                "&data mode=ascii no_row_counts=1 &end\n")
        for a, b in zip(t, A):
            f.write("%.17g %.17g\n" % (a, b))
    nsteps = 220
    cath = workloads.namelist("define_cathode", z_position=0.0, outer_radius=cfg.cathode_radius,
                              current_density=cfg.peak_current_density(), electrons_per_macroparticle=cfg.epm,
                              profile="prof.sdds", profile_time_name="t", profile_factor_name="A",
                              random_number_seed=cfg.seed)
    scr = workloads.namelist("define_screen", filename="exit", z_position=0.004)
    integ = workloads.namelist("integrate", dt_integration=cfg.dt, finish_time=(nsteps + 0.5) * cfg.dt, space_charge=1)
    res = pyoracle.run_reference([("command", cfg.geometry()), ("set_field", "Ez", ez0), ("command", cath),
                                  ("command", scr), ("command", integ), ("get_field", "Ez"), ("get_field", "Er"),
                                  ("get_field", "Bphi"), ("get_field", "Jz"), ("get_field", "Jr"), ("get_beam",),
                                  ("screen", 0), ("rng_counter",)], cwd=d, capacity=40000)
    Ezf, Erf, Bpf, Jzf, Jrf, rb, rs, rc = res
    save("pillbox_loop", flags=flags, dt=cfg.dt, steps=nsteps, Ez0=ez0, prof_t=t, prof_A=A, screen_z=0.004,
         Ez=Ezf, Er=Erf, Bphi=Bpf, Jz=Jzf, Jr=Jrf, rng_counter=rc, **beam_out(rb),
         **{"screen_" + k: v for k, v in rs.items()}, **mesh_arrays(mesh))

    # --- geometry rasterisation of the other two configurations' shapes
    _, mesh3, flags3, psi3 = geometry(workloads.geometry_command(301, 83, 0.0, 0.150, 0.041, "gun.geo"), "gun.geo",
                                      workloads.gun16_geo())
    save("gun16_geometry", flags=flags3, geo=np.array(workloads.gun16_geo()), **mesh_arrays(mesh3))
    save("dcgun_geometry", flags=flags2, PsiImposed=psi_imp0, geo=np.array(geo), **mesh_arrays(mesh2))


# TE fields (include_TE_fields=1, geometry.nl:25): the FDTD's TE part
# (integrate.c:434-540) on the gun mesh from random fields and currents, and
# one deposition and push whose gather reads Ephi, Br2 and Bz2
# (advance_particles.c:649-825) and whose deposit fills Jphi
# (space_charge.c:218).
TE_FIELDS = ("Ez", "Er", "Bphi", "Bphi2", "Ephi", "Br", "Bz", "Br2", "Bz2")


def f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def te():
    rng = np.random.default_rng(3)
    fx = np.load(os.path.join(HERE, "gun16_geometry.npz"))
    cmd = workloads.geometry_command(301, 83, 0.0, 0.150, 0.041, "gun.geo")
    d, mesh, flags, _ = geometry(cmd, "gun.geo", str(fx["geo"]))
    assert np.array_equal(flags, fx["flags"])
    modes = MODES | abi.FL_TE_FIELDS
    dt, steps = 2e-13, 25
    # inputs rounded to single precision (exact in double) keep the fixture small
    init = {n: f32(rng.normal(size=flags.shape)) for n in TE_FIELDS + ("Jz", "Jr", "Jphi")}
    prog = [("command", cmd), ("set_time", dt, 0.0, 0, modes)]
    prog += [("set_field", n, a) for n, a in init.items()]
    prog += [("call", "ref_advance_field_solutions")] * steps
    prog += [("get_field", n) for n in TE_FIELDS]
    out = pyoracle.run_reference(prog, cwd=d)[-len(TE_FIELDS):]
    arrays = dict(flags=flags, dt=dt, steps=steps, modes=modes,
                  **{"in_" + n: a.astype(np.float32) for n, a in init.items()},
                  **dict(zip(TE_FIELDS, out)), **mesh_arrays(mesh))

    # deposition and push on the pillbox mesh with TE fields present
    cfg = workloads.PillboxConfig()
    d2, mesh2, flags2, _ = geometry(cfg.geometry(), "pillbox.geo", cfg.geo_text())
    shape = flags2.shape
    scale = {"E": 1e7, "B": 0.05}
    fields = {n: f32(rng.normal(size=shape) * scale[n[0]]) for n in TE_FIELDS}
    fields["EzImposed"] = f32(rng.normal(size=shape) * 1e6)
    fields["ErImposed"] = f32(rng.normal(size=shape) * 1e6)
    fields["BzImposed"] = f32(rng.normal(size=shape) * 0.1)
    fields["BrImposed"] = f32(rng.normal(size=shape) * 0.1)
    N = 1500
    beam = random_beam(rng, N, -0.0003, cfg.L + 0.0003, cfg.R)
    beam["r_pphi"] = rng.normal(size=N) * 1e-4
    rs = np.where(beam["r"] != 0, beam["r"], 1.0)
    g = np.sqrt(1 + beam["pz"] ** 2 + beam["pr"] ** 2 + (beam["r_pphi"] / rs) ** 2)
    c = 2.99792458e8
    beam["vz"], beam["vr"], beam["vphi"] = c * beam["pz"] / g, c * beam["pr"] / g, c * beam["r_pphi"] / rs / g
    tstep = 11
    pmodes = modes | abi.FL_SPACE_CHARGE
    prog = [("command", cfg.geometry()), ("set_time", cfg.dt, 0.0, tstep, pmodes)]
    prog += [("set_field", n, a) for n, a in fields.items()]
    # the TE current array exists when define_geometry has include_TE_fields=1
    prog += [("set_field", "Jphi", np.zeros(shape))]
    prog += [("set_beam", (N, int(beam["status"].sum()), 0, N + 1), (QoMC, 1.0), beam),
             ("call", "ref_zero_current_arrays"), ("call", "ref_add_particle_currents"), ("get_field", "Jz"),
             ("get_field", "Jr"), ("get_field", "Jphi"), ("call", "ref_advance_particles", -1.0), ("get_beam",)]
    res = pyoracle.run_reference(prog, cwd=d2)
    Jz, Jr, Jphi, rb = res[-5], res[-4], res[-3], res[-1]
    arrays.update(p_flags=flags2, p_dt=cfg.dt, p_time_step=tstep, p_modes=pmodes, p_QoMC=QoMC,
                  p_Jz=Jz, p_Jr=Jr, p_Jphi=Jphi, **{"p_f_" + k: v.astype(np.float32) for k, v in fields.items()},
                  **{"p_in_" + k: v for k, v in beam.items()}, **{"p_" + k: v for k, v in beam_out(rb).items()},
                  **{"p_" + k: v for k, v in mesh_arrays(mesh2).items()})
    save("gun16_te", **arrays)


# Input decks run through the reference's own command processors and
# perform_integration (spiffe.c:213-308), for the command session.  The DC
# gun deck exercises the imposed-field ramp, a ring-coil solenoid, constant
# fields, a cathode with distribution correction, a screen and periodic
# Poisson correction; the test-beam deck exercises define_test_beam's
# emission and forced acceleration.  One screen each: the reference gives
# buffers to the first screen only (advance_particles.c:343-359 clears its
# allocation flag inside the screen loop), so a second screen that records a
# crossing writes through a null pointer.
DECK_DCGUN = """&define_geometry nz=151, nr=101, zmin=0.0, zmax=0.03, rmax=0.02, boundary="dc.geo" &end
&define_solenoid radius=0.025, z_start=0.012, z_end=0.02, turns=4, current=1000, Bz_peak=0.03 &end
&set_constant_fields Br=1e-4 &end
&define_cathode z_position=1e-6, outer_radius=0.002, current_density=2e6, start_time=0, stop_time=40e-12,
    number_per_step=10, initial_pz=1e-6, distribution_correction_interval=1 &end
&define_screen filename="deck.sc1", z_position=0.012, direction="forward" &end
&poisson_correction step_interval=4, accuracy=1e-4, error_charge_threshold=1e-15 &end
&integrate dt_integration=4e-13, start_time=0, finish_time=300e-12, space_charge=1, imposed_Efield_ramp_time=20e-12 &end
"""

DECK_TESTBEAM = """&define_geometry nz=151, nr=101, zmin=0.0, zmax=0.03, rmax=0.02, boundary="dc.geo" &end
&define_test_beam start_time=0, stop_time=30e-12, initial_z=0.0005, initial_r=0.0012, initial_pz=0.02,
    initial_pr=0.001, initial_rpphi=1e-7, electrons_per_macroparticle=2e5, z_force=5e9, r_force=1e8,
    z_start_deceleration=0.02, r_start_deceleration=0.003 &end
&define_screen filename="tb.sc1", z_position=0.012, direction="forward" &end
&poisson_correction step_interval=4, accuracy=1e-4, error_charge_threshold=1e-15 &end
&integrate dt_integration=4e-13, start_time=0, finish_time=200e-12, space_charge=1 &end
"""


# The DC gun deck for 300 steps with beam snapshots and field output (the
# reference's snapshots.c and field_output.c, compiled into the oracle).
DECK_DIAG = DECK_DCGUN.replace("finish_time=300e-12", "finish_time=120e-12").replace(
    "&integrate", '&define_snapshots filename="%s.snap", time_interval=40e-12, start_time=20e-12 &end\n'
    '&define_field_output filename="%s.fld", time_interval=40e-12, start_time=20e-12, z_interval=2, r_interval=4, '
    'separate_imposed_field=1 &end\n&integrate')
sys.path.insert(0, os.path.dirname(HERE))
from golden_columns import FLD_COLUMNS, ONAXIS_COLUMNS, SNAP_COLUMNS, STATUS_COLUMNS  # noqa: E402

# An on-axis RF field (add_on_axis_fields, onAxisFields.c) over the DC gun:
# a synthetic two-harmonic Ez(z) table of 201 equispaced points, offset to
# cover the cathode, pushed with the third-order off-axis expansion; the
# cathode's Richardson-Schottky current density (cathode.c:673-715) reads
# the same expansion at its position each step.
DECK_ONAXIS = """&define_geometry nz=151, nr=101, zmin=0.0, zmax=0.03, rmax=0.02, boundary="dc.geo" &end
&define_cathode z_position=1e-6, outer_radius=0.002, temperature=1800, work_function=2.0, start_time=0,
    stop_time=60e-12, number_per_step=10, initial_pz=1e-6 &end
&add_on_axis_fields filename="rf.sdds", z_name="z", Ez_name="Ez", Ez_peak=8e6, frequency=2.856e9, phase=220,
    z_offset=-0.001, fields_used="%s.oaf" &end
&define_screen filename="oa.sc1", z_position=0.012, direction="forward" &end
&poisson_correction step_interval=4, accuracy=1e-4, error_charge_threshold=1e-15 &end
&integrate dt_integration=4e-13, start_time=0, finish_time=140e-12, space_charge=1, imposed_Efield_ramp_time=20e-12 &end
"""


# The DC gun deck with the moving window (translate, translate.c): once a
# particle passes z = 8 mm the problem moves by dz each step that one lies
# past the (moving) trigger.
DECK_TRANSLATE = DECK_DCGUN.replace("&integrate", "&translate z_trigger=0.008 &end\n&integrate")


# The DC gun deck with integrate's lost_particles file (advance_particles.c:
# 437-487, 577-603; findLossCoordinates, secondaryEmission.c:239), a cathode
# wider than the anode hole and a stronger radial field, so particles are
# lost on the anode plate as well as through the exit.
DECK_LOST = DECK_DCGUN.replace("space_charge=1,", 'lost_particles="%s.lost", space_charge=1,').replace(
    "outer_radius=0.002", "outer_radius=0.0045").replace("Br=1e-4", "Br=2e-3")
LOST_COLUMNS = ["t", "rLost", "zLost", "pz", "pr", "z0", "r0", "q", "generation", "particleID"]


def deck_lost(geo):
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(geo)
    cmds = [b.strip() + " &end" for b in DECK_LOST.split("&end") if b.strip()]
    # the lost-particle table is the first the reference closes (integrate.c:203)
    res = pyoracle.run_reference([("command", c) for c in cmds] + [("table", 2, LOST_COLUMNS), ("get_beam",)], cwd=d,
                                 capacity=20000)
    lost, rb = res
    save("deck_lost", deck=np.array(DECK_LOST), geo=np.array(geo), lost_pages=lost["pages"],
         **{"lost_" + k: lost[k] for k in LOST_COLUMNS}, **beam_out(rb))


# Secondary emission (secondaryEmission.c): the lost-particle deck with the
# anode's face and hole edge drawn as material 1 (the &po material_id), a
# yield table in eV and secondaries of beta*gamma 0.01 released away from
# the surface; the gap field drives them back into the anode, so generations
# cascade: the primaries (300 keV) release about 2.5 each, the returning
# low-energy secondaries (tens of eV) fewer than one; at most 3 per source.
DECK_SECONDARY = DECK_LOST.replace(
    "&integrate", '&define_secondary_emission input_file="yield.sdds", kinetic_energy_column="K", '
    'yield_column="Y", emitted_momentum=0.01, yield_limit=3, verbosity=0, log_file="%s.sel" &end\n&integrate')
SECONDARY_LOG_COLUMNS = ["z", "r", "t", "K", "yield", "emitted", "directionCode", "generation"]
SECONDARY_YIELD = (np.array([0.0, 10.0, 50.0, 200.0, 1e3, 1e4, 1e5, 5e5, 2e6]),
                   np.array([0.0, 0.5, 0.9, 0.9, 1.0, 1.5, 2.0, 2.5, 2.0]))


def secondary_geo(geo):
    """The DC gun boundary with material_id=1 on the anode's face and hole edge."""
    out = []
    for line in geo.splitlines():
        if line.startswith("&po x=0.01, y=0.003,") or line.startswith("&po x=0.0102, y=0.003,"):
            line = line.replace(" &end", ", material_id=1 &end")
        out.append(line)
    assert sum("material_id" in x for x in out) == 2
    return "\n".join(out) + "\n"


def write_yield(path):
    with open(path, "w") as f:
        f.write("SDDS1\n&column name=K type=double units=eV &end\n&column name=Y type=double &end\n"
                "&data mode=ascii no_row_counts=1 &end\n")
        for a, b in zip(*SECONDARY_YIELD):
            f.write("%.17g %.17g\n" % (a, b))


def deck_secondary(geo):
    geo = secondary_geo(geo)
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(geo)
    write_yield(os.path.join(d, "yield.sdds"))
    cmds = [b.strip() + " &end" for b in DECK_SECONDARY.split("&end") if b.strip()]
    res = pyoracle.run_reference([("command", c) for c in cmds] + [("table", 2, LOST_COLUMNS), ("get_beam",),
                                                                   ("screen", 0),
                                                                   ("table", 200, SECONDARY_LOG_COLUMNS)],
                                 cwd=d, capacity=40000)
    lost, rb, rs, sel = res
    out = dict(deck=np.array(DECK_SECONDARY), geo=np.array(geo), yield_K=SECONDARY_YIELD[0],
               yield_Y=SECONDARY_YIELD[1], lost_pages=lost["pages"], **{"lost_" + k: lost[k] for k in LOST_COLUMNS},
               **beam_out(rb), log_pages=sel["pages"], **{"log_" + k: sel[k] for k in SECONDARY_LOG_COLUMNS})
    out.update({"screen0_" + k: v for k, v in rs.items()})
    save("deck_secondary", **out)


# Surface emitters (emitter.c): the DC gun's cathode plane drawn as material
# 2 out to r = 1 mm and material 3 out to 2 mm; no define_cathode.  Material
# 2 emits thermionically (Richardson-Schottky, with a time profile),
# material 3 by field emission; both from the emitter surface the boundary
# list yields (getBoundaryPoints).
DECK_EMITTER = """&define_geometry nz=151, nr=101, zmin=0.0, zmax=0.03, rmax=0.02, boundary="dc.geo" &end
&define_emitter material_id=2, temperature=2500, work_function=3.0, electrons_per_macroparticle=1e7,
    start_time=0, stop_time=40e-12, initial_p=1e-3, random_number_seed=12345,
    profile="prof.sdds", profile_time_name="t", profile_factor_name="A" &end
&define_emitter material_id=3, field_emission=1, work_function=4.5, field_emission_beta=100,
    electrons_per_macroparticle=1e6, stop_time=60e-12, initial_p=1e-3, random_number_seed=777 &end
&define_screen filename="deck.sc1", z_position=0.012, direction="forward" &end
&poisson_correction step_interval=4, accuracy=1e-4, error_charge_threshold=1e-15 &end
&integrate dt_integration=4e-13, start_time=0, finish_time=150e-12, space_charge=1, imposed_Efield_ramp_time=20e-12 &end
"""
EMITTER_PROFILE = (np.array([0.0, 20e-12, 40e-12]), np.array([0.5, 1.0, 0.8]))


def emitter_geo(geo):
    """The DC gun boundary with the cathode plane split at r = 1 and 2 mm into
    materials 2 and 3."""
    lines = geo.splitlines()
    assert lines[0].startswith("&po x=0.0, y=0.0,") and lines[1].startswith("&po x=0.0, y=0.02,")
    extra = ["&po x=0.0, y=0.001, potential=0.0, material_id=2 &end",
             "&po x=0.0, y=0.002, potential=0.0, material_id=3 &end"]
    return "\n".join(lines[:1] + extra + lines[1:]) + "\n"


def write_profile(path, t, A):
    with open(path, "w") as f:
        f.write("SDDS1\n&column name=t type=double &end\n&column name=A type=double &end\n"
                "&data mode=ascii no_row_counts=1 &end\n")
        for a, b in zip(t, A):
            f.write("%.17g %.17g\n" % (a, b))


def deck_emitter(geo):
    geo = emitter_geo(geo)
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(geo)
    write_profile(os.path.join(d, "prof.sdds"), *EMITTER_PROFILE)
    cmds = [b.strip() + " &end" for b in DECK_EMITTER.split("&end") if b.strip()]
    res = pyoracle.run_reference([("command", c) for c in cmds] + [("mesh",), ("get_beam",), ("screen", 0)] +
                                 [("get_field", n) for n in ("Ez", "Er", "Bphi", "Psi")] +
                                 [("boundary_points", m) for m in (2, 3)], cwd=d, capacity=40000)
    mesh, rb, rs = res[0], res[1], res[2]
    out = dict(deck=np.array(DECK_EMITTER), geo=np.array(geo), prof_t=EMITTER_PROFILE[0],
               prof_A=EMITTER_PROFILE[1], time=mesh["time"], **beam_out(rb))
    for m, (iz, ir, dr) in zip((2, 3), res[7:9]):
        out.update({f"bp{m}_iz": iz, f"bp{m}_ir": ir, f"bp{m}_dir": dr})
    out.update({"screen0_" + k: v for k, v in rs.items()})
    out.update(dict(zip(("Ez", "Er", "Bphi", "Psi"), res[3:7])))
    save("deck_emitter", **out)


# Field sampling (field_sampling.c) on the DC gun deck: pages of Ez, all of
# E, Br (the TM-only one of Br and Bphi, field_sampling.c:80-85), Phi (plus the imposed
# potential), Q (which, after a Phi definition, also gets the imposed
# potential added), Jz and Jr at 40 ps intervals; time sequences of Ez
# along z and of Er along r (which averages over the last z range and
# radius the call set) every 4 and 8 ps.
DECK_SAMPLING = DECK_DCGUN.replace("finish_time=300e-12", "finish_time=160e-12").replace(
    "&integrate",
    '&define_field_sampling filename="%s.ez", component="Ez", direction="z", min_coord=0, max_coord=0.03, '
    'position=0.001, time_interval=40e-12 &end\n'
    '&define_field_sampling filename="%s.e", component="EAll", direction="r", min_coord=0, max_coord=0.01, '
    'position=0.005, time_interval=40e-12, start_time=20e-12 &end\n'
    '&define_field_sampling filename="%s.br", component="Br", direction="z", min_coord=0.002, max_coord=0.02, '
    'position=0.002, time_interval=40e-12 &end\n'
    '&define_field_sampling filename="%s.phi", component="Phi", direction="r", min_coord=0, max_coord=0.015, '
    'position=0.008, time_interval=40e-12 &end\n'
    '&define_field_sampling filename="%s.q", component="Q", direction="z", min_coord=0, max_coord=0.012, '
    'position=0.0005, time_interval=40e-12 &end\n'
    '&define_field_sampling filename="%s.jz", component="Jz", direction="z", min_coord=0, max_coord=0.012, '
    'position=0.0004, time_interval=40e-12 &end\n'
    '&define_field_sampling filename="%s.jr", component="Jr", direction="r", min_coord=0, max_coord=0.004, '
    'position=0.003, time_interval=40e-12 &end\n'
    '&define_field_sampling filename="%s.ezt", component="Ez", direction="z", min_coord=0.002, max_coord=0.004, '
    'position=0.001, time_interval=4e-12, time_sequence=1 &end\n'
    '&define_field_sampling filename="%s.ert", component="Er", direction="r", min_coord=0, max_coord=0.004, '
    'position=0.006, time_interval=8e-12, time_sequence=1 &end\n'
    "&integrate")
SAMPLING_PAGES = [("ez", ["z", "Ez"]), ("e", ["r", "Ez", "Er", "Ephi"]), ("br", ["z", "Br"]), ("phi", ["r", "Phi"]),
                  ("q", ["z", "Q"]), ("jz", ["z", "Jz"]), ("jr", ["r", "Jr"])]
SAMPLING_SEQ = [("ezt", ["t", "Ez"]), ("ert", ["t", "Er"])]


def deck_sampling(geo):
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(geo)
    cmds = [b.strip() + " &end" for b in DECK_SAMPLING.split("&end") if b.strip()]
    prog = [("command", c) for c in cmds]
    prog += [("table", 300 + k, cols) for k, (_, cols) in enumerate(SAMPLING_PAGES)]
    prog += [("table", 100 + k, cols) for k, (_, cols) in enumerate(SAMPLING_SEQ)]
    res = pyoracle.run_reference(prog, cwd=d, capacity=20000)
    out = dict(deck=np.array(DECK_SAMPLING), geo=np.array(geo))
    for (name, cols), t in zip(SAMPLING_PAGES + SAMPLING_SEQ, res):
        out[name + "_pages"] = t["pages"]
        for c in cols:
            out[name + "_" + c] = t[c]
    save("deck_sampling", **out)


# The DC gun deck with define_field_saving (field_saving.c:46-213): saves at
# 0 and 100 ps and before exiting.  The saved columns are compared through
# SHA-256 digests of their values (bit-for-bit equality needs nothing more,
# and the fixture stays small).
DECK_FIELDSAVE = DECK_DCGUN.replace("finish_time=300e-12", "finish_time=140e-12").replace(
    "&integrate", '&define_field_saving filename="%s.flds", time_interval=100e-12, save_before_exiting=1 &end\n'
    "&integrate")
SAVE_COLUMNS = ["Ez", "Er", "Jz", "Jr", "Bphi", "Bphi2", "metalFlags"]


def digest(a):
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a, np.float64).tobytes()).hexdigest()


def deck_fieldsave(geo):
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(geo)
    cmds = [b.strip() + " &end" for b in DECK_FIELDSAVE.split("&end") if b.strip()]
    t, = pyoracle.run_reference([("command", c) for c in cmds] + [("table", 3 + 16, SAVE_COLUMNS)], cwd=d,
                                capacity=20000)
    save("deck_fieldsave", deck=np.array(DECK_FIELDSAVE), geo=np.array(geo), pages=t["pages"], rows=len(t["Ez"]),
         **{"sha_" + c: np.array(digest(t[c])) for c in SAVE_COLUMNS},
         **{"head_" + c: t[c][:64] for c in SAVE_COLUMNS})


def deck_translate(geo):
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(geo)
    cmds = [b.strip() + " &end" for b in DECK_TRANSLATE.split("&end") if b.strip()]
    res = pyoracle.run_reference([("command", c) for c in cmds] + [("mesh",), ("get_beam",), ("screen", 0)] +
                                 [("get_field", n) for n in ("Ez", "Er", "Bphi", "Psi")], cwd=d, capacity=20000)
    mesh, rb, rs = res[0], res[1], res[2]
    out = dict(deck=np.array(DECK_TRANSLATE), geo=np.array(geo), time=mesh["time"], zmin=mesh["zmin"],
               zmax=mesh["zmax"], **beam_out(rb))
    out.update({"screen0_" + k: v for k, v in rs.items()})
    out.update(dict(zip(("Ez", "Er", "Bphi", "Psi"), res[3:7])))
    save("deck_translate", **out)


# The on-axis deck with integrate's status file (status_pr.c): a row every
# 50 steps and one after the loop.
DECK_STATUS = None  # set after DECK_ONAXIS


def deck_status(geo):
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(geo)
    rz, rE = rf_profile()
    write_rf(os.path.join(d, "rf.sdds"), rz, rE)
    cmds = [b.strip() + " &end" for b in DECK_STATUS.split("&end") if b.strip()]
    res = pyoracle.run_reference([("command", c) for c in cmds] + [("table", 100, STATUS_COLUMNS)], cwd=d,
                                 capacity=20000)
    st = res[0]
    save("deck_status", deck=np.array(DECK_STATUS), geo=np.array(geo), rf_z=rz, rf_Ez=rE, rows=len(st["t"]),
         **{"st_" + k: st[k] for k in STATUS_COLUMNS})


def rf_profile():
    u = np.arange(201) / 200.0
    return u * 0.02, np.sin(np.pi * u) + 0.3 * np.sin(2 * np.pi * u)


DECK_STATUS = DECK_ONAXIS.replace("space_charge=1, imposed", 'status_interval=50, status_output="%s.status", '
                                  "space_charge=1, imposed")


def write_rf(path, z, Ez):
    with open(path, "w") as f:
        f.write("SDDS1\n&column name=z type=double units=m &end\n&column name=Ez type=double &end\n"
                "&data mode=ascii no_row_counts=1 &end\n")
        for a, b in zip(z, Ez):
            f.write("%.17g %.17g\n" % (a, b))


def decks():
    geo = str(np.load(os.path.join(HERE, "dcgun_geometry.npz"))["geo"])
    for name, deck, screens in (("deck_dcgun", DECK_DCGUN, 1), ("deck_testbeam", DECK_TESTBEAM, 1)):
        d = tempfile.mkdtemp()
        with open(os.path.join(d, "dc.geo"), "w") as f:
            f.write(geo)
        cmds = [b.strip() + " &end" for b in deck.split("&end") if b.strip()]
        prog = [("command", c) for c in cmds] + [("mesh",), ("get_beam",)]
        prog += [("screen", i) for i in range(screens)]
        prog += [("get_field", n) for n in ("Ez", "Er", "Bphi", "Psi")]
        res = pyoracle.run_reference(prog, cwd=d, capacity=20000)
        mesh, rb, scr, fields = res[0], res[1], res[2:2 + screens], res[2 + screens:]
        out = dict(deck=np.array(deck), geo=np.array(geo), time=mesh["time"], **beam_out(rb))
        for i, rs in enumerate(scr):
            out.update({f"screen{i}_{k}": v for k, v in rs.items()})
        out.update(dict(zip(("Ez", "Er", "Bphi", "Psi"), fields)))
        save(name, **out)
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(geo)
    cmds = [b.strip() + " &end" for b in DECK_DIAG.split("&end") if b.strip()]
    snap, fld = pyoracle.run_reference([("command", c) for c in cmds] + [("table", 0, SNAP_COLUMNS),
                                                                       ("table", 1, FLD_COLUMNS)],
                                       cwd=d, capacity=20000)
    save("deck_diagnostics", deck=np.array(DECK_DIAG), geo=np.array(geo), snap_pages=snap["pages"],
         fld_pages=fld["pages"], **{"snap_" + k: snap[k] for k in SNAP_COLUMNS},
         **{"fld_" + k: fld[k] for k in FLD_COLUMNS})
    deck_onaxis(geo)
    deck_translate(geo)
    deck_status(geo)
    deck_lost(geo)
    deck_fieldsave(geo)
    deck_secondary(geo)
    deck_emitter(geo)
    deck_sampling(geo)


def deck_onaxis(geo):
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(geo)
    rz, rE = rf_profile()
    write_rf(os.path.join(d, "rf.sdds"), rz, rE)
    cmds = [b.strip() + " &end" for b in DECK_ONAXIS.split("&end") if b.strip()]
    res = pyoracle.run_reference([("command", c) for c in cmds] + [("mesh",), ("get_beam",), ("screen", 0)] +
                                 [("get_field", n) for n in ("Ez", "Er", "Bphi", "Psi")] +
                                 [("table", 2, ONAXIS_COLUMNS)], cwd=d, capacity=20000)
    mesh, rb, rs, oaf = res[0], res[1], res[2], res[-1]
    out = dict(deck=np.array(DECK_ONAXIS), geo=np.array(geo), rf_z=rz, rf_Ez=rE, time=mesh["time"], **beam_out(rb))
    out.update({"screen0_" + k: v for k, v in rs.items()})
    out.update(dict(zip(("Ez", "Er", "Bphi", "Psi"), res[3:7])))
    out.update({"oaf_" + k.replace("/", "_"): oaf[k] for k in ONAXIS_COLUMNS})
    save("deck_onaxis", **out)


if __name__ == "__main__":
    if sys.argv[1:] == ["decks"]:
        decks()
    elif sys.argv[1:] == ["status"]:
        deck_status(str(np.load(os.path.join(HERE, "dcgun_geometry.npz"))["geo"]))
    elif sys.argv[1:] == ["translate"]:
        deck_translate(str(np.load(os.path.join(HERE, "dcgun_geometry.npz"))["geo"]))
    elif sys.argv[1:] == ["fieldsave"]:
        deck_fieldsave(str(np.load(os.path.join(HERE, "dcgun_geometry.npz"))["geo"]))
    elif sys.argv[1:] == ["sampling"]:
        deck_sampling(str(np.load(os.path.join(HERE, "dcgun_geometry.npz"))["geo"]))
    elif sys.argv[1:] == ["emitter"]:
        deck_emitter(str(np.load(os.path.join(HERE, "dcgun_geometry.npz"))["geo"]))
    elif sys.argv[1:] == ["secondary"]:
        deck_secondary(str(np.load(os.path.join(HERE, "dcgun_geometry.npz"))["geo"]))
    elif sys.argv[1:] == ["lost"]:
        deck_lost(str(np.load(os.path.join(HERE, "dcgun_geometry.npz"))["geo"]))
    elif sys.argv[1:] == ["te"]:
        te()
    elif sys.argv[1:] == ["onaxis"]:
        deck_onaxis(str(np.load(os.path.join(HERE, "dcgun_geometry.npz"))["geo"]))
    else:
        main()
        te()
        decks()
