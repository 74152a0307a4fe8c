"""The link-time drop-in: spiffe's own loop on the device library.

spiffe_b200/dropin/spiffe_dropin.c defines advance_field_solutions,
add_particle_currents, advance_particles, solve_poisson_cyl and the Poisson
correction with the reference's prototypes.  Built against the reference's
spiffe.h (oracle/Makefile, target dropin) and preloaded ahead of the
reference's own objects, its definitions are the ones the reference's
perform_integration (integrate.c:134-194) and command processors call.  The
reference then runs its input decks unchanged, with the hot path on the
GPU, and every result must equal the pure reference run's fixture bit for
bit: the drop-in uses the FP64 form with the reference's compaction,
screen-momentum and deposition order.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle
from spiffe_b200 import abi, workloads
from helpers import fields_from, load

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(pyoracle.DROPIN_SO) and pyoracle.reference_available()),
                                 reason="the drop-in and the reference build are absent")]


def run_with_dropin(program, cwd, capacity=40000):
    return pyoracle.run_reference(program, cwd=cwd, capacity=capacity, preload=[pyoracle.DROPIN_SO])


def write_profile(d, t, A):
    with open(os.path.join(d, "prof.sdds"), "w") as f:
        f.write("SDDS1\n&column name=t type=double &end\n&column name=A type=double &end\n"
                "&data mode=ascii no_row_counts=1 &end\n")
        for a, b in zip(t, A):
            f.write("%.17g %.17g\n" % (a, b))


def test_perform_integration_with_emission(tmp_path):
    """The config-1 pillbox through the reference's perform_integration for
    220 steps with cathode emission (20,251 particles) and a screen."""
    fx = load("pillbox_loop")
    cfg = workloads.PillboxConfig()
    d = str(tmp_path)
    with open(os.path.join(d, "pillbox.geo"), "w") as f:
        f.write(cfg.geo_text())
    write_profile(d, fx["prof_t"], fx["prof_A"])
    nsteps = int(fx["steps"])
    cath = workloads.namelist("define_cathode", z_position=0.0, outer_radius=cfg.cathode_radius,
                              current_density=cfg.peak_current_density(), electrons_per_macroparticle=cfg.epm,
                              profile="prof.sdds", profile_time_name="t", profile_factor_name="A",
                              random_number_seed=cfg.seed)
    scr = workloads.namelist("define_screen", filename="exit", z_position=float(fx["screen_z"]))
    integ = workloads.namelist("integrate", dt_integration=cfg.dt, finish_time=(nsteps + 0.5) * cfg.dt,
                               space_charge=1)
    res = run_with_dropin([("command", cfg.geometry()), ("set_field", "Ez", fx["Ez0"]), ("command", cath),
                           ("command", scr), ("command", integ), ("get_field", "Ez"), ("get_field", "Er"),
                           ("get_field", "Bphi"), ("get_field", "Jz"), ("get_field", "Jr"), ("get_beam",),
                           ("screen", 0)], d)
    Ez, Er, Bphi, Jz, Jr, rb, rs = res
    for n, a in (("Ez", Ez), ("Er", Er), ("Bphi", Bphi), ("Jz", Jz), ("Jr", Jr)):
        assert np.array_equal(a, fx[n]), n
    assert rb["np"] == int(fx["out_np"]) > 20000
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(rb[k], fx["out_" + k]), k
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rs[c], fx["screen_" + c]), c


def test_dc_gun_deck(tmp_path):
    """The DC gun deck: imposed-field Laplace solve and ramp, ring-coil
    solenoid, constant Br, cathode with distribution correction, a screen and
    the Poisson correction every 4 steps (compute_imposed_Efield,
    add_poisson_correction and solve_poisson_cyl from the drop-in)."""
    fx = load("deck_dcgun")
    d = str(tmp_path)
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(str(fx["geo"]))
    deck = str(fx["deck"])
    cmds = [b.strip() + " &end" for b in deck.split("&end") if b.strip()]
    res = run_with_dropin([("command", c) for c in cmds] + [("mesh",), ("get_beam",), ("screen", 0)] +
                          [("get_field", n) for n in ("Ez", "Er", "Bphi", "Psi")], d, capacity=20000)
    mesh, rb, rs = res[0], res[1], res[2]
    assert mesh["time"] == float(fx["time"])
    for n, a in zip(("Ez", "Er", "Bphi", "Psi"), res[3:7]):
        assert np.array_equal(a, fx[n]), n
    assert rb["np"] == int(fx["out_np"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(rb[k], fx["out_" + k]), k
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rs[c], fx["screen0_" + c]), c


def test_solve_poisson_cyl(tmp_path):
    """solve_poisson_cyl on row-pointer arrays: the same half-sweep count and
    potential as the reference's own routine."""
    fx = load("dcgun_poisson")
    d = str(tmp_path)
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(str(load("dcgun_geometry")["geo"]))
    cmd = workloads.geometry_command(int(fx["nz"]), int(fx["nr"]), 0.0, 0.030, 0.020, "dc.geo")
    f = fields_from(fx)
    rng = np.random.default_rng(7)
    psi = rng.normal(size=f.shape)
    rhs = rng.normal(size=f.shape) * 1e4
    prog = [("command", cmd), ("solve_poisson", psi, rhs, 1e-6, 3000), ("solve_poisson", psi, None, 1e-6, 200)]
    ref = pyoracle.run_reference(prog, cwd=d)
    got = run_with_dropin(prog, d)
    for (n_r, p_r), (n_g, p_g) in zip(ref, got):
        assert n_r == n_g
        assert np.array_equal(p_r, p_g)


def test_lost_particle_file(tmp_path):
    """integrate's lost_particles file through the drop-in: the reference's
    own perform_integration hands SDDSlost to the drop-in's
    advance_particles, which writes the rows it gets from the device."""
    fx = load("deck_lost")
    d = str(tmp_path)
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(str(fx["geo"]))
    cmds = [b.strip() + " &end" for b in str(fx["deck"]).split("&end") if b.strip()]
    cols = ["t", "rLost", "zLost", "pz", "pr", "z0", "r0", "q", "generation", "particleID"]
    lost, = run_with_dropin([("command", c) for c in cmds] + [("table", 2, cols)], d, capacity=20000)
    assert lost["pages"] == int(fx["lost_pages"])
    for c in cols:
        assert np.array_equal(lost[c], fx["lost_" + c]), c


def test_secondary_emission(tmp_path):
    """Secondary emission through the drop-in: the device pushes and reports
    each lost particle's loss point, impact momentum and side; the
    reference's own queueSecondaryEmission and emitSecondaryElectrons do the
    rest on the host beam.  The lost-particle file and the final beam equal
    the pure reference run's."""
    fx = load("deck_secondary")
    d = str(tmp_path)
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(str(fx["geo"]))
    with open(os.path.join(d, "yield.sdds"), "w") as f:
        f.write("SDDS1\n&column name=K type=double units=eV &end\n&column name=Y type=double &end\n"
                "&data mode=ascii no_row_counts=1 &end\n")
        for a, b in zip(fx["yield_K"], fx["yield_Y"]):
            f.write("%.17g %.17g\n" % (a, b))
    cmds = [b.strip() + " &end" for b in str(fx["deck"]).split("&end") if b.strip()]
    cols = ["t", "rLost", "zLost", "pz", "pr", "z0", "r0", "q", "generation", "particleID"]
    lost, rb = run_with_dropin([("command", c) for c in cmds] + [("table", 2, cols), ("get_beam",)], d,
                               capacity=40000)
    assert lost["pages"] == int(fx["lost_pages"])
    for c in cols:
        assert np.array_equal(lost[c], fx["lost_" + c]), c
    assert rb["np"] == int(fx["out_np"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(rb[k], fx["out_" + k]), k


def test_emitters(tmp_path):
    """Surface emitters through the drop-in: the reference's own
    emit_electrons_from_emitter and setEmitterCurrentDensity read the host
    fields the drop-in brings back each step and append to the host beam;
    fields, beam and screen equal the pure reference run's."""
    fx = load("deck_emitter")
    d = str(tmp_path)
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(str(fx["geo"]))
    write_profile(d, fx["prof_t"], fx["prof_A"])
    cmds = [b.strip() + " &end" for b in str(fx["deck"]).split("&end") if b.strip()]
    res = run_with_dropin([("command", c) for c in cmds] + [("mesh",), ("get_beam",), ("screen", 0)] +
                          [("get_field", n) for n in ("Ez", "Er", "Bphi", "Psi")], d, capacity=40000)
    mesh, rb, rs = res[0], res[1], res[2]
    assert mesh["time"] == float(fx["time"])
    for n, a in zip(("Ez", "Er", "Bphi", "Psi"), res[3:7]):
        assert np.array_equal(a, fx[n]), n
    assert rb["np"] == int(fx["out_np"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(rb[k], fx["out_" + k]), k
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rs[c], fx["screen0_" + c]), c


def test_field_sampling(tmp_path):
    """Field sampling through the drop-in: the reference's own sample_fields
    reads the host fields the drop-in brings back each step; every sampled
    file equals the pure reference run's."""
    fx = load("deck_sampling")
    d = str(tmp_path)
    with open(os.path.join(d, "dc.geo"), "w") as f:
        f.write(str(fx["geo"]))
    pages = [("ez", ["z", "Ez"]), ("e", ["r", "Ez", "Er", "Ephi"]), ("br", ["z", "Br"]), ("phi", ["r", "Phi"]),
             ("q", ["z", "Q"]), ("jz", ["z", "Jz"]), ("jr", ["r", "Jr"])]
    seq = [("ezt", ["t", "Ez"]), ("ert", ["t", "Er"])]
    cmds = [b.strip() + " &end" for b in str(fx["deck"]).split("&end") if b.strip()]
    prog = [("command", c) for c in cmds] + [("table", 300 + k, cols) for k, (_, cols) in enumerate(pages)]
    prog += [("table", 100 + k, cols) for k, (_, cols) in enumerate(seq)]
    res = run_with_dropin(prog, d, capacity=20000)
    for (name, cols), t in zip(pages + seq, res):
        assert t["pages"] == int(fx[name + "_pages"]), name
        for c in cols:
            assert np.array_equal(t[c], fx[name + "_" + c]), (name, c)
