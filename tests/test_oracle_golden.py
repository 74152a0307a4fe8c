"""The CPU oracle reproduces, bit for bit, the fixtures the reference wrote."""
import numpy as np

from spiffe_b200 import abi, workloads
from oracle import pyoracle
from helpers import MODES, TE_FIELDS, beam_from, fields_from, load, te_fdtd_state, te_push_state


def test_fdtd_pillbox_400_steps(oracle):
    fx = load("pillbox_fdtd")
    f = fields_from(fx, dt=float(fx["dt"]))
    f["Ez"] = fx["Ez0"]
    for _ in range(int(fx["steps"])):
        oracle.advance_fields(f)
    for n in ("Ez", "Er", "Bphi", "Bphi2"):
        assert np.array_equal(f[n], fx[n]), n


def test_push_and_deposit(oracle):
    fx = load("pillbox_push")
    f = fields_from(fx, modes=int(fx["modes"]), dt=float(fx["dt"]))
    f.mesh.time_step = int(fx["time_step"])
    f.mesh.time = f.mesh.time_step * f.mesh.dt
    for k in ("Ez", "Er", "Bphi", "Bphi2", "EzImposed", "ErImposed", "BzImposed", "BrImposed"):
        f[k] = fx["f_" + k]
    b = beam_from(fx)
    oracle.zero_currents(f)
    oracle.deposit(f, b)
    assert np.array_equal(f["Jz"], fx["Jz"]) and np.array_equal(f["Jr"], fx["Jr"])
    sc = abi.Screen(float(fx["screen_z"]))
    oracle.advance_particles(f, b, [sc], abi.push_options(compaction=abi.COMPACT_REFERENCE,
                                                           screen_momentum=abi.SCREEN_REFERENCE))
    assert b.np == int(fx["out_np"]) and b.npActive == int(fx["out_npActive"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(b[k], fx["out_" + k]), k
    rec = sc.records()
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rec[c], fx["screen_" + c]), c


def test_dcgun_imposed_field_and_poisson_correction(oracle):
    import ctypes as C

    fx = load("dcgun_poisson")
    modes = MODES | abi.FL_SPACE_CHARGE
    f = fields_from(fx, modes=modes, dt=float(fx["dt"]))
    f["PsiImposed"] = fx["PsiImposed0"]
    opts = abi.poisson_options(step_interval=1, accuracy=1e-6, maximum_iterations=1000)
    last, it = C.c_double(-1), C.c_int64(0)
    oracle.lib.orc_imposed_efield(C.byref(f.mesh), C.byref(f.c()), C.byref(opts), 1, C.byref(last), C.byref(it))
    for n in ("PsiImposed", "EzImposed", "ErImposed"):
        assert np.array_equal(f[n], fx[n]), n
    f["Ez"], f["Er"] = fx["Ez0"], fx["Er0"]
    b = beam_from(fx)
    rep = oracle.poisson_correction(f, b, 1, opts)
    assert rep.ran == 1 and rep.iterations > 0
    for n in ("Ez", "Er", "Psi", "Q"):
        assert np.array_equal(f[n], fx[n]), n


def test_loop_with_emission(oracle):
    fx = load("pillbox_loop")
    cfg = workloads.PillboxConfig()
    f = fields_from(fx, modes=MODES | abi.FL_SPACE_CHARGE, dt=float(fx["dt"]))
    f["Ez"] = fx["Ez0"]
    b = abi.Beam(40000)
    sc = abi.Screen(float(fx["screen_z"]), capacity=40000)
    run = pyoracle.OracleRun(oracle, f, b, space_charge=1, screens=[sc])
    run.add_cathode(cfg.cathode_options())
    run.begin()
    for _ in range(int(fx["steps"])):
        run.step()
    for n in ("Ez", "Er", "Bphi", "Jz", "Jr"):
        assert np.array_equal(f[n], fx[n]), n
    assert b.np == int(fx["out_np"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(b[k], fx["out_" + k]), k
    rec = sc.records()
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rec[c], fx["screen_" + c]), c


def test_fdtd_te_fields_25_steps(oracle):
    """The TE part of advance_field_solutions (integrate.c:434-540) with the
    TM part, from random fields and currents on the gun mesh."""
    fx = load("gun16_te")
    f = te_fdtd_state(fx)
    for _ in range(int(fx["steps"])):
        oracle.advance_fields(f)
    for n in TE_FIELDS:
        assert np.array_equal(f[n], fx[n]), n


def test_te_deposit_and_push(oracle):
    """Jphi deposition (space_charge.c:218-295) and the gather of Ephi, Br2
    and Bz2 (advance_particles.c:649-825) in a push with TE fields."""
    fx = load("gun16_te")
    f, b, sub = te_push_state(fx)
    oracle.zero_currents(f)
    oracle.deposit(f, b)
    for n in ("Jz", "Jr", "Jphi"):
        assert np.array_equal(f[n], sub[n]), n
    oracle.advance_particles(f, b, [], abi.push_options(compaction=abi.COMPACT_REFERENCE,
                                                        screen_momentum=abi.SCREEN_REFERENCE))
    assert b.np == int(sub["out_np"]) and b.npActive == int(sub["out_npActive"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(b[k], sub["out_" + k]), k
