"""Parity of the plain FP64 CUDA path with the reference, through the C ABI.

Bit-exact where the arithmetic is order-free (FDTD, push, SOR updates,
ordered deposition); within a stated tolerance where the device sums in a
different order (FP64 atomics: relative L2 <= 1e-12 after one step).
"""
import numpy as np
import pytest

from spiffe_b200 import abi, gpu, workloads
from oracle import pyoracle
from helpers import MODES, TE_FIELDS, beam_from, by_id, fields_from, load, rel_l2, te_fdtd_state, te_push_state

pytestmark = pytest.mark.gpu

ATOMIC_TOL = 1e-12


def push_fixture_state(fx):
    f = fields_from(fx, modes=int(fx["modes"]), dt=float(fx["dt"]))
    f.mesh.time_step = int(fx["time_step"])
    f.mesh.time = f.mesh.time_step * f.mesh.dt
    for k in ("Ez", "Er", "Bphi", "Bphi2", "EzImposed", "ErImposed", "BzImposed", "BrImposed"):
        f[k] = fx["f_" + k]
    return f, beam_from(fx)


def test_fdtd_pillbox_bit_exact():
    fx = load("pillbox_fdtd")
    f = fields_from(fx, dt=float(fx["dt"]))
    f["Ez"] = fx["Ez0"]
    g = gpu.GpuInstance(f)
    for _ in range(int(fx["steps"])):
        g.advance_fields()
    out = g.fields(f)
    for n in ("Ez", "Er", "Bphi", "Bphi2"):
        assert np.array_equal(out[n], fx[n]), n


def test_fdtd_te_fields_bit_exact():
    """TE and TM parts of advance_field_solutions (integrate.c:308-540) for
    25 steps from random fields and currents on the gun mesh, against the
    reference's own output (fixture gun16_te)."""
    fx = load("gun16_te")
    f = te_fdtd_state(fx)
    g = gpu.GpuInstance(f)
    for _ in range(int(fx["steps"])):
        g.advance_fields()
    out = g.fields(f)
    for n in TE_FIELDS:
        assert np.array_equal(out[n], fx[n]), n


@pytest.mark.parametrize("ordered", [1, 0])
def test_te_deposit(ordered):
    """Jz, Jr and Jphi (space_charge.c:34-295) with TE fields on."""
    fx = load("gun16_te")
    f, b, sub = te_push_state(fx)
    g = gpu.GpuInstance(f)
    g.set_deposit_order(ordered)
    g.upload_beam(b)
    g.zero_currents()
    g.deposit()
    out = g.fields(f)
    for n in ("Jz", "Jr", "Jphi"):
        if ordered:
            assert np.array_equal(out[n], sub[n]), n
        else:
            assert rel_l2(out[n], sub[n]) <= ATOMIC_TOL, n


def test_te_push_bit_exact():
    """A push whose gather reads Ephi, Br2 and Bz2 (advance_particles.c:
    649-825), against the reference's output."""
    fx = load("gun16_te")
    f, b, sub = te_push_state(fx)
    g = gpu.GpuInstance(f)
    g.upload_beam(b)
    g.advance_particles(abi.push_options(compaction=abi.COMPACT_REFERENCE, screen_momentum=abi.SCREEN_REFERENCE))
    out = g.download_beam(abi.Beam(b.capacity))
    assert out.np == int(sub["out_np"]) and out.npActive == int(sub["out_npActive"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(out[k], sub["out_" + k]), k


@pytest.mark.parametrize("ordered", [1, 0])
def test_deposit(ordered):
    fx = load("pillbox_push")
    f, b = push_fixture_state(fx)
    g = gpu.GpuInstance(f)
    g.set_deposit_order(ordered)
    g.upload_beam(b)
    g.zero_currents()
    g.deposit()
    out = g.fields(f)
    for n in ("Jz", "Jr"):
        if ordered:
            assert np.array_equal(out[n], fx[n]), n
        else:
            assert rel_l2(out[n], fx[n]) <= ATOMIC_TOL, n


def test_push_reference_policies_bit_exact():
    fx = load("pillbox_push")
    f, b = push_fixture_state(fx)
    g = gpu.GpuInstance(f)
    g.upload_beam(b)
    g.add_screen(float(fx["screen_z"]))
    g.advance_particles(abi.push_options(compaction=abi.COMPACT_REFERENCE, screen_momentum=abi.SCREEN_REFERENCE))
    out = g.download_beam(abi.Beam(b.capacity))
    assert out.np == int(fx["out_np"]) and out.npActive == int(fx["out_npActive"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(out[k], fx["out_" + k]), k
    rec = by_id(g.screen(0).records())
    ref = by_id({c: fx["screen_" + c] for c in abi.SCREEN_COLUMNS} | {"particleID": fx["screen_particleID"]})
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rec[c], ref[c]), c


def test_push_swap_compaction_matches_oracle(oracle):
    fx = load("pillbox_push")
    f, b = push_fixture_state(fx)
    opts = abi.push_options(compaction=abi.COMPACT_SWAP, screen_momentum=abi.SCREEN_PARTICLE)
    g = gpu.GpuInstance(f)
    g.upload_beam(b)
    g.add_screen(float(fx["screen_z"]))
    g.advance_particles(opts)
    out = g.download_beam(abi.Beam(b.capacity))
    ref_b = b.copy()
    sc = abi.Screen(float(fx["screen_z"]))
    oracle.advance_particles(f.copy(), ref_b, [sc], opts)
    assert out.np == ref_b.np and out.npActive == ref_b.npActive
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(out[k], ref_b[k]), k
    rec, ref = by_id(g.screen(0).records()), by_id(sc.records())
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rec[c], ref[c]), c


def test_single_test_particle_trajectory(oracle):
    """A single electron in the pillbox's TM010 field for 600 steps."""
    fx = load("pillbox_fdtd")
    f = fields_from(fx, dt=float(fx["dt"]))
    f["Ez"] = fx["Ez0"]
    b = abi.Beam(4)
    b.set(1, z=[0.002], r=[0.003], pz=[0.0], pr=[0.0], r_pphi=[0.0], vz=[0.0], vr=[0.0], vphi=[0.0], Q=[-1e-15],
          r0=[0.003], z0=[0.002], t0=[0.0], rmin=[1e300], rmax=[-1e300], zmin=[1e300], zmax=[-1e300],
          particleID=[1], generation=[0], status=[1])
    b.npActive, b.nextParticleID, b.QoMC, b.stiffness = 1, 2, abi_qomc(), 1.0
    g = gpu.GpuInstance(f)
    g.upload_beam(b)
    ref_f, ref_b = f.copy(), b.copy()
    opts = abi.push_options(compaction=abi.COMPACT_SWAP)
    traj_g, traj_o = [], []
    lost_at = None
    for step in range(600):
        ref_f.mesh.time = step * ref_f.mesh.dt
        g.mesh.time = ref_f.mesh.time
        g.set_mesh()
        g.advance_fields()
        oracle.advance_fields(ref_f)
        g.advance_particles(opts)
        oracle.advance_particles(ref_f, ref_b, [], opts)
        if step % 10 == 9 or ref_b.np == 0:
            out = g.download_beam(abi.Beam(4))
            # the electron is absorbed by the cavity wall on the same step on both sides
            assert out.np == ref_b.np, step
            if ref_b.np == 0:
                lost_at = step
                break
            traj_g.append([out["z"][0], out["r"][0], out["pz"][0], out["pr"][0]])
            traj_o.append([ref_b["z"][0], ref_b["r"][0], ref_b["pz"][0], ref_b["pr"][0]])
    assert len(traj_g) >= 10, lost_at
    traj_g, traj_o = np.array(traj_g), np.array(traj_o)
    assert np.max(np.abs(traj_g - traj_o) / np.maximum(np.abs(traj_o), 1e-30)) <= 1e-9
    assert np.array_equal(traj_g, traj_o)  # the FP64 form is bit-faithful


def abi_qomc():
    return -1.602176634e-19 / (9.1093837015e-31 * 2.99792458e8)


def test_imposed_field_and_sor_bit_exact():
    fx = load("dcgun_poisson")
    f = fields_from(fx, modes=MODES | abi.FL_SPACE_CHARGE, dt=float(fx["dt"]))
    f["PsiImposed"] = fx["PsiImposed0"]
    g = gpu.GpuInstance(f)
    opts = abi.poisson_options(step_interval=1, accuracy=1e-6, maximum_iterations=1000)
    g.imposed_efield(opts, 1)
    out = g.fields(f)
    for n in ("PsiImposed", "EzImposed", "ErImposed"):
        assert np.array_equal(out[n], fx[n]), n


def test_poisson_correction(oracle):
    fx = load("dcgun_poisson")
    modes = MODES | abi.FL_SPACE_CHARGE
    f = fields_from(fx, modes=modes, dt=float(fx["dt"]))
    f["PsiImposed"] = fx["PsiImposed"]
    f["EzImposed"], f["ErImposed"] = fx["EzImposed"], fx["ErImposed"]
    f["Ez"], f["Er"] = fx["Ez0"], fx["Er0"]
    b = beam_from(fx)
    opts = abi.poisson_options(step_interval=1, accuracy=1e-6, maximum_iterations=1000)
    # without particles the correction is order-free: bit-exact against the oracle
    g0 = gpu.GpuInstance(f)
    rep0 = g0.poisson_correction(0, opts)
    ref0 = f.copy()
    orep0 = oracle.poisson_correction(ref0, abi.Beam(1), 0, opts)
    assert rep0.ran == orep0.ran == 1 and rep0.iterations == orep0.iterations
    out0 = g0.fields(f)
    for n in ("Ez", "Er", "Psi", "Q"):
        assert np.array_equal(out0[n], ref0[n]), n
    # with particles the charge is scattered with FP64 atomics
    g = gpu.GpuInstance(f)
    g.upload_beam(b)
    rep = g.poisson_correction(1, opts)
    assert rep.ran == 1 and abs(rep.iterations - 527) <= 1
    out = g.fields(f)
    for n in ("Ez", "Er", "Psi"):
        assert rel_l2(out[n], fx[n]) <= ATOMIC_TOL, n


def test_loop_with_emission_bit_exact():
    """perform_integration for 220 steps with emission and space charge."""
    fx = load("pillbox_loop")
    cfg = workloads.PillboxConfig()
    f = fields_from(fx, modes=MODES | abi.FL_SPACE_CHARGE, dt=float(fx["dt"]))
    f["Ez"] = fx["Ez0"]
    g = gpu.GpuInstance(f, capacity=40000)
    g.set_deposit_order(1)
    g.add_screen(float(fx["screen_z"]), capacity=40000)
    g.add_cathode(cfg.cathode_options())
    g.configure_run(space_charge=1, push=abi.push_options())
    g.run_begin()
    g.run_steps(int(fx["steps"]))
    out = g.fields(f)
    for n in ("Ez", "Er", "Bphi", "Jz", "Jr"):
        assert np.array_equal(out[n], fx[n]), n
    b = g.download_beam(abi.Beam(40000))
    assert b.np == int(fx["out_np"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(b[k], fx["out_" + k]), k
    rec = by_id(g.screen(0, capacity=40000).records())
    ref = by_id({c: fx["screen_" + c] for c in abi.SCREEN_COLUMNS} | {"particleID": fx["screen_particleID"]})
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rec[c], ref[c]), c


def test_device_errors_are_reported():
    fx = load("pillbox_fdtd")
    f = fields_from(fx, dt=float(fx["dt"]))
    g = gpu.GpuInstance(f)
    with pytest.raises(gpu.SpiffeGpuError):
        g.solve_poisson(0, -1.0, 10)  # accuracy <= 0 is rejected as the reference does (poisson.c:27)
    with pytest.raises(gpu.SpiffeGpuError):
        g.add_screen(0.01, direction=2)


def test_counts_async_matches_counts():
    """The queued count read returns what the synchronous one does, step by step."""
    fx = load("pillbox_loop")
    cfg = workloads.PillboxConfig()
    f = fields_from(fx, modes=MODES | abi.FL_SPACE_CHARGE, dt=float(fx["dt"]))
    f["Ez"] = fx["Ez0"]
    g = gpu.GpuInstance(f, capacity=40000)
    g.add_cathode(cfg.cathode_options())
    g.configure_run(space_charge=1, push=abi.push_options())
    g.run_begin()
    g.run_steps(120)  # emission starts near step 70
    out = np.zeros((30, 2), np.int64)
    seen = []
    for k in range(30):
        g.run_steps(1)
        g.counts_async(out[k])
    g.synchronize()
    g2 = gpu.GpuInstance(f, capacity=40000)
    g2.add_cathode(cfg.cathode_options())
    g2.configure_run(space_charge=1, push=abi.push_options())
    g2.run_begin()
    g2.run_steps(120)
    for k in range(30):
        g2.run_steps(1)
        seen.append(g2.counts())
    assert [tuple(r) for r in out] == seen and seen[-1][0] > 0
    g.close()
    g2.close()


def test_on_axis_fields_at_matches_reference_profile():
    """spiffe_gpu_add_on_axis_field and the expansion through the C ABI against
    the reference's fields_used table (onAxisFields.c:130-170): r = 1e-6,
    sine and cosine 1, bit for bit at every z of the DC gun mesh."""
    fx = load("deck_onaxis")
    f = abi.Fields(151, 101, 0.0, 0.03, 0.02)
    g = gpu.GpuInstance(f, capacity=16)
    g.add_on_axis_field(fx["rf_z"], fx["rf_Ez"], Ez_peak=8e6, frequency=2.856e9, phase_rad=220 * np.pi / 180,
                        z_offset=-0.001)
    got = np.array([g.on_axis_fields_at(z, 1e-6, 0.0, profile=True) for z in fx["oaf_z"]])
    assert np.array_equal(got[:, 0], fx["oaf_Ez"])
    assert np.array_equal(got[:, 1] / 1e-6, fx["oaf_Er_r"])
    assert np.array_equal(got[:, 2] / 1e-6, fx["oaf_Bphi_r"])
    with pytest.raises(gpu.SpiffeGpuError):
        g.add_on_axis_field(fx["rf_z"][:4], fx["rf_Ez"][:4], Ez_peak=1e6, frequency=1e9, phase_rad=0.0)
    g.close()


@pytest.mark.parametrize("prec", [gpu.PRECISION_F64, gpu.PRECISION_SPLIT32])
def test_translate_problem_moves_rows(prec):
    """spiffe_gpu_translate_problem (translate.c:40-197): with a particle past
    the trigger the TM field and current rows move down one row, the top row
    is zeroed, zmin, zmax and the trigger grow by dz; without one nothing
    moves."""
    rng = np.random.default_rng(7)
    f = abi.Fields(41, 31, 0.0, 0.03, 0.02)
    for n in ("Ez", "Er", "Bphi", "Bphi2", "Jz", "Jr"):
        f[n] = rng.standard_normal(f.shape)
    g = gpu.GpuInstance(f, capacity=64, precision=prec)
    g.upload_fields(f)
    b = abi.Beam(16)
    b.set(1, z=[0.0251], r=[0.004], pz=[0.1], Q=[-1e-15], status=[1])
    b.npActive, b.nextParticleID, b.QoMC, b.stiffness = 1, 2, -5.866e2, 1.0
    g.upload_beam(b)
    dz = f.mesh.dz
    g.set_translation(1, 0.025)
    assert g.translate_problem() == (True, dz)
    m = g.get_mesh()
    assert m.zmin == dz and m.zmax == 0.03 + dz
    got = g.fields(f)
    for n in ("Ez", "Er", "Bphi", "Bphi2"):
        ref = f[n] if prec == gpu.PRECISION_F64 else f[n].astype(np.float32).astype(np.float64)
        assert np.array_equal(got[n][:-1], ref[1:]), n
        assert not got[n][-1].any(), n
    # the particle (z = 25.1 mm) is no longer past the trigger (25 mm + dz)
    assert g.translate_problem() == (False, dz)
    with pytest.raises(gpu.SpiffeGpuError):  # past zmax - dz of the moved mesh
        g.set_translation(1, 0.0301)
    g.close()
