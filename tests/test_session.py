"""The command session: spiffe input decks executed by libspiffe_b200.

CPU: namelist parsing and errors, define_geometry and define_solenoid against
the reference's own command processors (bit-exact), SDDS reading and
writing, load_fields (page choice, Ez_peak/factor scaling, overlay offset).
GPU: whole decks (define_geometry ... integrate) against the same decks run
by the reference's perform_integration (tests/golden/make_golden.py decks),
bit-exact in the FP64 form; field saving and reloading; multiple screens.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from spiffe_b200 import abi, gpu, session
from helpers import by_id, load, reference_file

ERR_INVALID, ERR_UNSUPPORTED = -1, -5


@pytest.fixture
def dcgeo(tmp_path, monkeypatch):
    """A working directory holding the DC gun boundary file dc.geo."""
    (tmp_path / "dc.geo").write_text(str(load("dcgun_geometry")["geo"]))
    monkeypatch.chdir(tmp_path)
    return tmp_path


GEOM = '&define_geometry nz=151, nr=101, zmin=0.0, zmax=0.03, rmax=0.02, boundary="dc.geo" &end\n'


def test_geometry_command_gives_the_reference_flags(dcgeo):
    fx = load("dcgun_geometry")
    with session.Session(verbose=0) as s:
        s.execute("! a comment line\n" + GEOM)
        m = s.mesh()
        f = s.fields()
    assert (m.nz, m.nr) == (151, 101) and m.dz == float(fx["dz"]) and m.dr == float(fx["dr"])
    assert [m.lower_bc, m.upper_bc, m.right_bc, m.left_bc] == list(fx["bcs"])
    assert m.modes == abi.FL_TM_FIELDS | abi.FL_RADIAL_INTERP | abi.FL_LONGIT_INTERP
    assert np.array_equal(f.flags, fx["flags"]) and np.array_equal(f["PsiImposed"], fx["PsiImposed"])


def test_geometry_switches(dcgeo):
    with session.Session(verbose=0) as s:
        s.execute('&define_geometry nz=41, nr=31, zmax=0.03, rmax=0.02, boundary="dc.geo", include_TE_fields=1, '
                  'radial_interpolation=0, longitudinal_smearing=1, turn_off_Bphi=1, right="dirichlet" &end')
        m = s.mesh()
        f = s.fields()
    assert m.modes == abi.FL_TM_FIELDS | abi.FL_TE_FIELDS | abi.FL_LONGIT_INTERP | abi.FL_LONGIT_SMEAR
    assert list(m.turn_off) == [0, 0, 0, 0, 0, 1] and m.right_bc == abi.DIRICHLET
    assert "Bz2" in f.a and "Ephi" in f.a


@pytest.mark.parametrize("text,code,msg", [
    ("&define_geometry nz=41, nr=31, zmax=0.03, rmax=0.02 &end", ERR_INVALID, "no boundary-points file"),
    ('&define_geometry nz=1, nr=31, zmax=0.03, rmax=0.02, boundary="dc.geo" &end', ERR_INVALID, "greater than 2"),
    ('&define_geometry nz=41, nr=31, zmax=0.03, rmax=0.02, boundary="dc.geo", lower="Neumann" &end', ERR_INVALID,
     "meaningless on the lower"),
    ('&define_geometry nz=41, nr=31, zmax=0.03, rmax=0.02, boundary="dc.geo", colour=3 &end', ERR_INVALID,
     "unknown variable colour"),
    ('&define_geometry nz=4x1, nr=31, zmax=0.03, rmax=0.02, boundary="dc.geo" &end', ERR_INVALID, "invalid value"),
    ("&define_cathode z_position=0, outer_radius=0.001, current_density=1e6 &end", ERR_INVALID, "before"),
    ("&frobnicate a=1 &end", ERR_INVALID, "unknown namelist frobnicate"),
    ("&space_charge &end", ERR_INVALID, "no longer used"),
    ("&define_emitter &end", ERR_INVALID, "must be non-zero"),
    ("&define_emitter current_density=1e6, electrons_per_macroparticle=1e6 &end", ERR_INVALID, "before"),
    ("&define_resistor &end", ERR_UNSUPPORTED, "not supported"),
])
def test_command_errors(dcgeo, text, code, msg):
    with session.Session(verbose=0) as s:
        with pytest.raises(gpu.SpiffeGpuError) as e:
            s.execute(text)
        assert f"error {code}" in str(e.value) and msg in str(e.value), str(e.value)


def test_checks_after_geometry(dcgeo):
    with session.Session(verbose=0) as s:
        s.execute(GEOM)
        for text, msg in [
            ("&define_cathode z_position=0.05, outer_radius=0.001, current_density=1e6 &end", "outside of simulation"),
            ("&define_cathode z_position=0, outer_radius=0.001 &end", "must be non-zero"),
            ("&define_cathode z_position=0, outer_radius=0.001, current_density=1e6, add_thermal_velocities=1, "
             "temperature=1000 &end", "not supported"),
            ("&define_screen z_position=0.01 &end", "no filename given"),
            ('&define_screen filename="a", z_position=0.01, direction="sideways" &end', "unknown screen direction"),
            ("&poisson_correction accuracy=0 &end", "accuracy <= 0"),
            ('&poisson_correction guess_type="psychic" &end', "unknown guess type"),
            ("&define_test_beam start_time=0, stop_time=1e-12, initial_z=0.001 &end", "electrons_per_macroparticle"),
            ("&define_emitter material_id=9, current_density=1e6, electrons_per_macroparticle=1e6 &end",
             "No surface elements"),
            ("&define_emitter material_id=9, current_density=1e6, electrons_per_macroparticle=1e6, "
             "add_thermal_velocities=1, temperature=1000 &end", "not supported"),
            ('&define_secondary_emission input_file="y.sdds" &end', "column containing energy values"),
            ("&integrate dt_integration=0 &end", "dt_integration <= 0"),
            ("&integrate dt_integration=1e-12, finish_time=1e-10 &end", "stable integration"),
            ("&integrate dt_integration=1e-13, finish_time=1e-11, smoothing_parameter=0.1 &end", "not supported"),
            ('&define_field_saving filename="f" &end', "Use one of"),
            ('&define_field_saving filename="f", z_Ez_trigger=0.01 &end', "not supported"),
            ('&load_fields filename="missing.sdds" &end', "unable to open"),
            ('&define_antenna start=0.001, end=0.002, position=0.001, frequency=1e9, waveform="none" &end',
             "unable to open"),
        ]:
            with pytest.raises(gpu.SpiffeGpuError) as e:
                s.execute(text)
            assert msg in str(e.value), (text, str(e.value))
        assert s.execute("&trace &end\n&define_snapshots filename=\"x\" &end\n&stop &end\n&frobnicate &end") == 1


def test_screens_open_their_files(dcgeo):
    """Every define_screen opens its SDDS file at once (screens.c:81-100), one
    file per screen of a template; the session owns each file until it ends."""
    with session.Session(verbose=0, rootname="run") as s:
        s.execute(GEOM + '&define_screen filename="%s.a", z_position=0.01 &end\n'
                  '&define_screen template="scr%02ld.sdds", z_position=0.005, delta_z=0.002, number_of_screens=4, '
                  'direction="backward" &end\n')
    for name in ["run.a"] + [f"scr{i:02d}.sdds" for i in range(4)]:
        assert session.read_sdds(str(dcgeo / name)) == []
    head = open(dcgeo / "scr03.sdds", "rb").read(4000).decode("latin-1")
    assert "backward" in head and "z=1.100000e-02 m" in head and "particleID" in head


def test_cathode_and_test_beam_exclude_each_other(dcgeo):
    with session.Session(verbose=0) as s:
        s.execute(GEOM + "&define_cathode z_position=0, outer_radius=0.001, current_density=1e6 &end")
        with pytest.raises(gpu.SpiffeGpuError, match="both cathode and test beam"):
            s.execute("&define_test_beam start_time=0, stop_time=1e-12, initial_z=0.001, "
                      "electrons_per_macroparticle=1 &end")


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libspiffe_ref.so")), reason="reference not built")
def test_solenoid_matches_reference(dcgeo):
    """define_solenoid through the session and through the reference's own
    process_solenoid_definition: ring coils, symmetry, the evaluation radius
    limit, Bz_peak scaling and a bucking coil, bit for bit."""
    from oracle import pyoracle

    cmds = [GEOM.strip(),
            "&define_solenoid radius=0.05, z_start=0.01, z_end=0.03, turns=5, current=1000, "
            "evaluation_radius_limit=0.013 &end",
            "&define_solenoid radius=0.03, z_start=0.004, z_end=0.005, turns=3, current=-200, symmetry=1, "
            "Bz_peak=0.2 &end",
            "&define_solenoid radius=0.02, z_start=0.02, z_end=0.026, turns=2, current=50, symmetry=-1 &end",
            "&define_solenoid radius=0.02, z_start=0.025, z_end=0.025, bucking=1, z_buck=0.02 &end"]
    with session.Session(verbose=0) as s:
        s.execute("\n".join(cmds))
        f = s.fields()
        assert s.mesh().has_solenoid == 1
    bz, br = pyoracle.run_reference([("command", c) for c in cmds] + [("get_field", "BzImposed"),
                                                                       ("get_field", "BrImposed")], cwd=str(dcgeo))
    assert np.array_equal(f["BzImposed"], bz) and np.array_equal(f["BrImposed"], br)
    assert np.abs(bz).max() > 0.1


def test_solenoid_function_on_abi_fields():
    f = abi.Fields(60, 40, 0.0, 0.1, 0.05)
    cur = session.solenoid_field(f, radius=0.04, z_start=0.03, z_end=0.07, current=100.0, turns=20)
    assert cur == 100.0 and f.mesh.has_solenoid == 1
    bz = f["BzImposed"][:, 0]
    # on axis the field peaks at the coil centre; mu0 n I for a long coil is the upper bound
    iz = int(np.argmax(bz))
    assert abs((iz * f.mesh.dz) - 0.05) <= f.mesh.dz
    assert 0 < bz.max() < 4e-7 * np.pi * 20 / 0.04 * 100
    assert np.all(f["BrImposed"][:, 0] == 0)


def test_sdds_ascii_tables(dcgeo):
    # the layout of the reference's antenna waveform files (a header, then
    # rows with no row count); the antenna and cathode profile read them
    with open("wave.wf", "w") as fh:
        fh.write("SDDS1\n&column name=t type=double &end\n&column name=W type=double &end\n"
                 "&data mode=ascii no_row_counts=1 &end\n")
        for k in range(5):
            fh.write("%e\t%e\n" % (k * 7e-12, (k / 4.0) ** 2))
    session.write_sdds_ascii("bad.wf", {"t": [0.0, 2e-12, 1e-12], "W": [0, 1, 1]})
    session.write_sdds_ascii("short.wf", {"t": [0.0, 1e-12], "W": [0, 1]})
    session.write_sdds_ascii("prof.sdds", {"tt": [0.0, 1e-12, 2e-12], "A": [0.0, 1.0, 0.0]})
    pages = session.read_sdds("wave.wf")
    assert len(pages) == 1 and np.allclose(pages[0]["columns"]["W"], [0, 1 / 16, 0.25, 9 / 16, 1])
    with session.Session(verbose=0) as s:
        s.execute(GEOM)
        s.execute('&define_antenna start=0.005, end=0.006, position=0.001, direction="z", current=2, '
                  'frequency=2.856e9, waveform="wave.wf", time_offset=1e-12 &end')
        with pytest.raises(gpu.SpiffeGpuError, match="not ordered"):
            s.execute('&define_antenna start=0.005, end=0.006, frequency=1e9, waveform="bad.wf" &end')
        with pytest.raises(gpu.SpiffeGpuError, match="empty or invalid"):
            s.execute('&define_antenna start=0.005, end=0.006, frequency=1e9, waveform="short.wf" &end')
        with pytest.raises(gpu.SpiffeGpuError, match="start or end out of range"):
            s.execute('&define_antenna start=0.005, end=0.05, frequency=1e9, waveform="wave.wf" &end')
        s.execute('&define_cathode z_position=0, outer_radius=0.001, current_density=1e6, profile="prof.sdds", '
                  'profile_time_name="tt", profile_factor_name="A" &end')
        with pytest.raises(gpu.SpiffeGpuError, match="no column"):
            s.execute('&define_cathode z_position=0, outer_radius=0.001, current_density=1e6, '
                      'profile="prof.sdds", profile_time_name="t", profile_factor_name="A" &end')


REF_WF = reference_file("examples", "apsTCRFGun", "excite", "spline4.wf")


@pytest.mark.skipif(REF_WF is None or not os.path.exists(REF_WF), reason="reference examples not present")
def test_reference_waveform_file_is_read(dcgeo):
    pages = session.read_sdds(REF_WF)
    t = pages[0]["columns"]["t"]
    assert len(t) > 10 and np.all(np.diff(t) > 0)
    with session.Session(verbose=0) as s:
        s.execute(GEOM + f'&define_antenna start=0.005, end=0.006, frequency=2.856e9, waveform="{REF_WF}" &end')


def field_file_problem(nz=40, nr=30, zmin=0.0, zmax=0.03, rmax=0.02, seed=0):
    rng = np.random.default_rng(seed)
    f = abi.Fields(nz, nr, zmin, zmax, rmax)
    for n in ("Ez", "Er", "Jz", "Jr", "Bphi", "Bphi2"):
        f[n] = rng.normal(size=f.shape)
    return f


def test_load_fields_page_scaling_and_overlay(dcgeo):
    """perform_field_loading: the first page at or after time_threshold, Ez_peak
    or factor scaling, and the sum into the problem's fields, shifted by the
    whole cells between the meshes' zmin."""
    geo = dcgeo / "box.geo"
    geo.write_text("&po x=0.0, y=0.0 &end\n&po x=0.0, y=0.02 &end\n&po x=0.03, y=0.02 &end\n"
                   "&po x=0.03, y=0.0 &end\n&po x=0.0, y=0.0 &end\n")
    src = field_file_problem()
    session.write_field_save("f.sdds", src, [1e-9, 2e-9, 3e-9])
    pages = session.read_sdds("f.sdds")
    assert len(pages) == 3 and pages[1]["parameters"]["time"] == 2e-9
    assert np.array_equal(pages[0]["columns"]["Ez"], src["Ez"].ravel())
    g = '&define_geometry nz=40, nr=30, zmin=0.0, zmax=0.03, rmax=0.02, boundary="box.geo" &end\n'
    with session.Session(verbose=0) as s:
        s.execute(g + '&load_fields filename="f.sdds", factor=3, time_threshold=1.5e-9 &end\n'
                  '&load_fields filename="f.sdds", factor=-1 &end')
        f = s.fields()
    for n in ("Ez", "Er", "Jz", "Jr", "Bphi", "Bphi2"):
        assert np.allclose(f[n], 2 * src[n], rtol=0, atol=1e-12), n
    # Ez_peak: the on-axis extremum of rows 1..nz scaled to Ez_peak
    ez_axis = src["Ez"][1:, 0]
    ext = ez_axis[np.argmax(np.abs(ez_axis))]
    with session.Session(verbose=0) as s:
        s.execute(g + '&load_fields filename="f.sdds", Ez_peak=5e7 &end')
        f = s.fields()
    assert np.array_equal(f["Er"], src["Er"] * (5e7 / ext))
    assert abs(np.abs(f["Ez"][1:, 0]).max() - 5e7) < 1e-6
    # a problem whose zmin is 7 cells further along: rows shift by 7
    dz = 0.03 / 39
    g2 = (f'&define_geometry nz=30, nr=30, zmin={7 * dz!r}, zmax={7 * dz + 29 * dz!r}, rmax=0.02, '
          'boundary="box2.geo" &end\n')
    (dcgeo / "box2.geo").write_text(f"&po x={7 * dz!r}, y=0.0 &end\n&po x={7 * dz!r}, y=0.02 &end\n"
                                    f"&po x={36 * dz!r}, y=0.02 &end\n&po x={36 * dz!r}, y=0.0 &end\n"
                                    f"&po x={7 * dz!r}, y=0.0 &end\n")
    with session.Session(verbose=0) as s:
        s.execute(g2 + '&load_fields filename="f.sdds" &end')
        f = s.fields()
    assert np.array_equal(f["Bphi"], src["Bphi"][7:38])
    with session.Session(verbose=0) as s:
        with pytest.raises(gpu.SpiffeGpuError, match="unable to get data"):
            s.execute(g + '&load_fields filename="f.sdds", time_threshold=1e-8 &end')


def test_cli_reports_errors_without_a_gpu(dcgeo):
    (dcgeo / "deck.spiffe").write_text(GEOM + "&define_frobnicator &end\n")
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PYTHONPATH=repo)
    p = subprocess.run([sys.executable, "-m", "spiffe_b200.session", "deck.spiffe", "--quiet"], capture_output=True,
                       text=True, env=env, timeout=300)
    assert p.returncode == 1 and "unknown namelist define_frobnicator" in p.stderr


# ------------------------------------------------------------------ GPU decks

def run_deck(fx, tmp_path, monkeypatch, precision="f64", extra="", **settings):
    (tmp_path / "dc.geo").write_text(str(fx["geo"]))
    monkeypatch.chdir(tmp_path)
    s = session.Session(precision, verbose=0, **settings)
    deck = str(fx["deck"])
    if extra:
        i = deck.index("&integrate")
        deck = deck[:i] + extra + deck[i:]
    s.execute(deck)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["deck_dcgun", "deck_testbeam"])
def test_deck_matches_reference_bit_for_bit(name, tmp_path, monkeypatch):
    """The whole deck (geometry, solenoid, constant fields, cathode or test
    beam, screen, Poisson correction, integrate) in the FP64 form against the
    reference's perform_integration on the same deck."""
    fx = load(name)
    s = run_deck(fx, tmp_path, monkeypatch)
    m = s.mesh()
    assert m.time == float(fx["time"])
    f = s.fields()
    for n in ("Ez", "Er", "Bphi", "Psi"):
        assert np.array_equal(f[n], fx[n]), n
    g = s.instance()
    b = g.download_beam(abi.Beam(max(int(fx["out_np"]), 1) + 16))
    assert b.np == int(fx["out_np"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(b[k][: b.np], fx["out_" + k]), k
    # the screen's SDDS file holds every crossing the reference recorded
    pages = session.read_sdds(str(tmp_path / ("deck.sc1" if name == "deck_dcgun" else "tb.sc1")))
    rec = {c: np.concatenate([p["columns"][c] for p in pages]) for c in abi.SCREEN_COLUMNS + ["particleID"]}
    ref = {c: fx["screen0_" + c] for c in abi.SCREEN_COLUMNS + ["particleID"]}
    assert len(rec["r"]) == len(ref["r"]) > 0
    if name == "deck_dcgun":
        rec, ref = by_id(rec), by_id(ref)
    else:  # test particles carry ID 0: order by crossing time
        o1, o2 = np.argsort(rec["t"], kind="stable"), np.argsort(ref["t"], kind="stable")
        rec, ref = {k: v[o1] for k, v in rec.items()}, {k: v[o2] for k, v in ref.items()}
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rec[c], ref[c]), c
    assert all(p["parameters"]["direction"] == "forward" for p in pages)
    s.close()


@pytest.mark.gpu
def test_split_form_runs_the_deck(tmp_path, monkeypatch):
    """The split-precision form on the same deck, against the FP64 form with
    the same loss handling (the reference's compaction ends the beam at the
    first lost particle, advance_particles.c:491-518; the split form removes
    exactly the lost ones).  The bar is the one for the split form's results:
    exit-screen moments within 0.5 %.  The fields agree to 1 % relative L2:
    this deck's Poisson corrections stop at accuracy 1e-4, so each correction
    may differ between the forms at that level."""
    from spiffe_b200 import moments

    fx = load("deck_dcgun")
    out = {}
    for prec, d in (("f64", "a"), ("split32", "b")):
        (tmp_path / d).mkdir()
        s = run_deck(fx, tmp_path / d, monkeypatch, precision=prec, compaction=abi.COMPACT_SWAP,
                     screen_momentum=abi.SCREEN_PARTICLE)
        f = s.fields()
        pages = session.read_sdds(str(tmp_path / d / "deck.sc1"))
        rec = {c: np.concatenate([p["columns"][c] for p in pages]) for c in abi.SCREEN_COLUMNS}
        out[prec] = (f, rec)
        s.close()
    (f64, r64), (f32, r32) = out["f64"], out["split32"]
    m64, m32 = moments.exit_moments(r64), moments.exit_moments(r32)
    assert m64["count"] > 900 and abs(m32["count"] - m64["count"]) <= 0.005 * m64["count"], (m32, m64)
    errs = moments.relative_errors(m32, m64)
    assert max(errs.values()) < 5e-3, errs
    for n in ("Ez", "Er"):
        err = np.sqrt(np.sum((f32[n] - f64[n]) ** 2) / np.sum(f64[n] ** 2))
        assert err < 1e-2, (n, err)


@pytest.mark.gpu
def test_field_saving_and_reload(tmp_path, monkeypatch):
    """define_field_saving writes the fields at its schedule; load_fields of
    the last page into a fresh problem reproduces them (times factor)."""
    fx = load("deck_dcgun")
    s = run_deck(fx, tmp_path, monkeypatch, extra='&define_field_saving filename="%s.fsave", time_interval=100e-12, '
                                                 'start_time=50e-12, save_before_exiting=1 &end\n',
                 flush_steps=64)
    f = s.fields()
    s.close()
    pages = session.read_sdds(str(tmp_path / "spiffe.fsave"))
    times = [p["parameters"]["time"] for p in pages]
    # steps 125, 375, 625 by the schedule (interval 250 steps from step 125), then the final save at 750
    assert np.allclose(times, [125 * 4e-13, 375 * 4e-13, 625 * 4e-13, 750 * 4e-13], rtol=1e-12)
    last = pages[-1]["columns"]
    for n in ("Ez", "Er", "Bphi"):
        assert np.array_equal(last[n], f[n].ravel()), n
    assert pages[0]["parameters"]["TMfields"] == "y" and int(pages[0]["parameters"]["nz"]) == 151
    with session.Session(verbose=0) as s2:
        s2.execute(str(fx["deck"]).split("&define_solenoid")[0] +
                   '&load_fields filename="spiffe.fsave", time_threshold=2.9e-10, factor=2 &end')
        g = s2.fields()
    for n in ("Ez", "Er", "Bphi"):
        assert np.array_equal(g[n], 2 * f[n]), n


@pytest.mark.gpu
def test_two_screens_record_crossings(tmp_path, monkeypatch):
    """Every screen records (the reference writes the second screen's records
    through a null buffer); both screens see the bunch, the far one later."""
    fx = load("deck_dcgun")
    s = run_deck(fx, tmp_path, monkeypatch, extra='&define_screen filename="far.sc", z_position=0.016 &end\n')
    s.close()
    near = session.read_sdds(str(tmp_path / "deck.sc1"))
    far = session.read_sdds(str(tmp_path / "far.sc"))
    tn = np.concatenate([p["columns"]["t"] for p in near])
    tf = np.concatenate([p["columns"]["t"] for p in far])
    assert len(tn) == len(fx["screen0_r"]) and len(tf) > 0
    assert np.median(tf) > np.median(tn)
    steps = [p["parameters"]["Timestep"] for p in far]
    assert steps == sorted(steps)


@pytest.mark.gpu
def test_snapshots_and_field_output_match_reference(tmp_path, monkeypatch):
    """define_snapshots and define_field_output through the session against the
    reference's own take_beam_snapshot and output_fields on the same deck:
    every row of every page, bit for bit (the charge density within single
    precision rounding: the FP64 form removes the particles' charge from Q
    with atomics)."""
    from golden_columns import FLD_COLUMNS, SNAP_COLUMNS

    fx = load("deck_diagnostics")
    s = run_deck(fx, tmp_path, monkeypatch)
    s.close()
    snap = session.read_sdds(str(tmp_path / "spiffe.snap"))
    fld = session.read_sdds(str(tmp_path / "spiffe.fld"))
    assert len(snap) == int(fx["snap_pages"]) == 3 and len(fld) == int(fx["fld_pages"]) == 3
    assert [p["parameters"]["Timestep"] for p in snap] == [50, 150, 250]
    for c in SNAP_COLUMNS:
        got = np.concatenate([p["columns"][c] for p in snap]).astype(np.float64)
        assert np.array_equal(got, fx["snap_" + c]), c
    for c in FLD_COLUMNS:
        got = np.concatenate([p["columns"][c] for p in fld]).astype(np.float64)
        if c == "rho":
            assert np.allclose(got, fx["fld_" + c], rtol=2e-7, atol=0), c
        else:
            assert np.array_equal(got, fx["fld_" + c]), c
    p0 = fld[0]["parameters"]
    assert p0["Variable1Name"] == "z" and p0["zDimension"] == 76 and p0["rDimension"] == 26


def write_rf(path, z, Ez):
    """The on-axis field table as tests/golden/make_golden.py writes it."""
    with open(path, "w") as f:
        f.write("SDDS1\n&column name=z type=double units=m &end\n&column name=Ez type=double &end\n"
                "&data mode=ascii no_row_counts=1 &end\n")
        for a, b in zip(z, Ez):
            f.write("%.17g %.17g\n" % (a, b))


def test_on_axis_profile_output_matches_reference(dcgeo):
    """add_on_axis_fields' fields_used table (the expansion near the axis with
    sine and cosine 1, onAxisFields.c:130-170) against the reference's, bit
    for bit: this checks the scaling, the three derivatives and the
    expansion's arithmetic on the host."""
    fx = load("deck_onaxis")
    write_rf(dcgeo / "rf.sdds", fx["rf_z"], fx["rf_Ez"])
    deck = str(fx["deck"])
    cmds = [b.strip() + " &end" for b in deck.split("&end") if b.strip()]
    with session.Session(verbose=0, rootname="run") as s:
        s.execute("\n".join(c for c in cmds if c.startswith(("&define_geometry", "&add_on_axis_fields"))))
    pages = session.read_sdds(str(dcgeo / "run.oaf"))
    assert len(pages) == 1
    for c in ("z", "Ez", "Er/r", "Bphi/r"):
        got = pages[0]["columns"][c]
        assert len(got) == 151 and np.array_equal(got, fx["oaf_" + c.replace("/", "_")]), c


@pytest.mark.parametrize("change,msg", [
    ("expansion_order=4", "expansion_order must by on [0, 3]"),
    ("frequency=-1", "frequency is negative"),
    ("rows=4", "Too few points"),
    ("reverse", "not monotonically increasing"),
    ("uneven", "not equispaced"),
])
def test_on_axis_errors(dcgeo, change, msg):
    z, Ez = np.linspace(0, 0.02, 41), np.sin(np.linspace(0, np.pi, 41))
    extra = ""
    if change == "rows=4":
        z, Ez = z[:4], Ez[:4]
    elif change == "reverse":
        z = z[::-1].copy()
    elif change == "uneven":
        z = z.copy()
        z[20] += 1e-5
    else:
        extra = ", " + change
    write_rf(dcgeo / "rf.sdds", z, Ez)
    with session.Session(verbose=0) as s:
        with pytest.raises(gpu.SpiffeGpuError) as e:
            s.execute(GEOM + '&add_on_axis_fields filename="rf.sdds", z_name="z", Ez_name="Ez", Ez_peak=1e6, '
                      f'frequency=1e9{extra} &end\n')
        assert msg in str(e.value), str(e.value)
    # Ez_peak = 0 ignores the definition (onAxisFields.c:45-49)
    write_rf(dcgeo / "rf.sdds", np.linspace(0, 0.02, 41), np.ones(41))
    with session.Session(verbose=0) as s:
        s.execute(GEOM + '&add_on_axis_fields filename="rf.sdds", z_name="z", Ez_name="Ez", Ez_peak=0 &end\n')


@pytest.mark.gpu
def test_on_axis_deck_matches_reference_bit_for_bit(tmp_path, monkeypatch):
    """The DC gun with an RF on-axis field (add_on_axis_fields) and a
    Richardson-Schottky cathode, in the FP64 form, against the reference's
    perform_integration on the same deck: the push adds the third-order
    off-axis expansion to every particle's fields, the cathode's current
    density reads it at the cathode each step."""
    fx = load("deck_onaxis")
    write_rf(tmp_path / "rf.sdds", fx["rf_z"], fx["rf_Ez"])
    s = run_deck(fx, tmp_path, monkeypatch)
    assert s.mesh().time == float(fx["time"])
    f = s.fields()
    for n in ("Ez", "Er", "Bphi", "Psi"):
        assert np.array_equal(f[n], fx[n]), n
    g = s.instance()
    b = g.download_beam(abi.Beam(int(fx["out_np"]) + 16))
    assert b.np == int(fx["out_np"]) > 2000
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(b[k][: b.np], fx["out_" + k]), k
    pages = session.read_sdds(str(tmp_path / "oa.sc1"))
    rec = by_id({c: np.concatenate([p["columns"][c] for p in pages]) for c in abi.SCREEN_COLUMNS + ["particleID"]})
    ref = by_id({c: fx["screen0_" + c] for c in abi.SCREEN_COLUMNS + ["particleID"]})
    assert len(rec["r"]) == len(ref["r"]) > 2000
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rec[c], ref[c]), c
    s.close()


@pytest.mark.gpu
def test_split_form_runs_the_on_axis_deck(tmp_path, monkeypatch):
    """The split-precision form on the on-axis deck against the FP64 form:
    exit-screen moments within 0.5 %, the beam's count within 0.5 %.  Both
    solve the deck's Poisson corrections with the reference's SOR: at the
    deck's accuracy of 1e-4 two solutions that meet the stop rule move the
    emittance by 0.7 % (the multigrid's does, against the SOR's)."""
    from spiffe_b200 import moments

    fx = load("deck_onaxis")
    out = {}
    for prec, d in (("f64", "a"), ("split32", "b")):
        (tmp_path / d).mkdir()
        write_rf(tmp_path / d / "rf.sdds", fx["rf_z"], fx["rf_Ez"])
        extra = {"poisson_solver": gpu.POISSON_SOR} if prec == "split32" else {}
        s = run_deck(fx, tmp_path / d, monkeypatch, precision=prec, compaction=abi.COMPACT_SWAP,
                     screen_momentum=abi.SCREEN_PARTICLE, **extra)
        pages = session.read_sdds(str(tmp_path / d / "oa.sc1"))
        out[prec] = {c: np.concatenate([p["columns"][c] for p in pages]) for c in abi.SCREEN_COLUMNS}
        s.close()
    m64, m32 = moments.exit_moments(out["f64"]), moments.exit_moments(out["split32"])
    assert m64["count"] > 2000 and abs(m32["count"] - m64["count"]) <= 0.005 * m64["count"], (m32, m64)
    errs = moments.relative_errors(m32, m64)
    assert max(errs.values()) < 5e-3, errs


def test_translate_checks(dcgeo):
    """translate's range check (translate.c:35-36); the region reduction of
    z_lower/z_upper is refused."""
    with session.Session(verbose=0) as s:
        with pytest.raises(gpu.SpiffeGpuError) as e:
            s.execute(GEOM + "&translate z_trigger=0.0299 &end\n")
        assert "z_trigger is not in range" in str(e.value)
    with session.Session(verbose=0) as s:
        with pytest.raises(gpu.SpiffeGpuError) as e:
            s.execute(GEOM + "&translate z_trigger=0.01, z_lower=0.005 &end\n")
        assert f"error {ERR_UNSUPPORTED}" in str(e.value) and "z_lower" in str(e.value)
    with session.Session(verbose=0) as s:
        s.execute(GEOM + "&translate &end\n")  # default trigger zmax - 5 dz


@pytest.mark.gpu
def test_translate_deck_matches_reference_bit_for_bit(tmp_path, monkeypatch):
    """The DC gun deck with the moving window (translate) in the FP64 form
    against the reference on the same deck: 316 translations, then the same
    mesh position, fields, beam and screen records."""
    fx = load("deck_translate")
    s = run_deck(fx, tmp_path, monkeypatch)
    m = s.mesh()
    assert m.time == float(fx["time"]) and m.zmin == float(fx["zmin"]) and m.zmax == float(fx["zmax"])
    assert m.zmin > 0.06
    f = s.fields()
    for n in ("Ez", "Er", "Bphi", "Psi"):
        assert np.array_equal(f[n], fx[n]), n
    b = s.instance().download_beam(abi.Beam(int(fx["out_np"]) + 16))
    assert b.np == int(fx["out_np"]) > 800
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(b[k][: b.np], fx["out_" + k]), k
    pages = session.read_sdds(str(tmp_path / "deck.sc1"))
    rec = by_id({c: np.concatenate([p["columns"][c] for p in pages]) for c in abi.SCREEN_COLUMNS + ["particleID"]})
    ref = by_id({c: fx["screen0_" + c] for c in abi.SCREEN_COLUMNS + ["particleID"]})
    assert len(rec["r"]) == len(ref["r"]) > 900
    for c in abi.SCREEN_COLUMNS:
        assert np.array_equal(rec[c], ref[c]), c
    s.close()


@pytest.mark.gpu
def test_split_form_runs_the_translate_deck(tmp_path, monkeypatch):
    """The split form (positions stored relative to the moving mesh) on the
    moving-window deck against the FP64 form: the same number of
    translations, exit moments within 0.5 %."""
    from spiffe_b200 import moments

    fx = load("deck_translate")
    out, zmin = {}, {}
    for prec, d in (("f64", "a"), ("split32", "b")):
        (tmp_path / d).mkdir()
        s = run_deck(fx, tmp_path / d, monkeypatch, precision=prec, compaction=abi.COMPACT_SWAP,
                     screen_momentum=abi.SCREEN_PARTICLE)
        zmin[prec] = s.mesh().zmin
        pages = session.read_sdds(str(tmp_path / d / "deck.sc1"))
        out[prec] = {c: np.concatenate([p["columns"][c] for p in pages]) for c in abi.SCREEN_COLUMNS}
        s.close()
    assert zmin["split32"] == zmin["f64"] > 0.06
    m64, m32 = moments.exit_moments(out["f64"]), moments.exit_moments(out["split32"])
    assert m64["count"] > 900 and abs(m32["count"] - m64["count"]) <= 0.005 * m64["count"], (m32, m64)
    errs = moments.relative_errors(m32, m64)
    assert max(errs.values()) < 5e-3, errs


@pytest.mark.gpu
def test_status_file_matches_reference(tmp_path, monkeypatch):
    """integrate's status_output (do_status_printouts, status_pr.c) on the
    on-axis deck in the FP64 form against the reference's status file: every
    column of every row identical (energies, charge, beam moments and
    extremes, the Schottky cathode's current density, the on-axis Ez
    extremes of the last push)."""
    from golden_columns import STATUS_COLUMNS

    fx = load("deck_status")
    write_rf(tmp_path / "rf.sdds", fx["rf_z"], fx["rf_Ez"])
    s = run_deck(fx, tmp_path, monkeypatch)
    s.close()
    pages = session.read_sdds(str(tmp_path / "spiffe.status"))
    assert len(pages) == 1 and int(fx["rows"]) == 8
    for c in STATUS_COLUMNS:
        got = np.asarray(pages[0]["columns"][c], np.float64)
        assert len(got) == 8 and np.array_equal(got, fx["st_" + c]), (c, got, fx["st_" + c])


LOST_COLUMNS = ["t", "rLost", "zLost", "pz", "pr", "z0", "r0", "q", "generation", "particleID"]


@pytest.mark.gpu
def test_lost_particle_file_matches_reference(tmp_path, monkeypatch):
    """integrate's lost_particles file (advance_particles.c:437-487, 577-603)
    on a DC gun deck whose cathode is wider than the anode hole: in the FP64
    form the rows (time, the loss point of findLossCoordinates,
    secondaryEmission.c:239, momenta, birth position, charge, generation, id)
    and the page breaks equal the reference's."""
    fx = load("deck_lost")
    s = run_deck(fx, tmp_path, monkeypatch)
    pages = session.read_sdds(str(tmp_path / "spiffe.lost"))
    got = {c: np.concatenate([p["columns"][c] for p in pages]) for c in LOST_COLUMNS}
    assert len(pages) == int(fx["lost_pages"])
    assert len(got["t"]) == len(fx["lost_t"]) > 40
    for c in LOST_COLUMNS:
        assert np.array_equal(np.asarray(got[c], np.float64), fx["lost_" + c]), c
    s.close()


@pytest.mark.gpu
def test_lost_particle_file_split_form(tmp_path, monkeypatch):
    """The split form writes the same file: the same particles lost, on the
    same step (or the next, one dt of 4e-13 s, for a few whose FP32 path
    crosses a face a step apart), with loss points within 1e-5 of a cell of
    the reference's, except for at most 5% that reach the anode's corner and
    leave through the other face (within a cell).  The corrections use the
    reference's SOR, as the comparison is of the split form's rounding."""
    fx = load("deck_lost")
    s = run_deck(fx, tmp_path, monkeypatch, precision="split32", poisson_solver=gpu.POISSON_SOR)
    pages = session.read_sdds(str(tmp_path / "spiffe.lost"))
    got = by_id({c: np.concatenate([p["columns"][c] for p in pages]) for c in LOST_COLUMNS}, "particleID")
    ref = by_id({c: fx["lost_" + c] for c in LOST_COLUMNS}, "particleID")
    # the reference ends the beam at its first lost index; the split form
    # removes only the lost particles, so it may lose more of them later
    common, ig, ir = np.intersect1d(got["particleID"], ref["particleID"], return_indices=True)
    assert len(common) == len(ref["particleID"])
    # the same step, or a neighbour where FP32 rounding moves a particle across a cell face
    assert np.max(np.abs(got["t"][ig] - ref["t"][ir])) <= 4.1e-13
    same = got["t"][ig] == ref["t"][ir]
    assert same.mean() > 0.9
    ig, ir = ig[same], ir[same]
    dz = 0.03 / 150
    # a particle that reaches the anode's corner may be lost on the other face
    # in one form (its loss point then moves by up to a cell); all others agree
    dzl = np.abs(got["zLost"][ig] - ref["zLost"][ir])
    drl = np.abs(got["rLost"][ig] - ref["rLost"][ir])
    close = (dzl <= 1e-5 * dz + 1e-9) & (drl <= 1e-5 * dz + 1e-9)
    assert close.mean() >= 0.95, (close.mean(), dzl.max(), drl.max())
    assert max(dzl.max(), drl.max()) <= dz
    s.close()


def write_yield(tmp_path, fx):
    with open(tmp_path / "yield.sdds", "w") as f:
        f.write("SDDS1\n&column name=K type=double units=eV &end\n&column name=Y type=double &end\n"
                "&data mode=ascii no_row_counts=1 &end\n")
        for a, b in zip(fx["yield_K"], fx["yield_Y"]):
            f.write("%.17g %.17g\n" % (a, b))


@pytest.mark.gpu
def test_secondary_emission_matches_reference(tmp_path, monkeypatch):
    """define_secondary_emission (secondaryEmission.c) on the lost-particle
    deck with the anode drawn as material 1: primaries that hit it release
    secondaries (a Poisson number from the yield table, random directions
    away from the face) that fall back and release more.  In the FP64 form
    the lost-particle file (every generation), the final beam and the screen
    equal the reference's bit for bit, so the queue, the yield draw, the
    directions and the shared random stream all follow the reference, and
    the emission log (log_file, which takes particle IDs) does too."""
    fx = load("deck_secondary")
    write_yield(tmp_path, fx)
    s = run_deck(fx, tmp_path, monkeypatch)
    pages = session.read_sdds(str(tmp_path / "spiffe.lost"))
    got = {c: np.concatenate([p["columns"][c] for p in pages]) for c in LOST_COLUMNS}
    assert len(pages) == int(fx["lost_pages"])
    assert len(got["t"]) == len(fx["lost_t"])
    assert np.max(fx["lost_generation"]) >= 3
    for c in LOST_COLUMNS:
        assert np.array_equal(np.asarray(got[c], np.float64), fx["lost_" + c]), c
    g = s.instance()
    b = g.download_beam(abi.Beam(max(int(fx["out_np"]), 1) + 16))
    assert b.np == int(fx["out_np"])
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(b[k][: b.np], fx["out_" + k]), k
    # the log_file: a page per emitting step, a row per emitting source
    log = session.read_sdds(str(tmp_path / "spiffe.sel"))
    assert len(log) == int(fx["log_pages"])
    for c in ("z", "r", "t", "K", "yield", "emitted", "directionCode", "generation"):
        v = np.concatenate([np.asarray(p["columns"][c], np.float64) for p in log])
        assert np.array_equal(v, fx["log_" + c]), c
    s.close()


@pytest.mark.gpu
def test_secondary_emission_split_form(tmp_path, monkeypatch):
    """The same deck in the split form: the primaries hit the anode on the
    reference's step and release secondaries of generation 1 and higher,
    which are lost on the anode face (z = 10 mm) in turn."""
    fx = load("deck_secondary")
    write_yield(tmp_path, fx)
    s = run_deck(fx, tmp_path, monkeypatch, precision="split32")
    pages = session.read_sdds(str(tmp_path / "spiffe.lost"))
    got = {c: np.concatenate([p["columns"][c] for p in pages]) for c in LOST_COLUMNS}
    gen = np.asarray(got["generation"])
    prim = gen == 0
    ref_prim = fx["lost_generation"] == 0
    assert prim.sum() >= ref_prim.sum()
    assert abs(np.min(got["t"][prim]) - np.min(fx["lost_t"][ref_prim])) <= 4.1e-13
    sec = ~prim
    assert sec.sum() >= 0.5 * (~ref_prim).sum() and gen.max() >= 2
    on_anode = np.abs(got["zLost"][sec] - 0.01) < 1e-6
    assert on_anode.mean() > 0.9
    # secondary IDs are new, and each generation is lost after the one before it
    assert not np.intersect1d(got["particleID"][sec], got["particleID"][prim]).size
    for k in range(1, int(gen.max()) + 1):
        assert got["t"][gen == k].min() > got["t"][gen == k - 1].min()
    s.close()


def write_emitter_inputs(tmp_path, fx):
    with open(tmp_path / "prof.sdds", "w") as f:
        f.write("SDDS1\n&column name=t type=double &end\n&column name=A type=double &end\n"
                "&data mode=ascii no_row_counts=1 &end\n")
        for a, b in zip(fx["prof_t"], fx["prof_A"]):
            f.write("%.17g %.17g\n" % (a, b))


@pytest.mark.gpu
def test_emitters_match_reference(tmp_path, monkeypatch):
    """define_emitter (emitter.c) on the DC gun with the cathode plane split
    into two materials: a thermionic emitter with a time profile and a
    field emitter, each emitting from the segments of its surface
    (getBoundaryPoints) with random_2 positions.  In the FP64 form the fields,
    the beam (IDs in emission order) and the screen equal the reference's bit
    for bit."""
    fx = load("deck_emitter")
    write_emitter_inputs(tmp_path, fx)
    s = run_deck(fx, tmp_path, monkeypatch)
    assert s.mesh().time == float(fx["time"])
    f = s.fields()
    for n in ("Ez", "Er", "Bphi", "Psi"):
        assert np.array_equal(f[n], fx[n]), n
    g = s.instance()
    b = g.download_beam(abi.Beam(int(fx["out_np"]) + 16))
    assert b.np == int(fx["out_np"]) > 500
    for k in abi.BEAM_DOUBLES + ["particleID", "status"]:
        assert np.array_equal(b[k][: b.np], fx["out_" + k]), k
    s.close()


@pytest.mark.gpu
def test_emitters_split_form(tmp_path, monkeypatch):
    """The same deck in the split form: the same emission (counts, birth
    points and times come from the host in FP64 with the same draws while the
    field-dependent current densities see FP32 fields), so the particle count
    is within 2% of the reference's and every particle was born on the
    emitter surface within the reference's birth-time window."""
    fx = load("deck_emitter")
    write_emitter_inputs(tmp_path, fx)
    s = run_deck(fx, tmp_path, monkeypatch, precision="split32")
    g = s.instance()
    b = g.download_beam(abi.Beam(2 * int(fx["out_np"]) + 16))
    n_ref = int(fx["out_np"])
    assert abs(b.np - n_ref) <= 0.02 * n_ref
    np_ = b.np
    assert np.all(b["z0"][:np_] == fx["out_z0"][0])
    assert b["r0"][:np_].min() >= 0.0002 - 1e-12 and b["r0"][:np_].max() <= 0.002 + 1e-12
    assert b["t0"][:np_].min() == fx["out_t0"].min() and b["t0"][:np_].max() <= fx["out_t0"].max() + 4.1e-13
    s.close()


SAMPLING_PAGES = [("ez", ["z", "Ez"]), ("e", ["r", "Ez", "Er", "Ephi"]), ("br", ["z", "Br"]), ("phi", ["r", "Phi"]),
                  ("q", ["z", "Q"]), ("jz", ["z", "Jz"]), ("jr", ["r", "Jr"])]
SAMPLING_SEQ = [("ezt", ["t", "Ez"]), ("ert", ["t", "Er"])]


@pytest.mark.gpu
def test_field_sampling_matches_reference(tmp_path, monkeypatch):
    """define_field_sampling (field_sampling.c) on the DC gun deck, sampled on
    the device at the top of each step: pages of interpolated fields (Ez,
    all of E, Br), of node arrays (Phi with the imposed potential, Q, Jz,
    Jr) and time sequences of range averages equal the reference's files in
    the FP64 form, including its call-wide state (Q after a Phi definition
    gets the imposed potential added; the r-direction time sequence averages
    over the last z range and radius set)."""
    fx = load("deck_sampling")
    s = run_deck(fx, tmp_path, monkeypatch)
    for name, cols in SAMPLING_PAGES + SAMPLING_SEQ:
        pages = session.read_sdds(str(tmp_path / ("spiffe." + name)))
        assert len(pages) == int(fx[name + "_pages"]), name
        for c in cols:
            got = np.concatenate([np.asarray(p["columns"][c], np.float64) for p in pages])
            assert np.array_equal(got, fx[name + "_" + c]), (name, c)
    s.close()


@pytest.mark.gpu
def test_field_sampling_split_form(tmp_path, monkeypatch):
    """The same sampling in the split form (Jz and Jr are not held in FP64
    there and are dropped from the deck): the same pages and rows, and the
    sampled fields within 1e-4 of the largest magnitude of the reference's."""
    fx = load("deck_sampling")
    deck = "\n".join(l for l in str(fx["deck"]).split("\n") if 'component="J' not in l)
    fx = dict(fx)
    fx["deck"] = np.array(deck)
    s = run_deck(fx, tmp_path, monkeypatch, precision="split32")
    for name, cols in SAMPLING_PAGES + SAMPLING_SEQ:
        if name in ("jz", "jr"):
            continue
        pages = session.read_sdds(str(tmp_path / ("spiffe." + name)))
        assert len(pages) == int(fx[name + "_pages"]), name
        for c in cols:
            got = np.concatenate([np.asarray(p["columns"][c], np.float64) for p in pages])
            ref = fx[name + "_" + c]
            assert got.shape == ref.shape, (name, c)
            assert np.max(np.abs(got - ref)) <= 1e-4 * max(np.max(np.abs(ref)), 1e-30), (name, c)
    s.close()


@pytest.mark.gpu
def test_field_saves_match_reference(tmp_path, monkeypatch):
    """define_field_saving (field_saving.c:46-213) on the DC gun deck in the
    FP64 form: the same pages, every column (Ez, Er, Jz, Jr, Bphi, Bphi2 and
    the metalFlags column the reference leaves at zero) equal to the
    reference's saves bit for bit (compared through SHA-256 digests)."""
    import hashlib

    fx = load("deck_fieldsave")
    s = run_deck(fx, tmp_path, monkeypatch)
    pages = session.read_sdds(str(tmp_path / "spiffe.flds"))
    assert len(pages) == int(fx["pages"])
    for c in ("Ez", "Er", "Jz", "Jr", "Bphi", "Bphi2", "metalFlags"):
        v = np.concatenate([np.asarray(p["columns"][c], np.float64) for p in pages])
        assert len(v) == int(fx["rows"])
        assert np.array_equal(v[:64], fx["head_" + c]), c
        assert hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest() == str(fx["sha_" + c]), c
    s.close()
