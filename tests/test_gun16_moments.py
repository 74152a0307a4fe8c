"""The 1.6-cell gun (the benchmark workload) in both forms, compared at the exit.

Both forms start from the same state, run the same perform_integration loop
(Poisson correction every 20 steps) until the bunch has crossed the exit
screen at z = 150 mm - dz, and record the crossings there.  The split form's
exit-plane moments (transmitted charge, mean kinetic energy, rms energy
spread, rms bunch length, normalized rms emittance), reduced on the device
(and checked against the host definition on the same records), must lie
within 0.5% of the FP64 form's.  The relative L2 differences of the fields are printed
beside them, taken half way (step 6,000, the bunch inside the gun): once the
bunch has left, the FP64 form's correction potential falls to round-off
(~1e-9 V) while the split form's stays at its FP32 rounding level (~0.3 V),
so a relative Psi difference at the end measures nothing.

The moments compare the split form with its default multigrid Poisson
solver.  The fields compare it with the reference's SOR, as the FP64 form
solves: that SOR stops at its iteration cap here, short of the stop rule,
and the multigrid solves past it, so with multigrid the field difference
measures the cap, not the split form's rounding (both are printed).

Field tolerance.  The beam-loaded fields are chaotic in the beam: two FP64
runs whose initial states differ only by the split form's rounding of that
state (positions to an FP32 offset in a cell, momenta, charge and fields to
FP32) already differ at step 6,000.  That FP64-vs-FP64 difference is the
sensitivity floor of this workload.  Without Poisson corrections the split
form, which rounds every step rather than once, stays within twice that
floor.  With them, the FP64 dynamics are far calmer (the floor falls by five
orders), and the split form's difference is set by the corrections
themselves: each solves for the error charge of div E, which in FP32 fields
includes the rounding of E (~1e-7 of the RF field), and subtracts that
potential's gradient from E.  Ez stays within max(FIELD_TOL, 4 x floor);
Er and Bphi, which carry the beam's own field, within 64 x floor.
"""
import numpy as np
import pytest

from spiffe_b200 import abi, gpu, moments, workloads
from helpers import rel_l2

pytestmark = pytest.mark.gpu

MOMENT_TOL = 5e-3
FIELD_TOL = 1e-5
FLOOR_FACTOR = 4.0      # Ez
CORRECTION_FACTOR = 64.0  # Er, Bphi: the corrections' FP32 div-E noise
STEPS = 12000  # the bunch needs about 9,000 steps of 17.7 um to reach the exit


def run(precision, cfg, f, b, steps=STEPS, solver=None, corrections=True):
    g = gpu.GpuInstance(f, capacity=b.capacity, precision=precision)
    if precision == gpu.PRECISION_F64:
        g.set_deposit_order(1)  # the reference's particle-order sums: a deterministic FP64 run
    if solver is not None:
        g.set_poisson_solver(solver)
    g.upload_beam(b)
    g.add_screen(cfg.screen_z(), 1, capacity=b.capacity)
    g.configure_run(space_charge=1, push=abi.push_options(abi.COMPACT_SWAP, abi.SCREEN_PARTICLE),
                    poisson=cfg.poisson() if corrections else None)
    g.run_begin()
    g.run_steps(STEPS // 2)
    mid = g.fields(f)
    if steps > STEPS // 2:
        g.run_steps(steps - STEPS // 2)
    rec = g.screen(0, capacity=b.capacity).records()
    dev = g.screen_moments(0)
    np_end, _ = g.counts()
    g.close()
    # the device reduction against the host definition on the same records
    host = moments.exit_moments(rec)
    assert dev["count"] == host["count"]
    for k, v in moments.relative_errors(dev, host).items():
        assert v <= 1e-12, (k, v)
    return rec, mid, np_end, dev


def rounded_by_split_form(f, b):
    """The initial state as the split form holds it, back in FP64."""
    g = gpu.GpuInstance(f, capacity=b.capacity, precision=gpu.PRECISION_SPLIT32)
    g.upload_beam(b)
    fr, br = g.fields(f), g.download_beam(abi.Beam(b.capacity))
    g.close()
    return fr, br


def test_gun16_exit_moments_split_vs_f64():
    cfg = workloads.Gun16Config()
    f, b = cfg.state()
    r64, o64, n64, m64 = run(gpu.PRECISION_F64, cfg, f, b)
    r32, o32, n32, m32 = run(gpu.PRECISION_SPLIT32, cfg, f, b)
    # the field comparison with the reference's solver on both sides: the
    # FP64 form's SOR stops at its 1000 half-sweep cap, short of the stop
    # rule, and the multigrid solves past it, so their fields differ by the
    # cap's error, not by the split form's rounding
    _, o32s, _, _ = run(gpu.PRECISION_SPLIT32, cfg, f, b, steps=STEPS // 2, solver=gpu.POISSON_SOR)
    fr, br = rounded_by_split_form(f, b)
    _, o64r, _, _ = run(gpu.PRECISION_F64, cfg, fr, br, steps=STEPS // 2)
    err = moments.relative_errors(m32, m64)
    fields = {n: rel_l2(o32s[n], o64[n]) for n in ("Ez", "Er", "Bphi", "Psi")}
    fields_mg = {n: rel_l2(o32[n], o64[n]) for n in ("Ez", "Er", "Bphi", "Psi")}
    floor = {n: rel_l2(o64r[n], o64[n]) for n in ("Ez", "Er", "Bphi", "Psi")}
    print("gun16 exit moments FP64 ", m64)
    print("gun16 exit moments split", m32)
    print("gun16 relative errors   ", err)
    print("gun16 field rel L2 (mid), both with SOR", fields)
    print("gun16 field rel L2 (mid), split with multigrid", fields_mg)
    print("gun16 FP64 floor (mid)  ", floor)
    print("gun16 particles left    ", n64, n32)
    assert m64["count"] > 0.5 * cfg.n_macro, "the bunch has not crossed the exit screen"
    assert abs(m32["count"] - m64["count"]) <= max(2, MOMENT_TOL * m64["count"])
    for k, v in err.items():
        assert v <= MOMENT_TOL, (k, v)
    assert fields["Ez"] <= max(FIELD_TOL, FLOOR_FACTOR * floor["Ez"]), (fields["Ez"], floor["Ez"])
    for n in ("Er", "Bphi"):
        assert fields[n] <= CORRECTION_FACTOR * floor[n], (n, fields[n], floor[n])
    # without corrections: rounding every step behaves as rounding once
    _, a, _, _ = run(gpu.PRECISION_F64, cfg, f, b, steps=STEPS // 2, corrections=False)
    _, r, _, _ = run(gpu.PRECISION_F64, cfg, fr, br, steps=STEPS // 2, corrections=False)
    _, sp, _, _ = run(gpu.PRECISION_SPLIT32, cfg, f, b, steps=STEPS // 2, corrections=False)
    off = {n: rel_l2(sp[n], a[n]) for n in ("Ez", "Er", "Bphi")}
    floor_off = {n: rel_l2(r[n], a[n]) for n in ("Ez", "Er", "Bphi")}
    print("gun16 without corrections: split", off, "floor", floor_off)
    for n in ("Ez", "Er", "Bphi"):
        assert off[n] <= 2 * floor_off[n], (n, off[n], floor_off[n])
