"""The DC gun (space-charge dominated, a Poisson correction every step) in both forms.

The gun of the DC-gun configuration -- 300 kV across a 10 mm gap, a 3 mm
anode hole, 0.5 nC in a 100 ps flat top already emitted from a 2 mm disk --
on a mesh coarsened by two (751 x 501 nodes at 40 um) with 1,000,000
macroparticles, run in both forms until the whole bunch has crossed the exit
screen at z = 30 mm - dz.  Every step runs a Poisson correction: the FP64
form with the reference's SOR (accuracy 1e-6, at most 1000 half-sweeps), the
split form with its default multigrid solver to the same stop rule.  The
split form's exit-plane moments (reduced on the device) must lie within
0.5% of the FP64 form's;
its corrections must all meet the stop rule (the per-step residual norms of
both forms are printed from the instances' correction logs).
"""
import numpy as np
import pytest

from spiffe_b200 import abi, gpu, moments, workloads

pytestmark = pytest.mark.gpu

MOMENT_TOL = 5e-3
STEPS = 3600  # the bunch tail needs about 3,300 steps of 47 fs to reach the exit


def run(precision, cfg, f, b):
    g = gpu.GpuInstance(f, capacity=b.capacity, precision=precision)
    g.upload_beam(b)
    g.add_screen(cfg.screen_z(), 1, capacity=b.capacity)
    g.configure_run(space_charge=1, push=abi.push_options(abi.COMPACT_SWAP, abi.SCREEN_PARTICLE),
                    poisson=cfg.poisson())
    g.run_begin()
    g.run_steps(STEPS)
    dev = g.screen_moments(0)
    log = g.poisson_log()
    g.close()
    return dev, log


def test_dcgun_exit_moments_split_vs_f64():
    cfg = workloads.DcGunConfig(nz=751, nr=501, n_macro=1_000_000)
    f, b = cfg.state()
    m64, log64 = run(gpu.PRECISION_F64, cfg, f, b)
    m32, log32 = run(gpu.PRECISION_SPLIT32, cfg, f, b)
    err = moments.relative_errors(m32, m64)
    rel64 = log64[:, 2] / log64[:, 3]
    rel32 = log32[:, 2] / log32[:, 3]
    print("dcgun exit moments FP64 ", m64)
    print("dcgun exit moments split", m32)
    print("dcgun relative errors   ", err)
    print("dcgun corrections: FP64 %d, half-sweeps mean %.0f, capped %d, residual/rhs median %.2e max %.2e"
          % (len(log64), np.mean(np.where(log64[:, 1] < 0, 1000, log64[:, 1])), np.sum(log64[:, 1] < 0),
             np.median(rel64), rel64.max()))
    print("dcgun corrections: split %d, V-cycles mean %.2f max %d, residual/rhs median %.2e max %.2e"
          % (len(log32), log32[:, 1].mean(), log32[:, 1].max(), np.median(rel32), rel32.max()))
    assert m64["count"] > 0.9 * cfg.n_macro, "the bunch has not crossed the exit screen"
    assert len(log32) == len(log64) >= STEPS - 1
    # every split-form correction met the stop rule
    assert np.all(log32[:, 1] > 0) and np.all(rel32 < 1e-6)
    assert abs(m32["count"] - m64["count"]) <= max(2, MOMENT_TOL * m64["count"])
    for k, v in err.items():
        assert v <= MOMENT_TOL, (k, v)
