"""Named single-kernel cases for profiling, on the benchmark's workloads.

    python -m spiffe_b200.cases sor [--half-sweeps 200] [--repeat 2] [--precision split32|f64]

``sor``: the SOR of the 1.6-cell gun mesh (3000 x 820 update nodes) on a
right-hand side of seeded normal noise (x 1e3), run for exactly the given
number of half-sweeps (an accuracy of 1e-300 never stops it early), the
given number of times on one instance, so that a profiler can skip the
first (setup) launch and capture a warm one.
"""
import argparse

import numpy as np

from . import gpu, workloads


def sor(half_sweeps, repeat, precision):
    cfg = workloads.Gun16Config()
    f, b = cfg.state()
    f["Q"] = np.random.default_rng(1).normal(size=f.shape) * 1e3
    g = gpu.GpuInstance(f, capacity=b.capacity,
                        precision=gpu.PRECISION_SPLIT32 if precision == "split32" else gpu.PRECISION_F64)
    n = None
    for _ in range(repeat):
        n = g.solve_poisson(0, 1e-300, half_sweeps)
    g.synchronize()
    g.close()
    return n


def main():
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["sor"])
    p.add_argument("--half-sweeps", type=int, default=200)
    p.add_argument("--repeat", type=int, default=2)
    p.add_argument("--precision", default="split32", choices=["split32", "f64"])
    a = p.parse_args()
    if a.case == "sor":
        print("sor", sor(a.half_sweeps, a.repeat, a.precision))


if __name__ == "__main__":
    main()
