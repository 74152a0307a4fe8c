"""Named single-kernel cases for profiling, on the benchmark's workloads.

    python -m spiffe_b200.cases sor [--half-sweeps 200] [--repeat 2] [--precision split32|f64]
    python -m spiffe_b200.cases mg [--repeat 2]

``sor``: the reference's SOR (selected explicitly: the split form's default
solver is the multigrid) on the 1.6-cell gun mesh (3000 x 820 update nodes)
with a right-hand side of seeded normal noise (x 1e3), run for exactly the
given number of half-sweeps (an accuracy of 1e-300 never stops it early),
the given number of times on one instance, so that a profiler can skip the
first (setup) launch and capture a warm one.

``mg``: the split form's multigrid on the same mesh and right-hand side,
solved from zero to the stop rule sum|r| < 1e-6 sum|rhs| the given number
of times (each from zero again).
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
    if precision == "split32":
        g.set_poisson_solver(gpu.POISSON_SOR)
    n = None
    for _ in range(repeat):
        n = g.solve_poisson(0, 1e-300, half_sweeps)
    g.synchronize()
    g.close()
    return n


def mg(repeat):
    cfg = workloads.Gun16Config()
    f, b = cfg.state()
    f["Q"] = np.random.default_rng(1).normal(size=f.shape) * 1e3
    f["Psi"] = np.zeros(f.shape)
    g = gpu.GpuInstance(f, capacity=b.capacity, precision=gpu.PRECISION_SPLIT32)
    n = None
    for _ in range(repeat):
        g.upload_fields(f)
        n = g.solve_poisson(0, 1e-6, 100)
    g.synchronize()
    g.close()
    return n


def main():
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["sor", "mg"])
    p.add_argument("--half-sweeps", type=int, default=200)
    p.add_argument("--repeat", type=int, default=2)
    p.add_argument("--precision", default="split32", choices=["split32", "f64"])
    a = p.parse_args()
    if a.case == "sor":
        print("sor", sor(a.half_sweeps, a.repeat, a.precision))
    elif a.case == "mg":
        print("mg", mg(a.repeat))


if __name__ == "__main__":
    main()
