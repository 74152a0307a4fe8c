"""Shared builders for the parity tests: fixtures -> abi containers."""
import os

import numpy as np

from spiffe_b200 import abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MODES = abi.FL_TM_FIELDS | abi.FL_RADIAL_INTERP | abi.FL_LONGIT_INTERP
QoMC = -1.602176634e-19 / (9.1093837015e-31 * 2.99792458e8)


def reference_root():
    """The reference checkout whose sources built oracle/_ref (SPIFFE_REFERENCE
    overrides), or None where it is absent, as on the GPU boxes."""
    root = os.environ.get("SPIFFE_REFERENCE")
    if not root:
        rec = os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "reference_root.txt")
        if os.path.exists(rec):
            root = open(rec).read().strip()
    return root if root and os.path.isdir(root) else None


def reference_file(*parts):
    root = reference_root()
    return os.path.join(root, *parts) if root else None


def load(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def fields_from(fx, modes=MODES, dt=None, **bcs):
    """abi.Fields of a fixture's mesh; left_bc / right_bc override the fixture's."""
    lo, up, right, left = (int(v) for v in fx["bcs"])
    left, right = bcs.get("left_bc", left), bcs.get("right_bc", right)
    f = abi.Fields(int(fx["nz"]), int(fx["nr"]), float(fx["zmin"]), float(fx["zmax"]), float(fx["rmax"]),
                   modes=modes, left_bc=left, right_bc=right, lower_bc=lo, upper_bc=up, flags=fx["flags"])
    assert f.mesh.dz == float(fx["dz"]) and f.mesh.dr == float(fx["dr"])
    if dt is not None:
        f.mesh.dt = dt
    return f


def beam_from(fx, prefix="in_", capacity=None):
    n = len(fx[prefix + "z"])
    b = abi.Beam(capacity or n + 16)
    arrays = {k[len(prefix):]: v for k, v in fx.items() if k.startswith(prefix)}
    b.set(n, **arrays)
    b.npActive = int(np.sum(fx[prefix + "status"] & 1)) if (prefix + "status") in fx else n
    b.nextParticleID = n + 1
    b.QoMC = float(fx.get("QoMC", QoMC))
    b.stiffness = 1.0
    return b


def rel_l2(a, b):
    den = np.sqrt(np.sum(np.asarray(b, float) ** 2))
    num = np.sqrt(np.sum((np.asarray(a, float) - np.asarray(b, float)) ** 2))
    return num / den if den else num


def by_id(records, key="particleID"):
    order = np.argsort(records[key], kind="stable")
    return {k: np.asarray(v)[order] for k, v in records.items()}


TE_FIELDS = ("Ez", "Er", "Bphi", "Bphi2", "Ephi", "Br", "Bz", "Br2", "Bz2")


def te_fdtd_state(fx):
    """The gun16_te fixture's FDTD case: the gun mesh with TE and TM fields
    and constant currents, before its `steps` field steps."""
    f = fields_from(fx, modes=int(fx["modes"]), dt=float(fx["dt"]))
    for n in TE_FIELDS + ("Jz", "Jr", "Jphi"):
        f[n] = fx["in_" + n].astype(np.float64)
    return f


def te_push_state(fx):
    """The gun16_te fixture's deposition and push case (pillbox mesh, TE and
    TM fields, imposed fields, 1,500 particles with angular momentum)."""
    sub = {k[2:]: v for k, v in fx.items() if k.startswith("p_")}
    f = fields_from(sub, modes=int(sub["modes"]), dt=float(sub["dt"]))
    f.mesh.time_step = int(sub["time_step"])
    f.mesh.time = f.mesh.time_step * f.mesh.dt
    for k, v in sub.items():
        if k.startswith("f_"):
            f[k[2:]] = v.astype(np.float64)
    return f, beam_from(sub), sub


def poisson_residual(f, psi, rhs):
    """sum |rhs - A psi| over the nodes solve_poisson_cyl updates
    (poisson.c:57-117, both colours at once) and sum |rhs| over iz < nz,
    ir < nr-1 (poisson.c:40-43), in FP64."""
    m = f.mesh
    nz, nr = m.nz, m.nr
    a = 1 / m.dz ** 2
    dr2 = m.dr ** 2
    e = -2 * (1 / m.dz ** 2 + 1 / dr2)
    lo = 0 if m.left_bc == abi.DIRICHLET else 1
    hi = nz - 1 if m.right_bc == abi.DIRICHLET else nz - 2
    rows = np.arange(lo, hi + 1)
    up = np.where(rows == nz - 1, rows - 1, rows + 1) if hi == nz - 1 else rows + 1
    dn = np.where(rows == 0, rows + 1, rows - 1) if lo == 0 else rows - 1
    cols = nr - 1
    ir = np.arange(cols, dtype=float)
    c = np.where(ir > 0, 1 / dr2 * (1 + 0.5 / np.maximum(ir, 1)), 4 / dr2)
    d = np.where(ir > 0, 1 / dr2 * (1 - 0.5 / np.maximum(ir, 1)), 0.0)
    dg = np.where(ir > 0, e, e - 2 / dr2)
    P = psi
    left = np.concatenate([np.zeros((len(rows), 1)), P[rows, : cols - 1]], axis=1)
    ap = a * (P[up, :cols] + P[dn, :cols]) + c * P[rows, 1: cols + 1] + d * left + dg * P[rows, :cols]
    rh = rhs[rows, :cols] if rhs is not None else 0.0
    upd = (f.flags[rows, :cols] & abi.FL_IS_METAL) == 0
    res = np.abs(np.where(upd, rh - ap, 0.0)).sum()
    drive = np.abs(rhs[:nz, :cols]).sum() if rhs is not None else 0.0
    return res, drive
