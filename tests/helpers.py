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


def fields_from(fx, modes=MODES, dt=None):
    lo, up, right, left = (int(v) for v in fx["bcs"])
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
