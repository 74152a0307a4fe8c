"""define_geometry: the product's rasteriser gives the reference's flags."""
import os

import numpy as np
import pytest

from spiffe_b200 import geometry, workloads
from helpers import load, reference_file


@pytest.mark.parametrize("name", ["pillbox_fdtd", "dcgun_geometry", "gun16_geometry"])
def test_flags_match_reference(name):
    fx = load(name)
    geo = str(fx["geo"]) if "geo" in fx else workloads.PillboxConfig().geo_text()
    flags, psi = geometry.rasterise(int(fx["nz"]), int(fx["nr"]), float(fx["zmin"]), float(fx["zmax"]),
                                    float(fx["rmax"]), geo)
    assert np.array_equal(flags, fx["flags"])
    if "PsiImposed" in fx:
        assert np.array_equal(psi, fx["PsiImposed"])


REF_EXAMPLES = reference_file("examples")


@pytest.mark.skipif(REF_EXAMPLES is None, reason="reference examples not present")
@pytest.mark.parametrize("rel,nz,nr,zmax,rmax", [
    ("dcGun/dc.geo", 165, 165, 0.072, 0.042),
    ("apsTCRFGun/excite/mg6mm-3.geo", 165, 165, 0.0959148653920, 0.04289777777),
])
def test_reference_example_geometries(rel, nz, nr, zmax, rmax, tmp_path):
    """The reference's own example boundaries, rasterised by both."""
    from oracle import pyoracle

    src = os.path.join(REF_EXAMPLES, rel)
    text = open(src).read()
    (tmp_path / "b.geo").write_text(text)
    cmd = workloads.geometry_command(nz, nr, 0.0, zmax, rmax, "b.geo")
    ref_flags, ref_psi = pyoracle.run_reference([("command", cmd), ("get_flags",), ("get_field", "PsiImposed")],
                                                cwd=str(tmp_path))
    flags, psi = geometry.rasterise(nz, nr, 0.0, zmax, rmax, text)
    assert np.array_equal(flags, ref_flags)
    assert np.array_equal(psi, ref_psi)


def test_bad_boundary_is_rejected():
    with pytest.raises(Exception):
        geometry.rasterise(20, 20, 0.0, 0.01, 0.01, "&po x=0, y=0 &end\n&po x=0.5, y=0 &end\n")
