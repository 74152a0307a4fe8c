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


def test_emitter_surfaces_match_reference_fixture():
    """getBoundaryPoints (grid_drawing.c:541-760) on the emitter deck's
    boundary: the nodes and emission sides of materials 2 and 3 equal the
    reference's."""
    fx = load("deck_emitter")
    for m in (2, 3):
        iz, ir, d = geometry.boundary_points(151, 101, 0.0, 0.03, 0.02, str(fx["geo"]), m)
        assert np.array_equal(iz, fx[f"bp{m}_iz"]) and np.array_equal(ir, fx[f"bp{m}_ir"]), m
        assert np.array_equal(d, fx[f"bp{m}_dir"]), m


@pytest.mark.skipif(REF_EXAMPLES is None, reason="reference examples not present")
@pytest.mark.parametrize("tag", [(5, (2, 3, 4, 5)), (6, (10, 11)), (7, (8, 9, 10, 11, 12))])
def test_emitter_surfaces_match_reference(tag, tmp_path):
    """The reference's DC gun example boundary with some of its points tagged
    as a material: a slanted line and an arc (corner nodes inserted), the
    anode nose, the anode face and drift pipe.  Both give the same surface
    nodes and emission sides."""
    from oracle import pyoracle

    material, rows = tag
    lines = open(os.path.join(REF_EXAMPLES, "dcGun/dc.geo")).read().splitlines()
    for k in rows:
        lines[k] = lines[k].replace("&end", ", material_id=%d &end" % material)
    text = "\n".join(lines) + "\n"
    (tmp_path / "b.geo").write_text(text)
    nz, nr, zmax, rmax = 165, 165, 0.072, 0.042
    cmd = workloads.geometry_command(nz, nr, 0.0, zmax, rmax, "b.geo")
    (riz, rir, rd), = pyoracle.run_reference([("command", cmd), ("boundary_points", material)], cwd=str(tmp_path))
    iz, ir, d = geometry.boundary_points(nz, nr, 0.0, zmax, rmax, text, material)
    assert len(riz) > 3
    assert np.array_equal(iz, riz) and np.array_equal(ir, rir)
    assert np.array_equal(d, rd)
