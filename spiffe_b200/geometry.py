"""define_geometry: &po boundary text -> metal flags (host code in libspiffe_b200)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, gpu


class GeometryOptions(C.Structure):
    _fields_ = [("nz", C.c_int32), ("nr", C.c_int32), ("zmin", C.c_double), ("zmax", C.c_double),
                ("rmax", C.c_double), ("zr_factor", C.c_double)]


def rasterise(nz, nr, zmin, zmax, rmax, boundary_text, zr_factor=1.0):
    """Returns (flags int16, PsiImposed float64), each (nz+1, nr+1)."""
    lib = gpu.load()
    fn = lib.spiffe_geometry_rasterise
    fn.argtypes = [C.POINTER(GeometryOptions), C.c_char_p, C.POINTER(C.c_int16), C.POINTER(C.c_double),
                   C.POINTER(C.c_int16)]
    fn.restype = C.c_int
    o = GeometryOptions(nz, nr, zmin, zmax, rmax, zr_factor)
    flags = np.zeros((nz + 1, nr + 1), np.int16)
    psi = np.zeros((nz + 1, nr + 1))
    rc = fn(C.byref(o), boundary_text.encode(), flags.ctypes.data_as(C.POINTER(C.c_int16)),
            psi.ctypes.data_as(C.POINTER(C.c_double)), None)
    if rc != 0:
        raise gpu.SpiffeGpuError(f"define_geometry: {lib.spiffe_gpu_last_error().decode()}")
    return flags, psi


def boundary_points(nz, nr, zmin, zmax, rmax, boundary_text, material_id, zr_factor=1.0):
    """The emitter surface of a material (getBoundaryPoints): (iz, ir,
    direction) arrays, one entry per node, direction[k] the side segment
    k -> k+1 emits to (abi.EMITS_*), the last entry 0."""
    lib = gpu.load()
    fn = lib.spiffe_geometry_boundary_points
    fn.argtypes = [C.POINTER(GeometryOptions), C.c_char_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.POINTER(C.c_int64)]
    fn.restype = C.c_int
    o = GeometryOptions(nz, nr, zmin, zmax, rmax, zr_factor)
    n = C.c_int64(0)
    if fn(C.byref(o), boundary_text.encode(), material_id, 0, None, None, None, C.byref(n)) != 0:
        raise gpu.SpiffeGpuError(f"define_emitter: {lib.spiffe_gpu_last_error().decode()}")
    iz, ir, d = np.zeros(n.value, np.int32), np.zeros(n.value, np.int32), np.zeros(n.value, np.int16)
    if n.value and fn(C.byref(o), boundary_text.encode(), material_id, n.value, iz.ctypes.data, ir.ctypes.data,
                      d.ctypes.data, C.byref(n)) != 0:
        raise gpu.SpiffeGpuError(f"define_emitter: {lib.spiffe_gpu_last_error().decode()}")
    return iz, ir, d


def fields_for(nz, nr, zmin, zmax, rmax, boundary_text, modes=abi.FL_TM_FIELDS | abi.FL_RADIAL_INTERP |
               abi.FL_LONGIT_INTERP, **bcs):
    """An abi.Fields whose flags and PsiImposed come from the boundary text."""
    flags, psi = rasterise(nz, nr, zmin, zmax, rmax, boundary_text)
    f = abi.Fields(nz, nr, zmin, zmax, rmax, modes=modes, flags=flags, **bcs)
    f["PsiImposed"] = psi
    return f
