"""The allocation-free SOR entry point gives the instance path's answer.

spiffe_gpu_solve_poisson_cyl_noalloc exists for callers that may not allocate
device memory (their device memory belongs to another framework's pool, or
their loop forbids allocation after start-up).  Here it is called through the
C ABI on device arrays this test owns, twice in a row -- the second call
warm-starts from the first's result with a new driving term, so the shared
scratch array is reused with stale contents -- and each result is compared
with spiffe_gpu_solve_poisson_cyl on an instance holding the same inputs.
Both run the same kernel with the same grid, so the comparison is exact
(the tolerance the other SOR parity tests use).
"""
import ctypes as C

import numpy as np
import pytest

from spiffe_b200 import abi, gpu
from helpers import MODES, fields_from, load

pytestmark = pytest.mark.gpu


def noalloc_fn():
    lib = gpu.load()
    fn = lib.spiffe_gpu_solve_poisson_cyl_noalloc
    fn.argtypes = [C.POINTER(abi.Mesh), C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int64,
                   C.POINTER(C.c_int64), C.c_void_p]
    fn.restype = C.c_int
    return lib, fn


def test_noalloc_sor_matches_instance_path_twice():
    import torch

    fx = load("dcgun_poisson")
    f = fields_from(fx, modes=MODES, dt=float(fx["dt"]))
    rng = np.random.default_rng(11)
    shape = f.shape
    lib, fn = noalloc_fn()
    accuracy, limit = 1e-6, 3000

    psi_dev = torch.zeros(shape, dtype=torch.float64, device="cuda")
    flags_dev = torch.tensor(f.flags, dtype=torch.int16, device="cuda")
    psi_host = np.zeros(shape)
    for call in range(2):
        rhs = rng.normal(size=shape) * (1e4 if call == 0 else 3e3)
        rhs_dev = torch.tensor(rhs, dtype=torch.float64, device="cuda")
        # existing entry point on an instance with the same Psi and driving term
        ref = f.copy()
        ref["Psi"] = psi_host
        ref["Q"] = rhs
        g = gpu.GpuInstance(ref)
        n_ref = g.solve_poisson(0, accuracy, limit)
        psi_ref = g.fields(ref)["Psi"]
        g.close()
        # allocation-free entry point on the caller's device arrays
        torch.cuda.synchronize()
        n = C.c_int64(-7)
        rc = fn(C.byref(f.mesh), psi_dev.data_ptr(), rhs_dev.data_ptr(), flags_dev.data_ptr(), accuracy, limit,
                C.byref(n), None)
        assert rc == 0, lib.spiffe_gpu_last_error().decode()
        torch.cuda.synchronize()
        got = psi_dev.cpu().numpy()
        assert n.value == n_ref and 0 < n.value < limit
        assert np.array_equal(got, psi_ref), call
        psi_host = psi_ref


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    fx = load("dcgun_poisson")
    f = fields_from(fx, modes=MODES, dt=float(fx["dt"]))
    lib, fn = noalloc_fn()
    psi = torch.zeros(f.shape, dtype=torch.float64, device="cuda")
    flags = torch.tensor(f.flags, dtype=torch.int16, device="cuda")
    n = C.c_int64()
    rc = fn(C.byref(f.mesh), psi.data_ptr(), None, flags.data_ptr(), 1e-6, 20000, C.byref(n), None)
    assert rc != 0 and b"exceeds" in lib.spiffe_gpu_last_error()
    # meshes past the fixed row tables or the fixed block-sum array: each is
    # refused on the host before anything is launched, so a one-element
    # array stands in for the (absent) large one
    tiny = torch.zeros(1, dtype=torch.float64, device="cuda")
    tiny_flags = torch.zeros(1, dtype=torch.int16, device="cuda")
    for nz, nr in ((200, 5000), (1100, 4096)):
        mesh = abi.Mesh.from_buffer_copy(f.mesh)
        mesh.nz, mesh.nr = nz, nr
        n = C.c_int64(-7)
        rc = fn(C.byref(mesh), tiny.data_ptr(), tiny.data_ptr(), tiny_flags.data_ptr(), 1e-6, 100, C.byref(n), None)
        assert rc != 0 and b"exceeds" in lib.spiffe_gpu_last_error(), (nz, nr)
        assert n.value == -7
