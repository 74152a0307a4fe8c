"""The C-ABI libraries load and export every entry point their headers declare
(no GPU needed: nothing is called)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(spiffe_[a-z0-9_]+)\s*\(", re.M)


def declared(header):
    with open(os.path.join(ROOT, "include", header)) as f:
        text = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
    return sorted(set(DECL.findall(text)))


def test_product_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(os.path.join(ROOT, "spiffe_b200", "libspiffe_b200.so"))
    names = declared("spiffe_b200.h")
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_all_public_headers_are_covered():
    lib = ctypes.CDLL(os.path.join(ROOT, "spiffe_b200", "libspiffe_b200.so"))
    for h in os.listdir(os.path.join(ROOT, "include")):
        for n in declared(h):
            if n.startswith("spiffe_gpu_"):
                assert hasattr(lib, n), (h, n)


def test_oracle_library_loads():
    from oracle import pyoracle

    pyoracle.Oracle()


def test_binding_without_gpu_fails_loudly():
    """With no device the binding raises instead of computing anything."""
    import numpy as np

    from spiffe_b200 import abi, gpu

    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    f = abi.Fields(10, 10, 0.0, 0.01, 0.01)
    with pytest.raises(gpu.SpiffeGpuError):
        gpu.GpuInstance(f)
