"""CPU-side checks of the C ABI library: it loads, exports exactly what include/fp_capi.h declares, and
refuses to compute without a CUDA device (no CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest

from focalors_poisson_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(fp_\w+)\s*\(", src, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(capi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 7
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert names == set(capi.SIGNATURES), names ^ set(capi.SIGNATURES)


def test_no_cpu_fallback_without_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    f = np.ones((4, 6))
    with pytest.raises(capi.FpError) as e:
        capi.transform(0, 0, f)
    assert e.value.code == 2
    with pytest.raises(capi.FpError):
        capi.Rect(4, 6, 0.1, 0.1, [0, 0, 0, 0])
