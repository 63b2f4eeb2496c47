"""C ABI checks that need no GPU: the built library loads, exports every
function include/cabanapd_b200.h declares with the binding's signature
table covering all of them, and refuses to run without a CUDA device
instead of falling back to the CPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "cabanapd_b200.h")) as fh:
        text = fh.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cpd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from cabanapd_b200 import system
    lib = ctypes.CDLL(system.LIB_PATH)
    names = _declared()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(system.SIGNATURES), set(names) ^ set(system.SIGNATURES)


def test_abi_version_and_params_layout():
    from cabanapd_b200 import system
    lib = system.load()
    assert lib.cpd_abi_version() == 4
    # cpd_params: 4 int32, 10 double, 5 int32 (+4 padding), 2 double
    # -> 16 + 80 + 20 + 4 + 16
    assert ctypes.sizeof(system.CpdParams) == 136


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import cabanapd_b200
    with pytest.raises(cabanapd_b200.CpdError):
        cabanapd_b200.System(dict(pd_model=1, horizon=0.1, K=1.0, dt=1.0))
