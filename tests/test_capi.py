"""CPU checks of the C-ABI library: it loads and exports every symbol the header declares."""
import os
import re

from coral_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    hdr = open(os.path.join(ROOT, "include", "coral_b200.h")).read()
    names = set(re.findall(r"\b(coral_[a-z0-9_]+)\s*\(", hdr))
    assert names, "no declarations found"
    assert names == set(_lib.SIGNATURES), names ^ set(_lib.SIGNATURES)
    for n in names:
        assert hasattr(lib, n)


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        return
    from coral_b200.solver import PlaneLayer, CoralError
    from tests.problems import equations, params
    try:
        PlaneLayer(equations(), params(16, 16, 16))
    except CoralError as e:
        assert e.code == -9
    else:
        raise AssertionError("expected CORAL_ENODEV")
