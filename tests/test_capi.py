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


def _build_harness(out_dir):
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    assert gcc, "gcc not found"
    lib_dir = os.path.join(ROOT, "coral_b200")
    exe = os.path.join(out_dir, "harness")
    subprocess.run([gcc, "-O2", "-std=c99", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_harness", "harness.c"), "-L" + lib_dir, "-lcoral_b200",
                    "-L/usr/local/cuda/lib64", "-lcudart", "-lm", "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    return exe


def test_plain_c_caller_compiles_and_links():
    """The header is plain C: a C99 driver (tests/c_harness/harness.c) compiles
    without warnings and links against the library."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        assert os.path.exists(_build_harness(d))


def test_fortran_module_binds_every_entry_point():
    """include/coral_b200.f90 declares a bind(C) interface for every function of
    the C header, under the same C name."""
    hdr = open(os.path.join(ROOT, "include", "coral_b200.h")).read()
    names = set(re.findall(r"\b(coral_[a-z0-9_]+)\s*\(", hdr))
    f90 = open(os.path.join(ROOT, "include", "coral_b200.f90")).read()
    bound = set(re.findall(r'bind\(C, name="(coral_[a-z0-9_]+)"\)', f90))
    assert names == bound, names ^ bound


def test_replacement_marching_include_defines_the_bound_procedures():
    """include/PL_IMEX_timestepping_marching_b200.f90 (the replacement for
    src/plane_layer/PL_IMEX_timestepping_marching.f90, checked textually: no
    Fortran compiler here) defines every procedure of the original include
    (names in tests/golden/marching_procedures.txt) except Compute_1dCheby_transform,
    which the type does not bind and only the original transform_sources calls;
    its subroutines and functions are closed; every coral_* it calls has a
    bind(C) interface in coral_b200.f90; the user's source and mask includes
    are kept."""
    src = open(os.path.join(ROOT, "include", "PL_IMEX_timestepping_marching_b200.f90")).read()
    code = "\n".join(l.split("!")[0] for l in src.splitlines())
    want = [n.strip() for n in open(os.path.join(ROOT, "tests", "golden", "marching_procedures.txt")) if n.strip()]
    defined = set(m.lower() for m in re.findall(r"^\s*(?:real\(kind=dp\)\s+)?(?:subroutine|function)\s+(\w+)",
                                                   code, re.I | re.M))
    missing = [n for n in want if n.lower() not in defined and n != "Compute_1dCheby_transform"]
    assert not missing, missing
    for kind in ("subroutine", "function"):
        opened = re.findall(r"^\s*(?:real\(kind=dp\)\s+)?%s\s+(\w+)" % kind, code, re.I | re.M)
        closed = re.findall(r"^\s*end\s+%s\s+(\w+)" % kind, code, re.I | re.M)
        assert [n.lower() for n in opened] == [n.lower() for n in closed], kind
    f90 = open(os.path.join(ROOT, "include", "coral_b200.f90")).read()
    bound = set(re.findall(r'bind\(C, name="(coral_[a-z0-9_]+)"\)', f90))
    called = set(re.findall(r"\b(coral_[a-z_]+)\s*\(", code)) - {n.lower() for n in defined}
    called = {c for c in called if not c.startswith("coral_b200_")}
    assert called and called <= bound, called - bound
    assert 'include "PL_user_sources_definitions.f90"' in code
    assert 'include "PL_user_penalisation_mask.f90"' in code
    assert "coral_b200_handle" in f90
