"""The plain C driver (tests/c_harness/harness.c) on the GPU: create from the
files, import QuickSave, factorise, march, read back -- and the same state
change as the Python path."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from tests.problems import equations, params
from tests.test_capi import _build_harness

pytestmark = pytest.mark.gpu


def test_c_driver_runs_and_matches_python():
    from coral_b200 import initial_conditions as ic
    from coral_b200.solver import PlaneLayer
    with tempfile.TemporaryDirectory() as d:
        exe = _build_harness(d)
        eq, par = os.path.join(d, "eq"), os.path.join(d, "par")
        open(eq, "w").write(equations())
        open(par, "w").write(params(16, 16, 24, dt=1e-4))
        qs = os.path.join(d, "qs")
        ic.white_noise_temperature(qs, 16, 16, 24, seed=11)
        out = subprocess.run([exe, eq, par, qs, "5", "1e-4"], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        tok = out.stdout.split()
        rel_c = float(tok[tok.index("rel_change") + 1])
        pl = PlaneLayer.from_files(eq, par)
        pl.import_quicksave(qs)
        f0 = pl.get_field(0)
        pl.march_forward(1e-4, 5)
        f1 = pl.get_field(0)
        rel_py = np.linalg.norm(f1 - f0) / np.linalg.norm(f0)
        assert abs(rel_c - rel_py) <= 1e-12 * rel_py
        pl.close()
