"""The allocation-free inverse transform (coral_spec_to_phys_noalloc).

Callers that cannot call cudaMalloc -- their device memory belongs to another
allocator or runtime, or allocation is forbidden once they are running -- use
this entry point with their own device buffers; its scratch is a fixed 64 MiB
__device__ array inside the library.  This file is collected last so that a run
that stops at the first failure has run every other test first; it also passes
on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from tests.problems import equations, params

pytestmark = pytest.mark.gpu


def _dptr(t):
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), ctypes.POINTER(ctypes.c_double))


@pytest.mark.parametrize("N", [(32, 24, 24), (8, 16, 8)])
def test_noalloc_spec_to_phys_matches_handle_path_twice(N):
    """Two calls in a row (they share the scratch array) agree with the handle's
    coral_spec_to_phys and with the oracle's c2r transform.  (32, 24, 24) has
    transform lengths 48 / 36 / 36, all compiled FFT plans; (8, 16, 8) has
    12 / 24 / 12, so the x and z passes take the run-time plans and their
    second shared-memory buffer."""
    import torch
    from coral_b200 import _lib
    from coral_b200.solver import PlaneLayer
    from oracle import coral_oracle as co

    lib = _lib.load()
    torch.cuda.set_device(0)
    NX, NY, NZ = N
    pl = PlaneLayer(equations(), params(NX, NY, NZ, Lx=2.0, Ly=3.0))
    g = co.Geometry(NX, NY, NZ, 2.0, 3.0, 1.0, 0.5)
    rng = np.random.default_rng(123)
    for call in range(2):
        spec = rng.standard_normal((pl.NXH, pl.NYAA, pl.NZ)) + 1j * rng.standard_normal((pl.NXH, pl.NYAA, pl.NZ))
        ref = pl.spec_to_phys(spec)
        ora = co.spec_to_phys(spec, g)
        d_spec = torch.from_numpy(np.ascontiguousarray(spec).view(np.float64).ravel()).cuda()
        d_phys = torch.full((pl.NYAA * pl.NXAA * pl.NZAA,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.coral_spec_to_phys_noalloc(NX, NY, NZ, _dptr(d_spec), _dptr(d_phys), None)
        assert rc == 0, lib.coral_last_error(None).decode()
        torch.cuda.synchronize()
        got = d_phys.cpu().numpy().reshape(pl.NYAA, pl.NXAA, pl.NZAA)
        # same tolerance as the transform parity tests
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), call
        assert np.abs(got - ora).max() <= 1e-13 * np.abs(ora).max(), call
    pl.close()


def test_noalloc_rejects_grids_beyond_the_scratch_limit():
    import torch
    from coral_b200 import _lib

    lib = _lib.load()
    torch.cuda.set_device(0)
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.coral_spec_to_phys_noalloc(384, 384, 192, _dptr(d), _dptr(d), None)
    assert rc == -1
    assert "64 MiB" in lib.coral_last_error(None).decode()
    # sizes far out of range are refused before any arithmetic on them
    rc = lib.coral_spec_to_phys_noalloc(1 << 30, 384, 192, _dptr(d), _dptr(d), None)
    assert rc == -1
    assert "multiples of 4" in lib.coral_last_error(None).decode()
