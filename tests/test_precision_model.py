"""CPU checks of the split-precision error model (oracle/precision_model.py):
its contraction form of the z transforms reproduces the oracle's transforms, and
its BF16 slicing is exact and converges."""
import numpy as np

from oracle import coral_oracle as co
from oracle import precision_model as pm
from tests.problems import equations, params


def test_bf16_slices_reconstruct():
    rng = np.random.default_rng(0)
    x = rng.standard_normal(1000) * np.exp(rng.uniform(-20, 20, 1000))
    s0 = pm.bf16(x)
    # 8 significant bits: relative rounding error <= 2^-8
    assert np.all(np.abs(s0 - x) <= 2.0 ** -8 * np.abs(x))
    for k, bound in ((2, 2.0 ** -16), (3, 2.0 ** -24), (4, 2.0 ** -32)):
        r = x - sum(pm.slices(x, k))
        assert np.all(np.abs(r) <= bound * np.abs(x))


def test_contraction_form_matches_oracle_transforms():
    eq, par = equations(), params(16, 12, 24)
    g = co.Solver(eq, par).g
    rng = np.random.default_rng(1)
    spec = rng.standard_normal((g.NXH, g.NYAA, g.NZ)) + 1j * rng.standard_normal((g.NXH, g.NYAA, g.NZ))
    s2p, p2s = pm.make_transforms(0, fp32_acc=False, fp32_fft=False)
    ph, b = co.spec_to_phys(spec, g), s2p(spec, g)
    assert np.abs(ph - b).max() <= 1e-12 * np.abs(ph).max()
    phys = rng.standard_normal((g.NYAA, g.NXAA, g.NZAA))
    a, b = co.phys_to_spec(phys, g), p2s(phys, g)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
    # four slices with exact accumulation: within ~2^-30 of the exact contraction
    s2p4, _ = pm.make_transforms(4, fp32_acc=False, fp32_fft=False)
    c = s2p4(spec, g)
    assert np.abs(c - ph).max() <= 1e-8 * np.abs(ph).max()


def test_int8_slice_contraction_accuracy():
    """Integer slices (shared exponent per row / column, exact accumulation):
    each slice adds ~7 bits relative to the row / column maximum."""
    rng = np.random.default_rng(2)
    inv, _ = pm.dct_matrices(48, 72)
    B = rng.standard_normal((48, 40)) * np.exp(rng.uniform(-6, 0, (48, 1)))
    ex = inv @ B
    errs = [np.abs(pm.gemm_int8(inv, B, k) - ex).max() / np.abs(ex).max() for k in (3, 4, 5, 6)]
    assert errs[0] < 1e-4 and errs[2] < 1e-8 and errs[3] < 1e-10
    assert all(b < a for a, b in zip(errs, errs[1:]))
