"""CPU checks of the test infrastructure and host-side logic added with the
split-precision form, the time loop and the learned closure: the closure
network's restatement against finite differences, the integer-digit
contraction model against the exact contraction, the Nusselt post-processing
against a direct evaluation of the benchmark's rule."""
import math
import os
import tempfile

import numpy as np

from oracle import closure_oracle as clo
from oracle import precision_model as pm


def test_closure_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = 0.1 * rng.standard_normal(clo.param_count())
    X = rng.standard_normal((30, clo.NIN))
    T = rng.standard_normal((30, clo.OUT))
    _, g = clo.loss_and_grad(p, X, T)
    # biases are not rounded to BF16, so central differences apply exactly
    offs = np.cumsum([0] + [o * i + o for o, i in clo.SIZES])
    for li, (o, i) in enumerate(clo.SIZES):
        for k in (0, o - 1):
            j = offs[li] + o * i + k
            e = 1e-6
            pp, pm_ = p.copy(), p.copy()
            pp[j] += e
            pm_[j] -= e
            fd = (clo.loss_and_grad(pp, X, T)[0] - clo.loss_and_grad(pm_, X, T)[0]) / (2 * e)
            assert abs(fd - g[j]) <= 1e-6 * max(1.0, abs(g[j])), (li, k, fd, g[j])


def test_digit_contraction_error_bounds():
    """Five signed base-256 digits per operand, 15 digit products, exact
    accumulation: the REDFT01 / REDFT10 contractions at NZ = 192 within 1e-10
    relative L2 and 3e-9 of each column's maximum."""
    inv, fwd = pm.dct_matrices(192, 288)
    rng = np.random.default_rng(1)
    X = rng.standard_normal((192, 200)) * np.exp2(rng.integers(-30, 30, 200))[None, :]
    P = rng.standard_normal((288, 200))
    for M, A in ((inv, X), (fwd, P)):
        a, b = pm.gemm_digits256(M, A), M @ A
        assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)
        assert (np.abs(a - b).max(axis=0) / np.abs(A).max(axis=0)).max() <= 3e-9
    d = pm.balanced_digits(np.array([2 ** 38, -2 ** 38, 12345678901, -1], dtype=np.int64), 5)
    assert all(np.all(np.abs(x) <= 128) for x in d)
    back = sum(x * 256 ** (4 - s) for s, x in enumerate(d))
    assert np.array_equal(back, np.array([2 ** 38, -2 ** 38, 12345678901, -1]))


def test_nusselt_rule():
    from coral_b200 import nusselt
    NZAA = 72
    n = 401
    t = np.cumsum(np.full(n, 1e-3)) + 0.1 * np.sin(np.arange(n))[:] * 1e-4
    rng = np.random.default_rng(2)
    top = 0.02 + 1e-3 * rng.standard_normal(n)
    bot = -0.02 + 1e-3 * rng.standard_normal(n)
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(os.path.join(d, "Timeseries"))
        t.tofile(os.path.join(d, "Timeseries", "time.dat"))
        top.tofile(os.path.join(d, "Timeseries", "tFull_XYavg_z00001.dat"))
        bot.tofile(os.path.join(d, "Timeseries", "tFull_XYavg_z%05d.dat" % NZAA))
        m, s, q = nusselt.mean_nusselt(d, NZAA)
    dz = 0.5 - 0.5 * math.cos(math.pi / 2 / NZAA)
    dt = np.diff(t)
    k = (n - 1) // 4
    vals = []
    for i in range(1, 4):
        sl = slice(i * k, (i + 1) * k)
        vals += [np.sum(dt[sl] * top[sl]) / np.sum(dt[sl]) / dz, -np.sum(dt[sl] * bot[sl]) / np.sum(dt[sl]) / dz]
    assert abs(m - np.mean(vals)) <= 1e-12 * abs(m)
    assert abs(s - np.std(vals)) <= 1e-12 * abs(m)
