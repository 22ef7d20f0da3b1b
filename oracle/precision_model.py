"""Error model of a split-precision form of the timestep (test infrastructure).

TEST INFRASTRUCTURE ONLY, like ``coral_oracle``: a CPU model, not product code
and not imported by the product.  It answers one design question before any
tensor-core kernel is written: how accurate must the transforms be for the
timestep to stay within a given relative error of the FP64 oracle?

The model swaps the oracle's transforms (``spec_to_phys`` / ``phys_to_spec``,
which restate src/slabs.fftw3mpi/transforms.f90:155-301) for variants in which

* the z (Chebyshev) transform is a dense contraction with the REDFT01 /
  REDFT10 matrices (NZAA x NZ and NZ x NZAA), both operands split into k
  BF16 slices (round to nearest even), the slice products with i + j < k
  (i + j <= 2 for k = 3: six products) formed exactly and accumulated either in
  FP32 (a tensor-core accumulator) or exactly (FP64 here: the accumulation of
  an integer-slice scheme is exact);
* or the z contraction uses int8 slices with one shared exponent per matrix
  row and per data column, the slice products accumulated exactly (an integer
  tensor-core GEMM accumulates in INT32) and combined in FP64;
* the x / y FFTs run in FP32 or FP64.

Everything else (band LU, stage sums, the state) stays the oracle's FP64.  The
state after n steps is compared with the FP64 oracle started from the same
seeded initial condition as the benchmark (white-noise temperature, amplitude
1e-3, times sin(pi z'), PCG64 seed 2; Ra = 1e8 no-slip recipe, dt = 1e-6).

    python oracle/precision_model.py NX NZ STEPS
"""
import os
import sys
import time

import numpy as np
import scipy.fft as sfft

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import coral_oracle as co  # noqa: E402


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    u = (u + (0x7FFF + ((u >> 16) & 1))) & np.uint32(0xFFFF0000)
    return u.view(np.float32).astype(np.float64)


def slices(x, k):
    """x = s_0 + s_1 + ... + s_{k-1} + remainder, each s_i a BF16 value."""
    out, r = [], np.asarray(x, dtype=np.float64)
    for _ in range(k):
        s = bf16(r)
        out.append(s)
        r = r - s
    return out


def gemm_sliced(A, B, k, fp32_acc):
    """A @ B from the slice products with i + j < k; products are exact (8-bit
    significands), accumulation in FP32 or exact (FP64)."""
    As, Bs = slices(A, k), slices(B, k)
    dt = np.float32 if fp32_acc else np.float64
    acc = np.zeros((A.shape[0], B.shape[1]), dtype=dt)
    for i in range(k):
        for j in range(k - i):
            acc += As[i].astype(dt) @ Bs[j].astype(dt)
    return acc.astype(np.float64)


def int8_slices(x, k, axis):
    """Integer slices with one shared exponent per row (axis=1) or column
    (axis=0): x = 2^e (d_0 + d_1 2^-7 + ... + d_{k-1} 2^-7(k-1)) / 127 + rem,
    every d_s an integer in [-127, 127].  Returns the digit arrays (float64
    holding integers) and the scale per row / column."""
    m = np.abs(x).max(axis=axis, keepdims=True)
    e = np.where(m > 0, np.ceil(np.log2(np.where(m > 0, m, 1.0))), 0.0)
    scale = np.exp2(e)
    r = x / scale * 127.0                     # |r| <= 127
    out = []
    for s in range(k):
        d = np.rint(r)
        out.append(d)
        r = (r - d) * 128.0
    return out, scale


def gemm_int8(A, B, k):
    """A @ B from int8 slices (shared exponent per row of A and per column of
    B): the products with i + j < k are integer GEMMs (exact: |sum| < 2^31 for
    K = 192), combined in FP64."""
    As, sa = int8_slices(A, k, axis=1)
    Bs, sb = int8_slices(B, k, axis=0)
    acc = np.zeros((A.shape[0], B.shape[1]))
    for i in range(k):
        for j in range(k - i):
            acc += (As[i] @ Bs[j]) * 2.0 ** (-7 * (i + j))   # integer-valued products, exact in FP64
    return acc * (sa / 127.0) * (sb / 127.0)


def balanced_digits(a, ndig):
    """Signed base-256 digits of the int64 array a, most significant first:
    a = sum_s d_s 256^(ndig-1-s) with every d_s in [-128, 127] (each lower digit
    the centred residue (a + 128) mod 256 - 128; the top digit what is left)."""
    out = []
    r = a.copy()
    for _ in range(ndig - 1):
        d = ((r + 128) & 255) - 128
        out.append(d)
        r = (r - d) >> 8
    out.append(r)
    return out[::-1]


def gemm_digits256(M, cols, ndig=5):
    """M @ cols in the integer-digit scheme of the tensor-core z kernels
    (coral_b200/csrc/zsplit.cu), restated exactly: per data column an exponent
    e with max|col| < 2^e, m = rint(col 2^(38-e)); matrix entries (|c| <= 2)
    mc = rint(c 2^36); both written in ndig signed base-256 digits (centred,
    so the dropped low-order products carry random signs instead of a bias);
    the digit products with i + j <= ndig - 1 summed exactly per anti-diagonal
    d; S = sum_d D_d 2^(8(ndig-1-d)) in 64-bit integers; one rounding to FP64:
    S 2^(e - 74 + 8(ndig-1))."""
    mx = np.abs(cols).max(axis=0)
    e = np.where(mx > 0, np.frexp(np.where(mx > 0, mx, 1.0))[1], 0)
    m = np.rint(cols * np.exp2(38 - e)[None, :]).astype(np.int64)
    mc = np.rint(M * 2.0 ** 36).astype(np.int64)
    top = 8 * (ndig - 1)
    dm, dx = balanced_digits(mc, ndig), balanced_digits(m, ndig)
    S = np.zeros((M.shape[0], cols.shape[1]), dtype=np.int64)
    for i in range(ndig):
        for j in range(ndig - i):
            S += (dm[i] @ dx[j]) << (top - 8 * (i + j))
    return S.astype(np.float64) * np.exp2(e - 74 + top)[None, :]


_MATS = {}


def dct_matrices(NZ, NZAA):
    """REDFT01 of the zero-padded series (NZAA x NZ) and REDFT10 truncated to NZ
    outputs (NZ x NZAA), unnormalised as FFTW's."""
    if (NZ, NZAA) not in _MATS:
        z = np.arange(NZAA)[:, None]
        n = np.arange(NZ)[None, :]
        C = np.cos(np.pi * n * (2 * z + 1) / (2.0 * NZAA))
        inv = 2.0 * C
        inv[:, 0] = 1.0
        _MATS[(NZ, NZAA)] = (inv, 2.0 * C.T)
    return _MATS[(NZ, NZAA)]


def make_transforms(k, fp32_acc=True, fp32_fft=True):
    """spec_to_phys / phys_to_spec with the z transform as a sliced contraction
    (k > 0: k BF16 slices; k < 0: -k int8 slices with exact integer
    accumulation; k = 0: the exact FP64 contraction) and the x / y FFTs in FP32
    or FP64."""
    cd = np.complex64 if fp32_fft else np.complex128
    rd = np.float32 if fp32_fft else np.float64

    def zgemm(M, cols):
        if k == "digits256":
            return gemm_digits256(M, cols)
        if k < 0:
            return gemm_int8(M, cols, -k)
        return gemm_sliced(M, cols, k, fp32_acc) if k else M @ cols


    def spec_to_phys(spec, g):
        b = sfft.ifft(spec.astype(cd), axis=1, norm="forward")
        b[:, :, 0] *= 2.0
        X = np.zeros((g.NYAA, g.NXAA // 2 + 1, g.NZ), dtype=cd)
        X[:, :g.NXH, :] = b.transpose(1, 0, 2) * 0.5
        r = sfft.irfft(X, n=g.NXAA, axis=1, norm="forward")
        inv, _ = dct_matrices(g.NZ, g.NZAA)
        ph = zgemm(inv, r.reshape(-1, g.NZ).T.astype(np.float64))
        return ph.T.reshape(g.NYAA, g.NXAA, g.NZAA)

    def phys_to_spec(phys, g):
        _, fwd = dct_matrices(g.NZ, g.NZAA)
        a = zgemm(fwd, phys.reshape(-1, g.NZAA).T).T.reshape(g.NYAA, g.NXAA, g.NZ)
        c = sfft.rfft(a.astype(rd), axis=1)[:, :g.NXH, :]
        c = np.ascontiguousarray(c.transpose(1, 0, 2))
        c[:, :, 0] *= 0.5
        s = sfft.fft(c, axis=1).astype(np.complex128)
        return s * (1.0 / (g.NXAA * g.NYAA * g.NZAA))

    return spec_to_phys, phys_to_spec


def benchmark_ic(solver, seed=2):
    """The benchmark's initial condition (bench.make_ic) on the oracle."""
    from coral_b200.initial_conditions import gauss_chebyshev_z
    g = solver.g
    rng = np.random.Generator(np.random.PCG64(seed))
    zp = gauss_chebyshev_z(g.NZAA, 0.5, 1.0)
    th = rng.uniform(-1e-3, 1e-3, size=(g.NXAA, g.NYAA, g.NZAA)) * np.sin(np.pi * zp)[None, None, :]
    mean = th.mean(axis=(0, 1))
    th -= mean[None, None, :]
    solver.set_var_from_phys(0, 4, np.ascontiguousarray(th.transpose(1, 0, 2)))
    solver.set_zero_var_from_phys(1, 0, mean)


VARIANTS = [  # (label, slices, FP32 accumulation, FP32 FFTs)
    ("3 BF16 slices, FP32 acc, FP32 FFTs", 3, True, True),
    ("3 BF16 slices, FP32 acc, FP64 FFTs", 3, True, False),
    ("exact z, FP32 FFTs", 0, True, True),
    ("2 BF16 slices, FP32 acc, FP32 FFTs", 2, True, True),
    ("3 BF16 slices, exact acc, FP64 FFTs", 3, False, False),
    ("4 BF16 slices, exact acc, FP64 FFTs", 4, False, False),
    ("5 BF16 slices, exact acc, FP64 FFTs", 5, False, False),
    ("4 int8 slices, INT32 acc, FP64 FFTs", -4, False, False),
    ("5 int8 slices, INT32 acc, FP64 FFTs", -5, False, False),
    ("6 int8 slices, INT32 acc, FP64 FFTs", -6, False, False),
    ("5 base-256 digits (zsplit.cu), FP64 FFTs", "digits256", False, False),
]


def main(NX, NZ, steps, checkpoints=(1, 10, 100)):
    from tests.problems import equations, params
    dt = 1e-6
    eq, par = equations("rbc_noslip_ra1e8"), params(NX, NX, NZ, dt=dt)

    def fresh():
        s = co.Solver(eq, par)
        benchmark_ic(s)
        return s

    keep = [c for c in checkpoints if c <= steps] or [steps]
    base, ref = fresh(), {}
    t0 = time.time()
    for i in range(1, steps + 1):
        base.step(dt)
        if i in keep:
            ref[i] = ([f.copy() for f in base.field], [z.copy() for z in base.zfield])
    print("FP64 oracle, %dx%dx%d, %d steps: %.0f s" % (NX, NX, NZ, steps, time.time() - t0), flush=True)
    s2p, p2s = co.spec_to_phys, co.phys_to_spec
    for label, k, acc32, fft32 in VARIANTS:
        co.spec_to_phys, co.phys_to_spec = make_transforms(k, acc32, fft32)
        try:
            m, out = fresh(), []
            for i in range(1, steps + 1):
                m.step(dt)
                if i in keep:
                    f, z = ref[i]
                    e = max(np.linalg.norm(m.field[j] - f[j]) / np.linalg.norm(f[j]) for j in range(len(f)))
                    ez = max(np.linalg.norm(m.zfield[j] - z[j]) / max(np.linalg.norm(z[j]), 1e-300)
                             for j in range(len(z)))
                    out.append("step %d: %.1e / %.1e" % (i, e, ez))
        finally:
            co.spec_to_phys, co.phys_to_spec = s2p, p2s
        print("%-38s kxky / mean rel L2: %s" % (label, "; ".join(out)), flush=True)


if __name__ == "__main__":
    main(int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]))
