"""Seeded initial conditions written as QuickSave files.

The reference injects initial conditions through its restart path: every
coupled variable is stored as a physical field in z-fastest, then y, then x
order in ``QuickSave.kxky.sysSSS.varVVV.rollingR`` and every mean variable as
an NZAA profile in ``QuickSave.zero.sysSSS.varVVV.rollingR``
(src/plane_layer/PL_IMEX_timestepping_output.f90:309-383), with ``dt.sav``
holding (dt, t) (src/misc/timeKeeping.f90:92-134).  The generators below write
the same files for the Rayleigh-Benard recipes of ``coral_b200/configs``
(variables u, v, w, p, t, chi in one kxky system; uMean, vMean and tMean in two
mean systems), temperature perturbations only, velocity zero.
"""
import math
import os

import numpy as np


def gauss_chebyshev_z(NZAA, center, gap):
    i = np.arange(1, NZAA + 1)
    return center + np.cos(math.pi * (2 * i - 1) / (2 * NZAA)) * 0.5 * gap


def _write(directory, NXAA, NYAA, NZAA, theta, dt, n_kxky_vars=6, t_index=5,
           zero_layout=((1, 2), (2, 1)), t_zero=(2, 1)):
    os.makedirs(directory, exist_ok=True)
    mean = theta.mean(axis=(0, 1))
    fluct = theta - mean[None, None, :]
    zero3 = np.zeros((NXAA, NYAA, NZAA))
    for v in range(1, n_kxky_vars + 1):
        a = fluct if v == t_index else zero3
        a.astype(np.float64).tofile(os.path.join(directory, "QuickSave.kxky.sys001.var%03d.rolling1" % v))
    for sysi, nvars in zero_layout:
        for v in range(1, nvars + 1):
            prof = mean if (sysi, v) == t_zero else np.zeros(NZAA)
            prof.astype(np.float64).tofile(os.path.join(directory, "QuickSave.zero.sys%03d.var%03d.rolling1" % (sysi, v)))
    np.array([dt, 0.0], dtype=np.float64).tofile(os.path.join(directory, "dt.sav"))


def white_noise_temperature(directory, NX, NY, NZ, center=0.5, gap=1.0, amplitude=1e-3, seed=0, dt=1e-4):
    """theta = U[-a, a] i.i.d. per grid point (drawn in file order: x slowest,
    z fastest) times sin(pi z'), z' = z - center + gap/2 in [0, 1]."""
    NXAA, NYAA, NZAA = 3 * NX // 2, 3 * NY // 2, 3 * NZ // 2
    rng = np.random.Generator(np.random.PCG64(seed))
    z = gauss_chebyshev_z(NZAA, center, gap)
    zp = z - center + gap / 2
    theta = rng.uniform(-amplitude, amplitude, size=(NXAA, NYAA, NZAA)) * np.sin(math.pi * zp)[None, None, :]
    _write(directory, NXAA, NYAA, NZAA, theta, dt)
    return theta


def fourier_modes_temperature(directory, NX, NY, NZ, Lx, Ly, center=0.5, gap=1.0, amplitude=1e-4, kmax=8,
                              seed=1, dt=5e-6):
    """theta = sum over integer wavevectors 0 < |k| <= kmax (units 2 pi / L) of
    a cos(kx x + ky y + phi) sin(pi z'), phi ~ U[0, 2 pi) seeded."""
    NXAA, NYAA, NZAA = 3 * NX // 2, 3 * NY // 2, 3 * NZ // 2
    rng = np.random.Generator(np.random.PCG64(seed))
    x = np.arange(NXAA) * Lx / NXAA
    y = np.arange(NYAA) * Ly / NYAA
    z = gauss_chebyshev_z(NZAA, center, gap)
    zp = z - center + gap / 2
    plane = np.zeros((NXAA, NYAA))
    for m in range(-kmax, kmax + 1):
        for n in range(-kmax, kmax + 1):
            if m * m + n * n == 0 or m * m + n * n > kmax * kmax:
                continue
            phi = rng.uniform(0.0, 2 * math.pi)
            plane += amplitude * np.cos(2 * math.pi * m / Lx * x[:, None] + 2 * math.pi * n / Ly * y[None, :] + phi)
    theta = plane[:, :, None] * np.sin(math.pi * zp)[None, None, :]
    _write(directory, NXAA, NYAA, NZAA, theta, dt)
    return theta


def noisy_modes(pl, Lx, Ly, amp=1e-16, amp0=1e-16, seed=0):
    """A seeded form of the reference's default initial condition
    (noisy_initial_conditions, src/plane_layer/PL_IMEX_timestepping.f90:425-483),
    written straight into the coupled-system states of a PlaneLayer: every
    coefficient t of every kxky system at (kx, ky) gets
        amp [exp(-(n - 3.5)^2 / 8) exp(-(|k| - 6 kx_box)^2 / 8) e^{i phi1}
             + 3 exp(-(n - 1.5)^2 / 8) exp(-(|k| - 3 kx_box)^2 / 32) e^{i phi2}],
    with phi1, phi2 uniform in [0, 2 pi) (PCG64 seed) and n = t // (coupled
    variables) the Chebyshev degree of the coefficient in the interleaved
    layout; every mean-system coefficient t gets amp0 exp(-(n - 1.5)^2 / 8) cos(t + 1).
    The reference draws its phases from an unseeded generator and uses amplitude
    1e-16 by default (its --noises-amplitude option changes it)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    kxb, kyb = 2 * math.pi / Lx, 2 * math.pi / Ly
    kx = np.arange(pl.NXH) * kxb
    iy = np.arange(pl.NYAA)
    ky = np.where(iy <= pl.NYAA // 2, iy, iy - pl.NYAA) * kyb
    kk = np.sqrt(kx[:, None] ** 2 + ky[None, :] ** 2)
    for s in range(pl.n_kxky):
        T = pl.T[s]
        nv = pl.query(300 + s)
        n = (np.arange(T) // nv).astype(np.float64)
        e1 = np.exp(-(n - 3.5) ** 2 / 8.0)[None, None, :] * np.exp(-(kk - 6 * kxb) ** 2 / 8.0)[:, :, None]
        e2 = np.exp(-(n - 1.5) ** 2 / 8.0)[None, None, :] * np.exp(-(kk - 3 * kxb) ** 2 / 32.0)[:, :, None]
        p1 = rng.uniform(0.0, 2 * math.pi, size=(pl.NXH, pl.NYAA, T))
        p2 = rng.uniform(0.0, 2 * math.pi, size=(pl.NXH, pl.NYAA, T))
        pl.set_field(s, amp * (e1 * np.exp(1j * p1) + 3.0 * e2 * np.exp(1j * p2)))
    for s in range(pl.n_zero):
        T = pl.Tz[s]
        nv = pl.query(400 + s)
        t = np.arange(T)
        n = (t // nv).astype(np.float64)
        pl.set_mean_field(s, amp0 * np.exp(-(n - 1.5) ** 2 / 8.0) * np.cos(t + 1.0))
