"""The reference's benchmark 01 on the GPU: linear growth of stress-free
Rayleigh-Benard convection (Ra = 2000, Pr = 7, 96 x 96 x 24 modes, box
10 x 10 x 1, ARS_222) from its own input files (read unmodified), checked
against the analytic growth rate the benchmark compares with
(etc/benchmarks/01_Rayleigh_Benard_stressFree/linearGrowthrate_numerical_vs_analytical.py:39-62):
    s(k) = [-D2 (Pr + 1) + sqrt((Pr + 1)^2 D2^2 - 4 (Pr D2^2 - Ra Pr k^2 / D2))] / 2,
    D2 = k^2 + pi^2, over the box's wavenumbers; the kinetic energy grows at 2 max s.

Two measures, from a seeded form of the reference's default initial condition
(amplitude 1e-16, so the run stays linear for a while): the kinetic energy's
growth rate (1/E dE/dt from the Timeseries files, as the benchmark's script
computes it; it approaches 2 max s from below as the slower modes fall behind)
and the growth rate of the fastest mode's coefficients alone (every coefficient
of the (kx, ky) column that maximises s), which equals max s up to the time
discretisation's error.

usage: python -m coral_b200.benchmark01 --out DIR [--inputs DIR] [--time T] [--dt DT] [--seed S]
"""
import argparse
import json
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def analytic_growth(Ra, Pr, Lx, Ly, NX, NY):
    """(max s, kx index, ky index) over the box's wavenumbers (kx, ky >= 0)."""
    kx = 2 * math.pi / Lx * np.arange(NX // 2)
    ky = 2 * math.pi / Ly * np.arange(NY // 2)
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    k2 = KX ** 2 + KY ** 2
    D2 = k2 + math.pi ** 2
    s = 0.5 * (-D2 * (Pr + 1) + np.sqrt((Pr + 1) ** 2 * D2 ** 2 - 4 * (Pr * D2 ** 2 - Ra * Pr * k2 / D2)))
    i, j = np.unravel_index(np.argmax(s), s.shape)
    return float(s[i, j]), int(i), int(j)


def published_growth():
    """The maximum growth rate the benchmark's notebook prints
    (benchmark_01_stressfree_rayleigh_benard.ipynb:68), from the extracted
    fixture; None when the fixture is absent."""
    p = os.path.join(ROOT, "tests", "golden", "heat_equation_published.json")
    if not os.path.exists(p):
        return None
    return json.load(open(p)).get("stressfree_rb_max_growthrate")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--inputs", default=os.path.join(ROOT, "tests", "golden", "benchmark01"))
    ap.add_argument("--time", type=float, default=1.0, help="simulated time")
    ap.add_argument("--dt", type=float, default=None, help="override dt_max (the CFL rule stays)")
    ap.add_argument("--chunk", type=int, default=50)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args(argv)

    from coral_b200 import initial_conditions as ic
    from coral_b200.solver import PlaneLayer

    eq = open(os.path.join(a.inputs, "coral.equations")).read()
    lines = open(os.path.join(a.inputs, "coral.parameters.in")).read().splitlines(True)
    if a.dt is not None:
        lines[10] = "%r ! dt_max (overridden)\n" % a.dt
    pl = PlaneLayer(eq, "".join(lines))
    pl.set_timeseries(open(os.path.join(a.inputs, "coral.timeseries")).read())
    Lx = float(lines[5].split()[0].replace("d", "e"))
    Ly = float(lines[6].split()[0].replace("d", "e"))
    smax, ix, iy = analytic_growth(2000.0, 7.0, Lx, Ly, pl.NX, pl.NY)
    ic.noisy_modes(pl, Lx, Ly, amp=1e-16, amp0=1e-16, seed=a.seed)
    os.makedirs(a.out, exist_ok=True)
    times, norms = [], []
    while pl.get_time()["time"] < a.time:
        pl.run(a.chunk, a.out)
        times.append(pl.get_time()["time"])
        norms.append(float(np.linalg.norm(pl.get_field(0)[ix, iy, :])))
    t = np.array(times)
    mode_rate = np.diff(np.log(norms)) / np.diff(t)
    ts = np.fromfile(os.path.join(a.out, "Timeseries", "time.dat"))
    ke = sum(np.fromfile(os.path.join(a.out, "Timeseries", n + "_volAvg.dat")) for n in ("uu", "vv", "ww"))
    ke_rate = np.diff(np.log(ke)) / np.diff(ts)
    res = dict(case="benchmark01 stress-free RB Ra 2000 Pr 7 %dx%dx%d" % (pl.NX, pl.NY, pl.NZ),
               analytic_max_growth=smax, analytic_mode=[ix, iy],
               published_max_growth=published_growth(),
               mode_growth_last=float(mode_rate[-1]), mode_growth_rel_err=float(mode_rate[-1] / smax - 1),
               ke_growth_last=float(ke_rate[-1]), ke_growth_over_2s=float(ke_rate[-1] / (2 * smax)),
               steps=pl.get_time()["i_timestep"] - 1, time=float(t[-1]))
    print(json.dumps(res))
    with open(os.path.join(a.out, "growth.json"), "w") as f:
        json.dump(res, f, indent=1)
    pl.close()
    return res


if __name__ == "__main__":
    main()
