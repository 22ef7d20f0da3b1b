"""Mean Nusselt number from the Timeseries files of a run, by the rule of the
reference's benchmark 02 (etc/benchmarks/02_RRBC_julien_JFM96/compute_nusselt.py:7-30):

* Ttop, Tbot = horizontal averages of tFull at the first and the last z grid
  points (tFull_XYavg_z00001.dat, tFull_XYavg_z<NZAA>.dat), time = time.dat;
* dz = 1/2 - cos(pi / (2 NZAA)) / 2, the distance between a wall and its
  nearest Gauss-Chebyshev point (gap 1);
* the series is cut into four quarters; in each, the time-weighted average of
  Ttop / dz (top) and of -Tbot / dz (bottom), weights t[i+1] - t[i] paired
  with the value at t[i];
* mean = average of the six top / bottom values of quarters 2-4, spread =
  their root-mean-square deviation from that mean.

usage: python -m coral_b200.nusselt <output directory> [NZAA]
"""
import math
import os
import sys

import numpy as np


def quarters(directory, NZAA):
    ts = os.path.join(directory, "Timeseries")
    t = np.fromfile(os.path.join(ts, "time.dat"), dtype=np.float64)
    top = np.fromfile(os.path.join(ts, "tFull_XYavg_z00001.dat"), dtype=np.float64)
    bot = np.fromfile(os.path.join(ts, "tFull_XYavg_z%05d.dat" % NZAA), dtype=np.float64)
    n = min(len(t), len(top), len(bot))
    t, top, bot = t[:n], top[:n], bot[:n]
    dt = np.diff(t)
    dz = 0.5 - 0.5 * math.cos(math.pi / 2.0 / NZAA)
    q = (n - 1) // 4
    out = []
    for k in range(4):
        sl = slice(k * q, (k + 1) * q)
        w = dt[sl]
        out.append((float(np.sum(w * top[sl]) / np.sum(w) / dz), float(-np.sum(w * bot[sl]) / np.sum(w) / dz)))
    return out


def mean_nusselt(directory, NZAA=72):
    """(mean, spread, per-quarter (top, bottom) values)."""
    qs = quarters(directory, NZAA)
    vals = [v for pair in qs[1:] for v in pair]
    mean = sum(vals) / 6.0
    std = math.sqrt(sum((v - mean) ** 2 for v in vals) / 6.0)
    return mean, std, qs


if __name__ == "__main__":
    d = sys.argv[1]
    nz = int(sys.argv[2]) if len(sys.argv) > 2 else 72
    m, s, qs = mean_nusselt(d, nz)
    for k, (a, b) in enumerate(qs):
        print("quarter %d: top %.6f  bottom %.6f" % (k + 1, a, b))
    print("mean Nusselt number (quarters 2-4): %.6f  spread %.6f" % (m, s))
