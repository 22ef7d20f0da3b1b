"""The learned subgrid closure end to end, on the GPU: fine-grid Rayleigh-Benard
runs of the solver itself give the training data, the closure's own kernels
train the network, and the trained network is judged against the plain coarse
method.

Default sizes are those of the closure configuration: coarse 64^2 x 48 at
Ra = 1e7, Pr = 1, no-slip, box 2 pi x 2 pi x 1, trained on snapshots of a
256^2 x 128 run truncated to the coarse modes (coral_b200.closure.subgrid_snapshot).

  1. fine run: seeded form of the reference's default initial condition
     (amplitude --amp, small: the instability grows it; large random states of
     all six variables are far from balance and blow up), CFL-adaptive time
     loop (CFL_C 0.3, dt_max 1e-4), the
     kx = 0 line kept Hermitian; after --spinup time units one snapshot every
     --every steps;
  2. training: the first 80% of the snapshots, Adam, random batches of points;
  3. a-priori judgement on the last 20%: the error of the coarse quadratic
     variables (in the modes the coarse NL assembly uses) against the filtered
     fine ones, with and without the network (gain = 1 - err_with / err_without);
  4. a-posteriori judgement: from the last fine state truncated to the coarse
     grid, coarse runs with and without the network and the fine run advance
     the same simulated time; their time-averaged Nusselt numbers (heat flux at
     the walls from the horizontal averages of tFull, as in the benchmark's
     rule) and horizontal kinetic-energy spectra at mid-depth are compared.

usage: python -m coral_b200.closure_demo --out DIR [--fine NX NY NZ] [--coarse NX NY NZ] [--ra RA] ...
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

TS = (">>Horizontal_avg :: tFull ;; Position= 1 <<\n>>Horizontal_avg :: tFull ;; Position= %d <<\n"
      ">>Volume_average :: uu <<\n>>Volume_average :: vv <<\n>>Volume_average :: ww <<\n>>EOF<<\n")


def texts(ra, n, dt_max=1e-4, cfl=0.3):
    from coral_b200 import CONFIG_DIR
    eq = open(os.path.join(CONFIG_DIR, "rbc_noslip_ra1e5.equations")).read()
    eq = eq.replace(">>Param :: Rayleigh := 1.d5 <<", ">>Param :: Rayleigh := %r <<" % ra)
    par = open(os.path.join(CONFIG_DIR, "rbc_noslip_ra1e5_64x64x48.parameters.in")).read().splitlines(True)
    par[1], par[2], par[3] = "%d\n" % n[0], "%d\n" % n[1], "%d\n" % n[2]
    par[10], par[12] = "%r\n" % dt_max, "%r\n" % cfl
    return eq, "".join(par)


def hke_spectrum(pl):
    """Horizontal kinetic energy spectrum at mid-depth, binned by |k| (integer
    multiples of the box wavenumber), from the physical u and v."""
    z = pl.NZAA // 2
    e = np.zeros(pl.NXAA)
    for f in (0, 1):
        p = pl.full_phys(f)[:, :, z]
        s = np.abs(np.fft.rfft2(p) / p.size) ** 2
        ky = np.fft.fftfreq(p.shape[0]) * p.shape[0]
        kx = np.arange(s.shape[1])
        k = np.rint(np.sqrt(ky[:, None] ** 2 + kx[None, :] ** 2)).astype(int)
        np.add.at(e, np.minimum(k, len(e) - 1), s)
    return e


def nusselt_of(vals, dz):
    """time-weighted mean of (Ttop - Tbot) / (2 dz) over rows (t, dt, Ttop, Tbot)."""
    w = np.array([r[1] for r in vals])
    top = np.array([r[2] for r in vals])
    bot = np.array([r[3] for r in vals])
    return float(np.sum(w * (top - bot)) / np.sum(w) / (2 * dz))


def advance_recording(pl, t_span, chunk=20):
    """Advance t_span time units; rows (t, dt, Ttop, Tbot) every chunk steps."""
    rows = []
    t0 = pl.get_time()["time"]
    while pl.get_time()["time"] - t0 < t_span:
        st = pl.get_time()
        pl.run(chunk)
        v = pl.timeseries()
        rows.append((st["time"], pl.get_time()["time"] - st["time"], v[0], v[1]))
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--fine", type=int, nargs=3, default=(256, 256, 128))
    ap.add_argument("--coarse", type=int, nargs=3, default=(64, 64, 48))
    ap.add_argument("--ra", type=float, default=1e7)
    ap.add_argument("--amp", type=float, default=1e-6)
    ap.add_argument("--spinup", type=float, default=0.02)
    ap.add_argument("--snapshots", type=int, default=40)
    ap.add_argument("--every", type=int, default=40)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--judge-time", type=float, default=0.01)
    ap.add_argument("--seed", type=int, default=100)
    a = ap.parse_args(argv)

    import torch
    from coral_b200 import initial_conditions as ic
    from coral_b200.closure import Closure, detach, subgrid_snapshot, truncate
    from coral_b200.solver import PlaneLayer

    os.makedirs(a.out, exist_ok=True)
    res = {"fine": a.fine, "coarse": a.coarse, "Ra": a.ra}
    t_start = time.time()
    eqf, parf = texts(a.ra, a.fine)
    eqc, parc = texts(a.ra, a.coarse)
    fine = PlaneLayer(eqf, parf)
    coarse = PlaneLayer(eqc, parc)
    fine.set_hermitian_kx0(True)
    fine.set_timeseries(TS % fine.NZAA)
    ic.noisy_modes(fine, 2 * math.pi, 2 * math.pi, amp=a.amp, amp0=0.0, seed=a.seed)
    # 1. fine run and snapshots
    while fine.get_time()["time"] < a.spinup:
        fine.run(200)
    res["spinup_steps"] = fine.get_time()["i_timestep"] - 1
    xs, ys = [], []
    for k in range(a.snapshots):
        fine.run(a.every)
        x, y = subgrid_snapshot(fine, coarse)
        xs.append(x.astype(np.float32))
        ys.append(y.astype(np.float32))
    res["snapshot_time"] = fine.get_time()["time"]
    res["data_s"] = time.time() - t_start
    x = np.stack(xs)
    y = np.stack(ys)
    ntr = max(1, int(0.8 * len(xs)))
    # 2. training
    t0 = time.time()
    ins = 1.0 / (x[:ntr].std(axis=(0, 2, 3, 4)) + 1e-30)
    outs = y[:ntr].std(axis=(0, 2, 3, 4)) + 1e-30
    net = Closure(seed=a.seed)
    net.set_scales(ins, outs)
    dx, dy = torch.from_numpy(x[:ntr]).cuda(), torch.from_numpy(y[:ntr]).cuda()
    npoint = int(np.prod(x.shape[2:]))
    gen = torch.Generator(device="cpu").manual_seed(a.seed)
    losses = []
    for it in range(a.iters):
        lr = 1e-3 if it < 0.7 * a.iters else 3e-4
        pts = torch.randint(0, ntr * npoint, (a.batch,), generator=gen).cuda()
        losses.append(net.train(dx, dy, pts, lr=lr))
    torch.cuda.synchronize()
    res["train_s"] = time.time() - t0
    res["loss_first_last"] = [float(np.mean(losses[:10])), float(np.mean(losses[-50:]))]
    del dx, dy
    # 3. a-priori
    ew = ewo = 0.0
    per_q = np.zeros((9, 2))
    for s in range(ntr, len(xs)):
        tau = torch.zeros((9,) + x.shape[2:], dtype=torch.float64, device="cuda")
        net.infer(torch.from_numpy(x[s].astype(np.float64)).cuda(), tau)
        torch.cuda.synchronize()
        pred = tau.cpu().numpy()
        d = (y[s] - pred).reshape(9, -1)
        per_q[:, 0] += np.sum(d * d, axis=1)
        per_q[:, 1] += np.sum(y[s].astype(np.float64).reshape(9, -1) ** 2, axis=1)
    res["apriori_gain"] = float(1.0 - per_q[:, 0].sum() / per_q[:, 1].sum())
    res["apriori_gain_per_quad"] = [float(1.0 - a_ / b_) for a_, b_ in per_q]
    # 4. a-posteriori: coarse runs from the truncated fine state
    d = os.path.join(a.out, "fine_state")
    os.makedirs(d, exist_ok=True)
    fine.export_checkpoints(d)
    runs = {}
    for name in ("plain", "closure"):
        c = PlaneLayer(eqc, parc)
        c.set_hermitian_kx0(True)
        c.set_timeseries(TS % c.NZAA)
        # coupled variables: fine physical field -> fine spectrum -> coarse modes -> coarse field
        for v in range(6):
            f = np.fromfile(os.path.join(d, "QuickSave.kxky.sys001.var%03d.rolling1" % (v + 1)))
            f = np.ascontiguousarray(f.reshape(fine.NXAA, fine.NYAA, fine.NZAA).transpose(1, 0, 2))
            c.set_var_phys(0, v, c.spec_to_phys(truncate(fine.phys_to_spec(f), c)))
        for sidx, nv in ((0, 2), (1, 1)):
            for v in range(nv):
                prof = np.fromfile(os.path.join(d, "QuickSave.zero.sys%03d.var%03d.rolling1" % (sidx + 1, v + 1)))
                cheb = np.polynomial.chebyshev.chebfit(np.cos(np.pi * (2 * np.arange(1, fine.NZAA + 1) - 1) /
                                                              (2 * fine.NZAA)), prof, coarse.NZ - 1)
                zc = np.cos(np.pi * (2 * np.arange(1, c.NZAA + 1) - 1) / (2 * c.NZAA))
                c.set_mean_var_profile(sidx, v, np.polynomial.chebyshev.chebval(zc, cheb))
        c.set_time(fine.get_time()["time"], 1e-5, 1)
        if name == "closure":
            net.attach(c)
        t0 = time.time()
        rows = advance_recording(c, a.judge_time)
        dzc = 0.5 - 0.5 * math.cos(math.pi / 2 / c.NZAA)
        runs[name] = {"nusselt": nusselt_of(rows, dzc), "steps": c.get_time()["i_timestep"] - 1,
                      "wall_s": time.time() - t0, "hke_spectrum": hke_spectrum(c)[:24].tolist()}
        if name == "closure":
            detach(c)
        c.close()
    rows = advance_recording(fine, a.judge_time)
    dzf = 0.5 - 0.5 * math.cos(math.pi / 2 / fine.NZAA)
    runs["fine"] = {"nusselt": nusselt_of(rows, dzf), "hke_spectrum": hke_spectrum(fine)[:24].tolist()}
    for name in ("plain", "closure"):
        runs[name]["nusselt_err_vs_fine"] = abs(runs[name]["nusselt"] - runs["fine"]["nusselt"]) / abs(runs["fine"]["nusselt"])
        sf, sc = np.array(runs["fine"]["hke_spectrum"]), np.array(runs[name]["hke_spectrum"])
        k = slice(1, 16)
        runs[name]["spectrum_log_err_vs_fine"] = float(np.sqrt(np.mean((np.log(sc[k] + 1e-300) - np.log(sf[k] + 1e-300)) ** 2)))
    res["aposteriori"] = runs
    res["total_s"] = time.time() - t_start
    print(json.dumps(res))
    with open(os.path.join(a.out, "closure_demo.json"), "w") as f:
        json.dump(res, f, indent=1)
    net.close()


if __name__ == "__main__":
    main()
