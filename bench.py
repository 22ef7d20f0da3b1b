"""Benchmark of the plane-layer IMEX timestep on B200.

Workload (the headline configuration): Rayleigh-Benard convection, no-slip,
Ra = 1e8, Pr = 1, NX = NY = 384 Fourier x NZ = 192 Chebyshev modes (grid
576 x 576 x 288), ARS_222, dt = 1e-6, FP64 path; seeded white-noise temperature
initial condition (amplitude 1e-3, PCG64 seed 2) injected through the QuickSave
projection.  A "step" is one full IMEX timestep of the whole domain.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config NAME]

N > 1 runs N independent replicas (one process per GPU under torchrun): the
timestep does not shard across GPUs at this size (replicas only).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "rbc_384x384x192": dict(eq="rbc_noslip_ra1e8.equations", par="rbc_noslip_ra1e8_384x384x192.parameters.in",
                            NX=384, NY=384, NZ=192, dt=1e-6, seed=2, Ra=1e8),
    "rbc_64x64x48": dict(eq="rbc_noslip_ra1e5.equations", par="rbc_noslip_ra1e5_64x64x48.parameters.in",
                         NX=64, NY=64, NZ=48, dt=1e-4, seed=0, Ra=1e5),
    "rbc_96x96x192": dict(eq="rbc_noslip_ra1e8.equations", par="rbc_noslip_ra1e8_96x96x192.parameters.in",
                          NX=96, NY=96, NZ=192, dt=1e-6, seed=2, Ra=1e8),
    "rbc_128x128x192": dict(eq="rbc_noslip_ra1e8.equations", par="rbc_noslip_ra1e8_128x128x192.parameters.in",
                            NX=128, NY=128, NZ=192, dt=1e-6, seed=2, Ra=1e8),
    "rbc_192x192x192": dict(eq="rbc_noslip_ra1e8.equations", par="rbc_noslip_ra1e8_192x192x192.parameters.in",
                            NX=192, NY=192, NZ=192, dt=1e-6, seed=2, Ra=1e8),
    "rbc_32x32x192": dict(eq="rbc_noslip_ra1e8.equations", par="rbc_noslip_ra1e8_32x32x192.parameters.in",
                          NX=32, NY=32, NZ=192, dt=1e-6, seed=2, Ra=1e8),
    "rrbc_192x192x96": dict(eq="rrbc_stressfree_ek1e-4_ra5e7.equations", par="rrbc_stressfree_192x192x96.parameters.in",
                            NX=192, NY=192, NZ=96, dt=5e-6, seed=1, Ra=5e7),
    # the benchmark recipe with a penalised velocity (a mask field GAMMA, drag
    # - GAMMA u) and with the horizontal Smagorinsky viscosity: the cost of those
    # paths at full size
    "rbc_penalised_384x384x192": dict(eq="rbc_penalised_ra1e8.equations",
                                      par="rbc_noslip_ra1e8_384x384x192.parameters.in",
                                      NX=384, NY=384, NZ=192, dt=1e-6, seed=2, Ra=1e8),
    "rbc_smagorinsky_384x384x192": dict(eq="rbc_smagorinsky_ra1e8.equations",
                                        par="rbc_noslip_ra1e8_384x384x192.parameters.in",
                                        NX=384, NY=384, NZ=192, dt=1e-6, seed=2, Ra=1e8,
                                        args="--withHorizontalSmagorinsky --smagorinsky-prefactor 0.1"),
}
METRIC = "timesteps/s at 384\u00b2\u00d7192 (FP64 vs split-prec TC) at stated err vs FP64 oracle"
PHASES = ("inv_y", "inv_x", "inv_z", "z_products", "fwd_x", "fwd_y", "nl_assembly", "rhs_nl", "mean_systems",
          "substitution", "kstd_out")


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x, device):
    """Max of a float over all ranks of the process group (a tensor on `device`:
    the rank's GPU under NCCL, "cpu" under gloo)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        # nvidia-smi numbers GPUs physically, CUDA after CUDA_VISIBLE_DEVICES
        # remapping: select the timed GPU by its UUID (read-only query)
        self.index = str(index)
        try:
            import torch
            u = str(torch.cuda.get_device_properties(index).uuid)
            self.index = u if u.startswith("GPU-") else "GPU-" + u
        except Exception:
            pass
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.index, "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_ic(cfg, pl):
    """Seeded white-noise temperature (coral_b200.initial_conditions) projected
    into the state: fluctuation into the kxky variable t, horizontal mean into tMean."""
    from coral_b200.initial_conditions import gauss_chebyshev_z
    NXAA, NYAA, NZAA = pl.NXAA, pl.NYAA, pl.NZAA
    rng = np.random.Generator(np.random.PCG64(cfg["seed"]))
    zp = gauss_chebyshev_z(NZAA, 0.5, 1.0)
    theta = rng.uniform(-1e-3, 1e-3, size=(NXAA, NYAA, NZAA))  # file order: x, y, z
    theta *= np.sin(math.pi * zp)[None, None, :]
    mean = theta.mean(axis=(0, 1))
    theta -= mean[None, None, :]
    phys = np.ascontiguousarray(theta.transpose(1, 0, 2))  # (y, x, z)
    del theta
    pl.set_var_phys(0, 4, phys)  # t is the 5th coupled variable (u, v, w, p, t, chi)
    pl.set_mean_var_profile(1, 0, mean)


# kernels of each timed phase (names as ncu lists them)
PHASE_KERNELS = {
    "inv_y": "k_inv_y1", "inv_x": "k_inv_x", "inv_z": "k_inv_z", "z_products": "k_z_fused",
    "fwd_x": "k_fwd_x", "fwd_y": "k_fwd_y_pipe", "nl_assembly": "k_nl",
    "rhs_nl": "k_rhs_tiles", "mean_systems": "k_zero_step", "substitution": "k_subst_tpb", "kstd_out": "k_kstd_tiles",
}


def phase_bytes(g, nsys, nact, T, ncls, Tc, kl, ku, stages, factor_bytes, factor_entries=0):
    """Algorithmic HBM bytes of one launch of each phase (averaged over the
    stages): every array a phase must read from or write to HBM once.
    g: dict with NXH, NYA, NXA, NZ, NZA, nF (full variables), nQ (quadratic
    variables).  Transform intermediates are 16-byte complex where the data are
    complex (after an x r2c / before an x c2r) and 8-byte real otherwise.
    factor_entries: LU band entries per block that the substitution reads (the
    entries nonzero in some block; 0 = the whole band, 2 kl + ku + 1 per column)."""
    NXH, NYA, NXA, NZ, NZA, nF, nQ = (g[k] for k in ("NXH", "NYA", "NXA", "NZ", "NZA", "nF", "nQ"))
    y1 = lambda nv: nv * NYA * NXH * NZ * 16   # [var][y][kx][n] complex
    y2 = lambda nv: nv * NYA * NXA * NZ * 8    # [var][y][x][n] real
    ph = lambda nv: nv * NYA * NXA * NZA * 8   # [var][y][x][z] real
    out = {
        # the Chebyshev coefficients of each full variable from the state, Y1 out
        "inv_y": nsys * nF * NZ * 16 + y1(nF),
        "inv_x": y1(nF) + y2(nF),
        # the z passes are fused: Y2 of the full variables in, Y2 of the quadratic
        # variables out; the physical fields stay in shared memory
        "inv_z": 0,
        "z_products": y2(nF) + y2(nQ),
        "fwd_x": y2(nQ) + y1(nQ),
        "fwd_y": y1(nQ) + y1(nQ),
    }
    # the solve, kernel by kernel, averaged over the stages (stage i reads the
    # K arrays of the i earlier stages; the last stage writes no K_std):
    #   rhs_nl: state, K arrays and quadratic coefficients in, K_hat and the
    #     right-hand side (inactive systems: the stage output) out
    #   substitution: LU factors (the band entries that are nonzero in some
    #     block, or all 2 kl + ku + 1 per column, and one pivot byte per column of
    #     each block) and the block vectors (right-hand side in, intermediate out
    #     and in, solution out)
    #   kstd_out: split systems: the solution (already in the stage output) in,
    #     K_std out, in every stage but the last (which needs no K_std);
    #     whole systems: solution in, stage output and K_std out
    rhs = sub = kst = 0
    nblk_cols = nact * ncls * Tc
    for i in range(stages):
        last = (i == stages - 1)
        rhs += (nsys * 16 * T * (1 + 2 * i + (0 if last else 1) + 1) + nact * 16 * nQ * NZ
                + (nsys - nact) * 16 * T * (0 if last else 1))
        entries = factor_entries * nact * ncls if factor_entries else nblk_cols * (2 * kl + ku + 1)
        sub += entries * factor_bytes + nblk_cols + 4 * 16 * nblk_cols
        kst += 16 * nblk_cols + nact * 16 * T * (1 if last else 2)
    out["rhs_nl"] = rhs / stages
    out["substitution"] = sub / stages
    out["kstd_out"] = (2 * nact * 16 * T) if ncls == 2 else kst / stages
    return out


def phase_launches(stages, ncls):
    """Launches per step of each phase's kernel: one per stage, except the split
    systems' K_std kernel, which the last stage skips."""
    n = {k: stages for k in PHASE_KERNELS}
    if ncls == 2:
        n["kstd_out"] = max(stages - 1, 1)
    return n


def save_state(pl):
    return ([pl.get_field(s) for s in range(pl.n_kxky)], [pl.get_mean_field(s) for s in range(pl.n_zero)])


def load_state(pl, st):
    for s, f in enumerate(st[0]):
        pl.set_field(s, f)
    for s, z in enumerate(st[1]):
        pl.set_mean_field(s, z)


def field_errors(pl, got, ref):
    """Relative L2 difference per coupled variable (kxky system 0) and per mean system."""
    out = {}
    names = ("u", "v", "w", "p", "t", "chi")
    for v in range(pl.query(300)):
        pos = pl.var_positions(0, v)
        a, b = got[0][0][..., pos], ref[0][0][..., pos]
        out[names[v] if v < len(names) else "var%d" % v] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    for s in range(len(ref[1])):
        out["mean_system%d" % s] = float(np.linalg.norm(got[1][s] - ref[1][s]) / max(np.linalg.norm(ref[1][s]), 1e-300))
    return out


def measure_int8_peak(dev):
    """Dense int8 tensor-core throughput of this GPU, measured with the library
    int8 GEMM (torch._int_mm, 8192^3, best of 5); None if unavailable."""
    import torch
    try:
        n = 8192
        a = torch.randint(-100, 100, (n, n), dtype=torch.int8, device=dev)
        b = torch.randint(-100, 100, (n, n), dtype=torch.int8, device=dev)
        for _ in range(2):
            torch._int_mm(a, b)
        best = None
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize(dev)
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None else min(best, t)
        del a, b
        return 2.0 * n ** 3 / best / 1e12
    except Exception:
        return None


def split_leg(pl, dt, args, dev, stream, s0, nerr=100):
    """The split-precision form (int8-digit tensor-core z transforms) on the same
    handle: timed steps, per-phase times, and the per-field error against the
    FP64 form after nerr steps from the same initial state (the FP64 form
    matches the oracle to 1e-10 after 100 steps; tests/test_gpu_parity*.py)."""
    import torch
    load_state(pl, s0)
    pl.set_z_transform(1)
    pl.march_forward(dt, args.warmup)
    pl.synchronize()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pl.march_forward(dt, args.steps)
    e1.record(stream)
    pl.synchronize()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    prof = {k: 0.0 for k in PHASES}
    for _ in range(2):
        p = pl.profile_step(dt)
        for k in PHASES:
            prof[k] += p[k] / 2
    # error after nerr steps from s0: FP64 form, then split form
    pl.set_z_transform(0)
    load_state(pl, s0)
    pl.march_forward(dt, nerr)
    ref = save_state(pl)
    pl.set_z_transform(1)
    load_state(pl, s0)
    pl.march_forward(dt, nerr)
    got = save_state(pl)
    pl.synchronize()
    errs = field_errors(pl, got, ref)
    pl.set_z_transform(0)
    return ms, prof, errs


def run_ours(args, cfg):
    import torch
    import torch.distributed as dist
    from coral_b200 import CONFIG_DIR
    from coral_b200.solver import PlaneLayer

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = local
    torch.cuda.set_device(dev)
    eq = open(os.path.join(CONFIG_DIR, cfg["eq"])).read()
    par = open(os.path.join(CONFIG_DIR, cfg["par"])).read()
    pl = PlaneLayer(eq, par, device=dev, args=cfg.get("args"))
    for v in args.variant:
        knob, val = v.split("=")
        pl.set_variant(knob, int(val))
    make_ic(cfg, pl)
    dt = cfg["dt"]
    s0 = save_state(pl)
    t0 = time.perf_counter()
    pl.factorize_operators(dt)
    pl.synchronize()
    t_factor = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(pl.stream, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up (also captures the CUDA graph of one step)
    pl.march_forward(dt, args.warmup)
    pl.synchronize()
    launches0 = pl.kernel_launches
    barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        e0.record(stream)
        pl.march_forward(dt, args.steps)
        e1.record(stream)
        pl.synchronize()
        torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    barrier()
    gpu_launches = pl.kernel_launches - launches0
    if world > 1:
        ms = max_over_ranks(ms, f"cuda:{dev}")
    ms_per_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)
    diag = pl.diagnostics()

    # per-kernel times with events on the launching stream (eager steps)
    prof = {k: 0.0 for k in PHASES}
    nprof = 2
    for _ in range(nprof):
        p = pl.profile_step(dt)
        for k in PHASES:
            prof[k] += p[k] / nprof
    pl.synchronize()

    # end to end through the C-ABI with host buffers: the state goes host -> device,
    # every step the driver reads back its diagnostics (CFL dt, KE), and the final
    # state comes back to the host (both state buffers page-locked)
    field = pl.get_field(0)
    zf = [pl.get_mean_field(s) for s in range(pl.n_zero)]
    pin = torch.empty(field.size * 2, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128).reshape(field.shape)
    pin[...] = field
    pin_out = torch.empty(field.size * 2, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128).reshape(field.shape)
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    pl.set_field(0, pin)
    for s in range(pl.n_zero):
        pl.set_mean_field(s, zf[s])
    for _ in range(args.steps):
        pl.march_forward(dt, 1)
        pl.diagnostics()
    out = pl.get_field(0, out=pin_out)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        e2e_s = max_over_ranks(e2e_s, f"cuda:{dev}")
    del out
    state_bytes = field.nbytes + sum(z.nbytes for z in zf)
    diag_bytes = 3 * 8 + 8 + 4  # CFL maxima, KE total, non-finite flag
    e2e = {"value": world * args.steps / e2e_s, "unit": "timesteps/s",
           "h2d_bytes_per_step": state_bytes / args.steps,
           "d2h_bytes_per_step": state_bytes / args.steps + diag_bytes,
           "copies": ("the state (%.2f GB) host->device from page-locked memory before the first step and "
                      "device->host after the last, amortised over the %d steps (a driver that keeps the state "
                      "resident, as Coral's does); the CFL/KE diagnostics (%d bytes) device->host every step"
                      % (state_bytes / 1e9, args.steps, diag_bytes))}

    # the split-precision form on the same handle and initial state
    split = None
    if not args.no_split:
        try:
            sms, sprof, serr = split_leg(pl, dt, args, dev, stream, s0)
        except Exception as ex:  # e.g. a grid the tensor-core form does not support
            split = {"unavailable": str(ex)}
        else:
            ncol = pl.NXAA * pl.NYAA
            nF_, nQ_ = pl.query(8), pl.query(9)
            macs = 15 * (nF_ + nQ_) * pl.NZ * pl.NZAA * ncol * pl.stages  # executed int8 MACs per step
            zms = sprof["z_products"]
            i8 = measure_int8_peak(dev)
            split = {"form": "z transforms as tcgen05.mma kind::i8 contractions, 5 signed base-256 digits per operand "
                             "(15 digit products), exact INT32 accumulation, one FP64 rounding; x/y FFTs, band "
                             "solves and stage sums FP64",
                     "value": world * 1e3 / sms, "unit": "timesteps/s", "ms_per_step": sms,
                     "ratio_vs_fp64": ms_per_step / sms,
                     "err_vs_fp64_form_after_100_steps": serr,
                     "max_err": max(serr.values()),
                     "phase_ms_per_step": {k: round(v, 4) for k, v in sprof.items()},
                     "tensor_roofline": {"bound": "tensor", "kernels": "k_zsplit<false> + k_zsplit<true>",
                                         "executed_int8_ops_per_step": 2 * macs,
                                         "algorithmic_flops_per_step": 2 * (nF_ + nQ_) * pl.NZ * pl.NZAA * ncol * pl.stages,
                                         "z_phase_ms_per_step": zms,
                                         "achieved_tops": 2 * macs / (zms / 1e3) / 1e12 if zms > 0 else None,
                                         "peak_tops": i8, "peak_source": "measured (torch._int_mm, int8 dense 8192^3)",
                                         "frac": (2 * macs / (zms / 1e3) / 1e12) / i8 if (i8 and zms > 0) else None}}

    # roofline of every phase; the headline one is the phase with the largest time
    T = pl.T[0]
    nsys = pl.NXH * pl.NYAA
    nact = sum(1 for ix in range(pl.NXH) for iy in range(pl.NYAA)
               if not (iy_dealiased(iy, pl.NY, pl.NYAA)) and not (ix == 0 and iy == 0))
    fbytes = 8 if pl.query(700) else 16
    ncls, Tc, kl_c, ku_c = pl.query(800), pl.query(900), pl.query(1000), pl.query(1100)
    geo = {"NXH": pl.NXH, "NYA": pl.NYAA, "NXA": pl.NXAA, "NZ": pl.NZ, "NZA": pl.NZAA,
           "nF": pl.query(8), "nQ": pl.query(9)}
    fentries = pl.query(1200)  # after the factorisation of the timed steps
    pbytes = phase_bytes(geo, nsys, nact, T, ncls, Tc, kl_c, ku_c, pl.stages, fbytes, fentries)
    peak, src = read_peaks()
    phases = {}
    nlaunch = phase_launches(pl.stages, ncls)
    for k, b in pbytes.items():
        if prof[k] <= 0:
            continue
        launch_ms = prof[k] / nlaunch[k]
        gbs = b / (launch_ms / 1e3) / 1e9 if launch_ms > 0 else None
        phases[k] = {"kernels": PHASE_KERNELS[k], "ms_per_launch": round(launch_ms, 4),
                     "algorithmic_bytes": b, "achieved_gbs": round(gbs, 1) if gbs else None,
                     "frac": round(gbs / peak, 4) if gbs else None}
    top = max(pbytes, key=lambda k: prof[k])
    launch_ms = prof[top] / nlaunch[top]
    achieved = pbytes[top] / (launch_ms / 1e3) / 1e9
    traffic = read_traffic(PHASE_KERNELS[top])
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(cfg, eq, par, pl=pl)
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded white-noise temperature IC, PCG64 seed %d)" % cfg["seed"],
        "config": workload_config(args, cfg, pl.NX, pl.NY, pl.NZ, world),
        "layout": {"systems": nsys, "active_systems": nact, "T": T, "band": [pl.query(500), pl.query(600)],
                   "blocks": ncls, "block_T": Tc, "block_band": [kl_c, ku_c],
                   "lu_factors": ("real-scaled" if fbytes == 8 else "complex")
                                 + (", split into %d independent blocks per system" % ncls if ncls > 1 else ""),
                   "lu_factor_gb": nact * ncls * Tc * (2 * kl_c + ku_c + 1) * fbytes / 1e9},
        "grid_point_steps_per_s": value * pl.NXAA * pl.NYAA * pl.NZAA,
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "phase_ms_per_step": {k: round(v, 4) for k, v in prof.items()},
        "factorize_s": t_factor,
        "roofline": {"kernel": PHASE_KERNELS[top], "phase": top, "bound": "hbm", "achieved": achieved,
                     "peak": peak, "peak_source": src, "unit": "GB/s", "frac": achieved / peak,
                     "algorithmic_bytes_per_launch": pbytes[top], "launch_ms": launch_ms,
                     "traffic": traffic, "phases": phases},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "state_ok": not diag["nonfinite"],
        "variants": dict(v.split("=") for v in args.variant),
        "split": split,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    pl.close()
    if world > 1:
        dist.destroy_process_group()


def iy_dealiased(iy, NY, NYAA):
    """ky of FFT index iy is dealiased when |ky| >= NY/2 (PL_geometry.f90:181-198)."""
    k = -(NYAA - iy) if iy + 1 >= NYAA // 2 + 1 else iy
    return abs(k) >= NY / 2


def read_traffic(kernels):
    """DRAM bytes (read + write) per launch of the phase's kernel at 384^2 x 192,
    from the one-kernel ncu captures at 128^2 x 192 summarised in profiles/
    (scaled by the units processed), or None."""
    p = os.path.join(ROOT, "profiles", "dram_traffic_rbc_128x128x192.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if "=" in line and line.split("=")[0].strip() == kernels:
            return float(line.split("=")[1])
    return None


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(cfg, eq, par, pl=None):
    """The oracle timed on one bounded sample of the workload (OracleSample),
    and, as the checker of the GPU's FP64 transforms, the oracle's transforms
    compared with the GPU's on the same random input at full size."""
    from oracle import coral_oracle as co
    import scipy.fft as sfft
    procs = host_threads()
    t0 = time.perf_counter()
    smp = OracleSample(cfg, eq, par, procs)
    sec, desc = smp.step_seconds()
    check = None
    if pl is not None:
        g = smp.g
        rng = np.random.default_rng(5)
        spec = rng.standard_normal((g.NXH, g.NYAA, g.NZ)) + 1j * rng.standard_normal((g.NXH, g.NYAA, g.NZ))
        with sfft.set_workers(procs):
            ph = co.spec_to_phys(spec, g)
            sp2 = co.phys_to_spec(ph * ph, g)
        gp = pl.spec_to_phys(spec)
        gs = pl.phys_to_spec(ph * ph)
        check = {"spec_to_phys_max_err_over_max": float(np.abs(gp - ph).max() / np.abs(ph).max()),
                 "phys_to_spec_max_err_over_max": float(np.abs(gs - sp2).max() / np.abs(sp2).max())}
    return {"value": 1.0 / sec, "unit": "timesteps/s", "cores": procs, "kind": "port", "sample": desc,
            "seconds_per_step": sec, "sample_wall_s": time.perf_counter() - t0,
            "fp64_transforms_vs_oracle": check}


class OracleSample:
    """The oracle (the CPU restatement of the reference's timestep, numpy/scipy
    FP64) timed on the workload, for the reference arm and the CPU baseline.

    Small workloads (all (kx,ky) systems solvable in seconds) run whole oracle
    steps.  At larger sizes a step is measured component by component on a
    bounded sample -- every phase of one_step_beyond
    (src/plane_layer/PL_IMEX_timestepping_marching.f90:3-48) is timed, none is
    left out -- and the step time is the sum of the phases scaled by how often
    each occurs in a step:
      inverse 3-D transforms (nF per stage) and forward transforms with the
      pointwise products (nQ per stage), at full size (scipy workers);
      NL assembly (every NL term's truncated I^Iz M^mz contraction and
      Fourier factors), stage right-hand sides (M field + the stage sums of
      K_std and K_hat), K_std = L aux and the band solves (zgbtrs) on a sample
      of kx slabs / systems of at least 1% of the systems, scaled to all."""

    def __init__(self, cfg, eq, par, processes, seed=0):
        from oracle import coral_oracle as co
        import scipy.linalg.lapack as lapack
        self.co = co
        self.processes = processes
        self.cfg = cfg
        t0 = time.perf_counter()
        p = co.read_parameters_text(par)
        g = co.Geometry(p["NX"], p["NY"], p["NZ"], p["Lx"], p["Ly"], p["gap"], p["center"])
        self.g = g
        self.whole = g.NXH * g.NYAA <= 4096
        smago = "--withHorizontalSmagorinsky" in (cfg.get("args") or "")
        if self.whole:
            self.solver = co.Solver(eq, par, smagorinsky=smago)
            self.solver.factorize(cfg["dt"])
            rng = np.random.default_rng(seed)
            for sidx, lay in enumerate(self.solver.lay):
                self.solver.field[sidx] = 1e-3 * (rng.standard_normal(self.solver.field[sidx].shape)
                                                  + 1j * rng.standard_normal(self.solver.field[sidx].shape))
            self.setup_s = time.perf_counter() - t0
            return
        s = co.Solver.__new__(co.Solver)
        s.recipe = co.parse_equations(eq, smago)
        s.params = p
        s.g = g
        s.scheme = p["scheme"]
        s.nstages, s.A, s.Ah = co.ars_tableau(s.scheme)
        self.s = s
        rec = s.recipe.kxky[0]
        lay = co.SystemLayout(g.NZ, rec)
        self.lay, self.rec = lay, rec
        cache = {}
        self.mass = [(pc, co.build_piece_matrix(g.NZ, g.center, g.gap, lay, rec, pc, cache)) for pc in rec.mass]
        self.stif = [(pc, co.build_piece_matrix(g.NZ, g.center, g.gap, lay, rec, pc, cache)) for pc in rec.stif]
        self.nF, self.nQ = len(s.recipe.full_vars), len(s.recipe.quad_vars)
        self.T = lay.T
        kl = ku = 0
        for _, B in self.mass + self.stif:
            c = B.tocoo()
            kl = max(kl, int((c.row - c.col).max()))
            ku = max(ku, int((c.col - c.row).max()))
        self.kl, self.ku = kl, ku
        self.nsys = g.NXH * g.NYAA
        self.nact = int(g.active.sum())
        # sample of >= 1% of the active systems, factorised once (the factorisation
        # is not part of a step)
        act = np.argwhere(g.active)
        nsample = max(1, int(math.ceil(0.01 * self.nact)))
        pick = act[np.linspace(0, len(act) - 1, nsample).astype(int)]
        self.facs = []
        for ix, iy in pick:
            M = sum((pc.dsca * co.complex_pow(complex(g.py[iy]), pc.ky) * co.complex_pow(complex(g.px[ix]), pc.kx)) * B
                    for pc, B in self.mass)
            L = sum((pc.dsca * co.complex_pow(complex(g.py[iy]), pc.ky) * co.complex_pow(complex(g.px[ix]), pc.kx)) * B
                    for pc, B in self.stif)
            E = (M - cfg["dt"] * s.A[0, 0] * L).tocoo()
            ab = np.zeros((2 * kl + ku + 1, self.T), dtype=np.complex128)
            ab[kl + ku + E.row - E.col, E.col] = E.data
            lu, piv, info = lapack.zgbtrf(ab, kl, ku)
            self.facs.append((lu, piv))
        # kx slabs of the operator sample: >= 1% of the systems
        self.nslab = max(1, int(math.ceil(0.01 * g.NXH)))
        self.im = {}
        for t in rec.nl:
            key = (t.Iz, t.mz)
            if key not in self.im:
                self.im[key] = co.cheb_IM(g.NZ, g.center, g.gap, t.Iz, t.mz)
        self.setup_s = time.perf_counter() - t0

    def step_seconds(self):
        """One sample; returns (seconds per step, description)."""
        co, g = self.co, self.g
        if self.whole:
            t0 = time.perf_counter()
            self.solver.step(self.cfg["dt"])
            dt = time.perf_counter() - t0
            return dt, ("whole oracle timesteps (numpy/scipy FP64) at %dx%dx%d: all %d (kx,ky) systems, every phase"
                        % (g.NX, g.NY, g.NZ, g.NXH * g.NYAA))
        import scipy.fft as sfft
        import scipy.linalg.lapack as lapack
        rng = np.random.default_rng(1)
        s, lay = self.s, self.lay
        # (1) transforms and products at full size
        spec = rng.standard_normal((g.NXH, g.NYAA, g.NZ)) + 1j * rng.standard_normal((g.NXH, g.NYAA, g.NZ))
        with sfft.set_workers(self.processes):
            t0 = time.perf_counter()
            ph = co.spec_to_phys(spec, g)
            t_inv = time.perf_counter() - t0
            t0 = time.perf_counter()
            q = ph * ph
            co.phys_to_spec(q, g)
            t_fwd = time.perf_counter() - t0
        del ph, q
        # (2) NL assembly, stage right-hand side, K_std on nslab kx slabs
        ns = self.nslab
        qspec = spec[:ns]
        state = (rng.standard_normal((ns, g.NYAA, self.T)) + 1j * rng.standard_normal((ns, g.NYAA, self.T)))
        Ks = [state.copy() for _ in range(2)]
        t0 = time.perf_counter()
        K = np.zeros_like(state)
        for t in self.rec.nl:
            fx = np.array([co.complex_pow(complex(p_), t.dx) for p_ in g.px[:ns]])
            fy = np.array([co.complex_pow(complex(p_), t.dy) for p_ in g.py])
            buf = (t.dsca * fx[:, None] * fy[None, :])[:, :, None] * qspec
            trunc = self.im[(t.Iz, t.mz)][self.rec.orders[t.eqn]:, :]
            K[:, :, lay.eq_pos[t.eqn]] += buf @ trunc.T
        t_nl = time.perf_counter() - t0
        t0 = time.perf_counter()
        X = state.reshape(-1, self.T)
        rhs = np.zeros_like(X)
        for pc, B in self.mass:
            rhs += (B @ X.T).T
        rhs += 0.5 * Ks[0].reshape(-1, self.T) + 0.5 * Ks[1].reshape(-1, self.T) + 0.5 * K.reshape(-1, self.T)
        t_rhs = time.perf_counter() - t0
        t0 = time.perf_counter()
        Y = np.zeros_like(X)
        for pc, B in self.stif:
            Y += (B @ X.T).T
        t_kstd = time.perf_counter() - t0
        # (3) band solves on the factorised sample
        b = rng.standard_normal(self.T) + 1j * rng.standard_normal(self.T)
        t0 = time.perf_counter()
        for lu, piv in self.facs:
            lapack.zgbtrs(lu, self.kl, self.ku, b, piv)
        t_solve = (time.perf_counter() - t0) / len(self.facs)
        per_slab = (t_nl + t_rhs + t_kstd) / ns
        stage = self.nF * t_inv + self.nQ * t_fwd + g.NXH * per_slab + self.nact * t_solve
        step = s.nstages * stage
        desc = ("oracle (numpy/scipy FP64, %d host threads for the FFTs) at %dx%dx%d, every phase of a step timed: "
                "1 inverse + 1 forward transform with a product at full size (x %d / %d per stage), NL assembly "
                "(%d terms), stage right-hand side and K_std on %d of %d kx slabs (%.1f%% of the systems), zgbtrs on "
                "%d of %d active systems (%.1f%%); scaled to %d stages"
                % (self.processes, g.NX, g.NY, g.NZ, self.nF, self.nQ, len(self.rec.nl), ns, g.NXH,
                   100.0 * ns / g.NXH, len(self.facs), self.nact, 100.0 * len(self.facs) / self.nact, s.nstages))
        return step, desc


def workload_config(args, cfg, NX, NY, NZ, world):
    """The workload description shared by both arms."""
    return {"workload": "%s: RBC no-slip Ra=%g Pr=1, %dx%dx%d modes, grid %dx%dx%d, ARS_222, dt=%g, FP64 state"
                        % (args.config, cfg["Ra"], NX, NY, NZ, 3 * NX // 2, 3 * NY // 2, 3 * NZ // 2, cfg["dt"]),
            "grid_points": (3 * NX // 2) * (3 * NY // 2) * (3 * NZ // 2),
            "l2": "inputs larger than L2 at 384^2x192 (state 2.02 GB, LU factors 22.2 GB)",
            "parallelism": "replicas x%d" % world}


def run_reference(args, cfg):
    """The reference arm: the reference itself cannot be built here (Fortran
    2003 + MPI + FFTW3 + MKL, none installed), so its CPU restatement (the
    oracle) is timed on the host cores (OracleSample: whole steps where they
    take seconds, otherwise every phase of a step on a bounded sample)."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    from coral_b200 import CONFIG_DIR
    eq = open(os.path.join(CONFIG_DIR, cfg["eq"])).read()
    par = open(os.path.join(CONFIG_DIR, cfg["par"])).read()
    procs = host_threads()
    smp = OracleSample(cfg, eq, par, procs)
    vals = []
    desc = ""
    for i in range(args.warmup + args.steps):
        t, desc = smp.step_seconds()
        if i >= args.warmup:
            vals.append(t)
    sec = statistics.median(vals)
    v = 1.0 / sec
    r = {"value": v, "unit": "timesteps/s", "cores": procs, "kind": "port", "sample": desc,
         "seconds_per_step": sec, "setup_s": smp.setup_s}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "timesteps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, cfg, cfg["NX"], cfg["NY"], cfg["NZ"], world), "cpu_baseline": r,
            "e2e": {"value": v, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ensemble(args):
    """The seeded 64-member ensemble (coral_b200.ensemble.seeded_ensemble: grids
    32^2x32 ... 128^2x64, Ra log-uniform in [1e4, 1e6], Pr in [0.7, 7], dt 1e-4):
    member-timesteps/s of the whole ensemble, one CUDA graph per ensemble step,
    the band substitutions of all members in one persistent launch per stage."""
    import torch
    from coral_b200.ensemble import seeded_ensemble
    dev = 0
    torch.cuda.set_device(dev)
    ens, spec = seeded_ensemble(64)
    dt = 1e-4
    ens.march_forward(dt, args.warmup)
    ens.synchronize()
    stream = torch.cuda.ExternalStream(ens.members[0].stream, device=dev)
    l0 = ens.query(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        e0.record(stream)
        ens.march_forward(dt, args.steps)
        e1.record(stream)
        ens.synchronize()
        torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    pts = sum((3 * g[0] // 2) * (3 * g[1] // 2) * (3 * g[2] // 2) for _, _, g, _, _ in spec)
    line = {"metric": "member-timesteps/s, 64-member seeded Rayleigh-Benard ensemble in one graph",
            "value": 64 * 1e3 / ms, "unit": "member-timesteps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded white-noise temperature per member)",
            "config": {"workload": "ensemble64: 64 no-slip RBC members, grids {32^2x32, 64^2x48, 96^2x64, 128^2x64} "
                                   "(PCG64 seed 3), Ra in [1e4, 1e6], Pr in [0.7, 7], ARS_222, dt 1e-4, FP64",
                       "grid_points_all_members": pts, "batched_substitution": ens.batched},
            "grid_point_steps_per_s": pts * 1e3 / ms, "gpu_launches": ens.query(1) - l0,
            "launches_per_step": ens.query(3), "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    ens.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="rbc_384x384x192", choices=sorted(CONFIGS) + ["ensemble64"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-split", action="store_true", help="skip the split-precision leg")
    ap.add_argument("--variant", action="append", default=[], metavar="KNOB=0|1",
                    help="pin a kernel variant of the autotuner (coral_set_variant); repeatable")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.config == "ensemble64":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the ensemble workload is timed on the GPU arm only"}))
        else:
            run_ensemble(args)
        return
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
