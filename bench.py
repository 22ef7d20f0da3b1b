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
    "rbc_192x192x192": dict(eq="rbc_noslip_ra1e8.equations", par="rbc_noslip_ra1e8_192x192x192.parameters.in",
                            NX=192, NY=192, NZ=192, dt=1e-6, seed=2, Ra=1e8),
    "rbc_32x32x192": dict(eq="rbc_noslip_ra1e8.equations", par="rbc_noslip_ra1e8_32x32x192.parameters.in",
                          NX=32, NY=32, NZ=192, dt=1e-6, seed=2, Ra=1e8),
    "rrbc_192x192x96": dict(eq="rrbc_stressfree_ek1e-4_ra5e7.equations", par="rrbc_stressfree_192x192x96.parameters.in",
                            NX=192, NY=192, NZ=96, dt=5e-6, seed=1, Ra=5e7),
}
METRIC = "timesteps/s at 384^2x192 (FP64 path)"
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
    "inv_y": "k_inv_y", "inv_x": "k_inv_x", "inv_z": "k_inv_z", "z_products": "k_z_fused",
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
    pl = PlaneLayer(eq, par, device=dev)
    make_ic(cfg, pl)
    dt = cfg["dt"]
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
           "d2h_bytes_per_step": state_bytes / args.steps + diag_bytes}

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
        cpu = cpu_baseline(cfg, eq, par, max_seconds=args.cpu_seconds)
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded white-noise temperature IC, PCG64 seed %d)" % cfg["seed"],
        "config": {"workload": "%s: RBC no-slip Ra=%g Pr=1, %dx%dx%d modes, grid %dx%dx%d, ARS_222, dt=%g, FP64"
                               % (args.config, cfg["Ra"], pl.NX, pl.NY, pl.NZ, pl.NXAA, pl.NYAA, pl.NZAA, dt),
                   "grid_points": pl.NXAA * pl.NYAA * pl.NZAA, "systems": nsys, "active_systems": nact, "T": T,
                   "band": [pl.query(500), pl.query(600)], "blocks": ncls, "block_T": Tc, "block_band": [kl_c, ku_c],
                   "l2": "inputs larger than L2 (state %.2f GB, LU factors %.1f GB)"
                   % (field.nbytes / 1e9, nact * ncls * Tc * (2 * kl_c + ku_c + 1) * fbytes / 1e9),
                   "lu_factors": ("real-scaled" if fbytes == 8 else "complex")
                                 + (", split into %d independent blocks per system" % ncls if ncls > 1 else ""),
                   "parallelism": "replicas x%d" % world},
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
    """DRAM bytes (read + write) per launch of the phase's kernels at 384^2 x 192,
    from the ncu launch list summarised in profiles/, or None."""
    p = os.path.join(ROOT, "profiles", "dram_traffic_rbc_384x384x192.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if "=" in line and line.split("=")[0].strip() == kernels:
            return float(line.split("=")[1])
    return None


def _solve_worker(job):
    """Repeated zgbtrs on the sampled factors for about `seconds`; returns the
    number of solves (runs in a spawned process of the CPU baseline)."""
    facs, kl, ku, b, seconds = job
    import time as _t
    import scipy.linalg.lapack as _lapack
    n = 0
    t0 = _t.perf_counter()
    while _t.perf_counter() - t0 < seconds:
        for lu, piv in facs:
            _lapack.zgbtrs(lu, kl, ku, b, piv)
        n += len(facs)
    return n


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(cfg, eq, par, max_seconds=20.0, processes=None):
    """The oracle (CPU restatement, FP64) timed on a bounded sample of the same
    workload with `processes` host threads (default: all): one inverse and one
    forward 3-D transform at full size (scipy.fft workers), the band LU solves
    of a sample of (kx,ky) systems and the operator applications of a sample of
    kx slabs (a spawned process pool for the solves, a thread pool for the
    sparse products), as throughput; the step time is extrapolated to the full
    step.""" 
    from concurrent.futures import ThreadPoolExecutor
    from oracle import coral_oracle as co
    import scipy.fft as sfft
    import scipy.linalg.lapack as lapack
    processes = processes or host_threads()
    t_start = time.perf_counter()
    s = co.Solver.__new__(co.Solver)
    s.recipe = co.parse_equations(eq)
    p = co.read_parameters_text(par)
    s.params = p
    g = co.Geometry(p["NX"], p["NY"], p["NZ"], p["Lx"], p["Ly"], p["gap"], p["center"])
    s.g = g
    s.scheme = p["scheme"]
    s.nstages, s.A, s.Ah = co.ars_tableau(s.scheme)
    # operators of the kxky system (reduced to a few kx slabs for the timing sample)
    rec = s.recipe.kxky[0]
    lay = co.SystemLayout(g.NZ, rec)
    cache = {}
    mass = [(pc, co.build_piece_matrix(g.NZ, g.center, g.gap, lay, rec, pc, cache)) for pc in rec.mass]
    stif = [(pc, co.build_piece_matrix(g.NZ, g.center, g.gap, lay, rec, pc, cache)) for pc in rec.stif]
    T = lay.T
    nF, nQ = len(s.recipe.full_vars), len(s.recipe.quad_vars)
    rng = np.random.default_rng(0)
    # (a) transforms at full size
    spec = rng.standard_normal((g.NXH, g.NYAA, g.NZ)) + 1j * rng.standard_normal((g.NXH, g.NYAA, g.NZ))
    with sfft.set_workers(processes):
        t0 = time.perf_counter()
        ph = co.spec_to_phys(spec, g)
        t_inv = time.perf_counter() - t0
        t0 = time.perf_counter()
        co.phys_to_spec(ph * ph, g)
        t_fwd = time.perf_counter() - t0
    del ph, spec
    # (b) band LU solve per system: factor a handful, time zgbtrs on them
    kl = ku = 0
    for _, B in mass + stif:
        c = B.tocoo()
        kl = max(kl, int((c.row - c.col).max()))
        ku = max(ku, int((c.col - c.row).max()))
    nsample = 16
    facs = []
    for k in range(nsample):
        ix, iy = 1 + (k % max(g.NXH - 1, 1)), 1 + 7 * k % (g.NY // 2)
        M = sum((pc.dsca * co.complex_pow(complex(g.py[iy]), pc.ky) * co.complex_pow(complex(g.px[ix]), pc.kx)) * B
                for pc, B in mass)
        L = sum((pc.dsca * co.complex_pow(complex(g.py[iy]), pc.ky) * co.complex_pow(complex(g.px[ix]), pc.kx)) * B
                for pc, B in stif)
        E = (M - cfg["dt"] * s.A[0, 0] * L).tocoo()
        ab = np.zeros((2 * kl + ku + 1, T), dtype=np.complex128)
        ab[kl + ku + E.row - E.col, E.col] = E.data
        lu, piv, info = lapack.zgbtrf(ab, kl, ku)
        facs.append((lu, piv))
    b = rng.standard_normal(T) + 1j * rng.standard_normal(T)

    X = (rng.standard_normal((g.NYAA, T)) + 1j * rng.standard_normal((g.NYAA, T)))

    def mv_slab(_):
        for _, B in mass + stif:
            (B @ X.T)

    if processes > 1:
        # band solves in a spawned process pool (the LAPACK wrapper holds the
        # interpreter lock): total solves of all workers over the wall time
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(processes) as pp:
            pp.map(_solve_worker, [(facs[:1], kl, ku, b, 0.0)] * processes)  # start the workers
            t0 = time.perf_counter()
            counts = pp.map(_solve_worker, [(facs, kl, ku, b, 2.0)] * processes)
            t_solve = (time.perf_counter() - t0) / sum(counts)
    else:
        t_solve = 2.0 / _solve_worker((facs, kl, ku, b, 2.0))
    with ThreadPoolExecutor(processes) as pool:
        # (c) mass / stiffness applications, one kx slab per task
        t0 = time.perf_counter()
        list(pool.map(mv_slab, range(processes)))
        t_mv = (time.perf_counter() - t0) / (processes * g.NYAA)
    nsys = g.NXH * g.NYAA
    nact = int(g.active.sum())
    step = s.nstages * (nF * t_inv + nQ * t_fwd + nact * t_solve + nsys * t_mv)
    return {"value": 1.0 / step, "unit": "timesteps/s", "cores": processes, "kind": "port",
            "sample": ("oracle (numpy/scipy FP64, %d host threads) timed on: 1 inverse + 1 forward 3-D transform at "
                       "%dx%dx%d, zgbtrs on %d of the %d (kx,ky) systems (T=%d, kl=%d, ku=%d), M/L applications "
                       "on one kx slab; extrapolated to %d stages x (%d inverse + %d forward transforms + %d solves "
                       "+ %d operator applications); sample took %.1f s"
                       % (processes, g.NXAA, g.NYAA, g.NZAA, nsample, nact, T, kl, ku, s.nstages, nF, nQ, nact,
                          nsys, time.perf_counter() - t_start)),
            "seconds_per_step_extrapolated": step}


def run_reference(args, cfg):
    """The reference arm: the reference itself cannot be built here (Fortran
    2003 + MPI + FFTW3 + MKL, none installed), so its CPU restatement (the
    oracle) is timed on the host cores, one bounded sample per step."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    from coral_b200 import CONFIG_DIR
    eq = open(os.path.join(CONFIG_DIR, cfg["eq"])).read()
    par = open(os.path.join(CONFIG_DIR, cfg["par"])).read()
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(cfg, eq, par)
        if i >= args.warmup:
            vals.append(r["value"])
    v = statistics.median(vals)
    r["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "timesteps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.config}, "cpu_baseline": r,
            "e2e": {"value": v, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="rbc_384x384x192", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
