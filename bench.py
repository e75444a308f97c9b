#!/usr/bin/env python
"""Benchmark: C192 linear shallow-water RK4 on the Ch-staggered cubed sphere.

Workload (one bench step): one simulated day of C192 (6 x 192 x 192 cells),
dt = 150 s, 576 RK4 steps, Gaussian hill (d0 = 0.15 rad, 1 m) centred on a cube
corner with a seeded jitter <= 1e-3 rad, H = 1000 m, f = 2 Omega sin(lat).
Metric: cell-updates/s = 6 N^2 * 576 / seconds (one cell advanced by one full
RK4 step).  The headline ``value`` is the FP32 path (FP32 stencils, FP64 metric
precompute and reductions, Kahan-compensated state); the FP64 path is reported
beside it with the FP32-vs-FP64 relative L2/max errors after the day.

Timing: W untimed warm-up integrations, then K timed integrations; each starts
from the initial state restored on the device and after an L2 flush (a 512 MiB
device write), bracketed by CUDA events on the library's stream; max over ranks.
The stage kernels' tile size is autotuned per precision before the warm-up
(``--tile`` fixes it instead).

Also reported (``nonlinear``): C384 nonlinear Williamson test 2 with a tilted
axis, dt 75 s, 1152 RK4 steps, advective operator, FP32 and FP64, with errors
against the steady state.  And (``ensemble``): the batched ensemble, 256 members
of C48, dt 600 s, 144 RK4 steps, FP32, in one context, against the same 256
members run one after another through a single-member context.  And
(``serving``): a seeded Poisson stream (200 requests/s) of linear integrations,
N uniform over {24, 48, 96, 192, 384}, 24-576 RK4 steps, FP32/FP64 50/50,
served with continuous batching under an HBM budget; p50/p99 latency,
throughput, and the FP32 requests' errors against the same requests in FP64.
``--gpus N`` runs N independent replicas (one per GPU, weak scaling, no
data-path collective).  ``--impl reference`` times the CPU restatement of the
reference (the Fortran/MPI reference needs mpiifort, absent here).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELLS = 192
DT = 150.0
NSTEPS = 576
H_MEAN = 1000.0
SEED = 20261203 + 1


def workload_ic(N=N_CELLS, seed=SEED):
    """Cube-corner Gaussian with seeded jitter (same generator as the test cases)."""
    from ch_swe_b200 import testcases
    rng = np.random.default_rng(seed)
    lam0 = 0.25 * np.pi + rng.uniform(-1e-3, 1e-3)
    phi0 = np.arcsin(1.0 / np.sqrt(3.0)) + rng.uniform(-1e-3, 1e-3)
    return testcases.gaussian_hill(N, lam0=lam0, phi0=phi0, d0=0.15, amp=1.0), (lam0, phi0)


def cells_per_step(N):
    return 6 * N * N * NSTEPS


def dof(N):
    return 6 * (N + 1) ** 2 + 12 * N * (N + 1)


# ----------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        # the raw samples go to CHSWE_CLOCKS_DIR (default: the system's temporary directory)
        import tempfile
        out_dir = os.environ.get("CHSWE_CLOCKS_DIR", tempfile.gettempdir())
        self.path = os.path.join(out_dir, f"clocks_gpu{gpu_index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------
# CPU legs (the oracle): only here and in the reference arm
# ----------------------------------------------------------------------------
_WORKER = {}


def _cpu_init(N):
    sys.path.insert(0, ROOT)
    from oracle.oracle import Oracle
    _WORKER["ic"] = workload_ic(N)[0]
    _WORKER["o"] = Oracle(N, h_mean=H_MEAN)


def _cpu_worker(args):
    N, steps = args
    if "o" not in _WORKER:
        _cpu_init(N)
    h, u, v = _WORKER["ic"]
    t0 = time.perf_counter()
    _WORKER["o"].rk4(h, u, v, DT, steps)
    return time.perf_counter() - t0


def cpu_baseline(steps=40):
    """Oracle on one host core, bounded sample of the same workload."""
    from oracle import oracle as orc
    orc.build()
    t = _cpu_worker((N_CELLS, steps))
    return {"value": 6 * N_CELLS * N_CELLS * steps / t, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"C{N_CELLS}, {steps} RK4 steps of the same day (dt {DT:g} s), FP64 CPU restatement, 1 thread"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    from oracle import oracle as orc
    orc.build()
    cores = os.cpu_count() or 1
    steps = 12
    ctx = mp.get_context("spawn")
    times = []
    with ctx.Pool(cores, initializer=_cpu_init, initargs=(N_CELLS,)) as pool:
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            pool.map(_cpu_worker, [(N_CELLS, steps)] * cores)
            dt = time.perf_counter() - t0
            if k >= args.warmup:
                times.append(dt)
    tot = sum(times)
    value = cores * 6 * N_CELLS * N_CELLS * steps * len(times) / tot
    line = {
        "impl": "reference", "metric": "C192 RK4 cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"C{N_CELLS} linear SWE (Ch, SBP 4-2), dt {DT:g} s, bounded sample of {steps} "
                               f"RK4 steps per process", "N": N_CELLS, "l2_between_steps": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                         "sample": f"{cores} spawn processes x C{N_CELLS} x {steps} RK4 steps (FP64 CPU restatement; "
                                   "the Fortran/MPI reference needs mpiifort, absent)"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)), "measured"
        except Exception:
            pass
    return {"hbm_gbs": 6650.0}, "fallback"


def profile_traffic(key):
    """DRAM bytes per launch of the stage kernel at C192 from the ncu captures summarised
    under profiles/: key "fp32" (the split k_stage) or "fp32_fused" (k_fstage)."""
    p = os.path.join(ROOT, "profiles", "k_stage_c192_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)).get(key)
        except Exception:
            return None
    return None


def set_tile(dom, args):
    if args.kernel_config:
        dom.kernel_config = tuple(int(x) for x in args.kernel_config.split(","))
        return None
    if args.tile == "auto":
        return dom.autotune(nreps=10)
    dom.tile = int(args.tile)
    return None


def run_precision(precision, ic, args, torch, dist, world):
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from ch_swe_b200 import _lib
    dom = create_domain(N_CELLS, precision=precision, h_mean=H_MEAN)
    stream = torch.cuda.current_stream()
    dom.set_stream(stream.cuda_stream)
    tune = set_tile(dom, args)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": H_MEAN}, dom)
    st = create_stvec_swm(dom)
    ic_dev = create_stvec_swm(dom).upload(*ic)
    rk = create_timescheme(st, "rk4")
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def one():
        st.assign(1.0, ic_dev)
        rk.steps(st, op, dom, DT, NSTEPS)

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    evs = []
    n0 = dom.launch_count()
    for _ in range(args.steps):
        st.assign(1.0, ic_dev)
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rk.steps(st, op, dom, DT, NSTEPS)
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    launches = dom.launch_count() - n0
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    if world > 1:
        from ch_swe_b200 import replicas
        total_ms = replicas.max_over_ranks(total_ms, dist, device="cuda")
        dist.barrier()
    final = st.download()

    # end-to-end through the public API: pinned host -> device, the day, device -> host
    nbytes = st.device_view()[1]
    e2e_s = 0.0
    for _ in range(max(1, min(args.steps, 3))):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st.upload(*ic)
        rk.steps(st, op, dom, DT, NSTEPS)
        st.download()
        e2e_s += time.perf_counter() - t0
    e2e_n = max(1, min(args.steps, 3))

    # per-kernel durations (events around each launch, warm L2 as inside a day)
    import ctypes
    co = ctypes.c_double()
    ed = ctypes.c_double()
    sg = ctypes.c_double()
    st.assign(1.0, ic_dev)
    _lib.check(_lib.load().swe_kernel_times(dom.ctx, st.handle, DT, 20, ctypes.byref(co), ctypes.byref(ed), ctypes.byref(sg)),
               dom.ctx, "kernel times")
    return {
        "total_ms": total_ms, "launches": launches, "final": final,
        "e2e_value": cells_per_step(N_CELLS) * e2e_n / e2e_s, "e2e_bytes": nbytes,
        "ms_co2contra": co.value, "ms_edge": ed.value, "ms_stage": sg.value, "dom": dom,
        "tile": dom.tile, "kernel_config": list(dom.kernel_config), "tune_ms_per_rk4_step": tune,
    }


ENS_N, ENS_M, ENS_DT, ENS_STEPS, ENS_SEED = 48, 256, 600.0, 144, 20261203 + 4
SRV_REQUESTS, SRV_RATE, SRV_SEED, SRV_BUDGET = 120, 200.0, 20261203 + 5, 24 << 30
# a second stream of the same generator below the device's capacity (about 15 requests/s
# of this mix): there the latency is service time, not queueing
SRV_LOW_REQUESTS, SRV_LOW_RATE, SRV_LOW_SEED = 48, 4.0, 20261203 + 6
NL_N, NL_DT, NL_STEPS, NL_SEED = 384, 75.0, 1152, 20261203 + 3


def run_nonlinear(args, torch, dist, world):
    """Config 3: nonlinear Williamson test 2 (steady zonal flow about a tilted axis) at
    C384, dt 75 s, 1152 RK4 steps, advective operator; FP32 and FP64; errors against
    the analytic steady state (the initial state) and FP32 against FP64."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme, testcases
    from ch_swe_b200.testcases import EARTH_GRAV, EARTH_RADIUS
    rng = np.random.default_rng(NL_SEED)
    theta = float(rng.uniform(0.0, 0.5 * np.pi))
    axis = (np.sin(theta), 0.0, np.cos(theta))
    u0 = 2.0 * np.pi * EARTH_RADIUS / (12.0 * 86400.0)
    hm = 2.94e4 / EARTH_GRAV
    ic = testcases.williamson2(NL_N, u0=u0, h_mean=hm, axis=axis)
    stream = torch.cuda.current_stream()
    out, final = {}, {}
    for prec in ("fp32", "fp64"):
        dom = create_domain(NL_N, precision=prec, operator="advective", rotation_axis=axis)
        dom.set_stream(stream.cuda_stream)
        tune = set_tile(dom, args)
        op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom)
        x = create_stvec_swm(dom).upload(*ic)
        rk = create_timescheme(x, "rk4")
        rk.steps(x, op, dom, NL_DT, 4)
        x.upload(*ic)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rk.steps(x, op, dom, NL_DT, NL_STEPS)
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        if world > 1:
            from ch_swe_b200 import replicas
            ms = replicas.max_over_ranks(ms, dist, device="cuda")
        final[prec] = x.download()
        errs = {nm: {"rel_l2": float(np.linalg.norm(f - r) / np.linalg.norm(r)),
                     "rel_max": float(np.abs(f - r).max() / np.abs(r).max())}
                for nm, f, r in zip("huv", final[prec], ic)}
        out[prec] = {"value": world * 6 * NL_N ** 2 * NL_STEPS / (ms / 1e3), "ms_total": ms, "tile": dom.tile,
                     "tune_ms_per_rk4_step": tune, "error_vs_steady_state": errs}
        dom.destroy()
    out["fp32_vs_fp64"] = {nm: {"rel_l2": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                                "rel_max": float(np.abs(a - b).max() / np.abs(b).max())}
                           for nm, a, b in zip("huv", final["fp32"], final["fp64"])}
    out["workload"] = (f"C{NL_N} nonlinear SWE (advective operator, covariant Ch, up4 flux and advection), "
                       f"Williamson test 2, u0 = 2 pi a / 12 days, axis tilted by {theta:.4f} rad (seed {NL_SEED}), "
                       f"g h0 = 2.94e4 m2/s2, dt {NL_DT:g} s, {NL_STEPS} RK4 steps")
    out["unit"] = "cell-updates/s"
    return out


# the diffusion of the reference's Ah experiments (rh4_run.sh: uv 0.03, h 0.01, explicit_Eul1)
AH_DIFF = {"hordiff_uv_name": "hordiff_vec_xyz_Ah_sbp_42_narrow", "uv_diff_coeff": 0.03,
           "hordiff_h_name": "hordiff_scalar_Ah_sbp_42_narrow", "h_diff_coeff": 0.01}


def run_ah(args, torch, dist, world):
    """The Ah staggering of the linear operator (h, u, v on the vertices, node SBP 4-2
    operators with projections) on the day workload: C192, dt 150 s, 576 RK4 steps,
    FP32, the same cube-corner Gaussian with the wind at rest; mass and energy drift
    over the day from the FP64 SBP_Ah42 quadrature."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    ic = workload_ic()[0]
    h = ic[0]
    z = np.zeros_like(h)
    stream = torch.cuda.current_stream()
    dom = create_domain(N_CELLS, precision="fp32", h_mean=H_MEAN, horizontal_staggering="Ah")
    dom.set_stream(stream.cuda_stream)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": H_MEAN}, dom)
    x = create_stvec_swm(dom).upload(h, z, z)
    rk = create_timescheme(x, "rk4")
    rk.steps(x, op, dom, DT, 8)
    x.upload(h, z, z)
    m0, e0 = op.integrals(x)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    rk.steps(x, op, dom, DT, NSTEPS)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    if world > 1:
        from ch_swe_b200 import replicas
        ms = replicas.max_over_ranks(ms, dist, device="cuda")
    m1, e1 = op.integrals(x)
    # the driver loop with the diffusion step after every RK4 step, in the same graphs
    from ch_swe_b200 import create_swm_diff_operator
    dif = create_swm_diff_operator(AH_DIFF, dom)
    dom.set_diffusion(dif)
    x.upload(h, z, z)
    rk.steps(x, op, dom, DT, 8)
    x.upload(h, z, z)
    md0, _ = op.integrals(x)
    torch.cuda.synchronize()
    a.record(stream)
    rk.steps(x, op, dom, DT, NSTEPS)
    b.record(stream)
    torch.cuda.synchronize()
    msd = a.elapsed_time(b)
    if world > 1:
        from ch_swe_b200 import replicas
        msd = replicas.max_over_ranks(msd, dist, device="cuda")
    md1, _ = op.integrals(x)
    dom.set_diffusion(None)
    dom.destroy()
    return {"workload": f"C{N_CELLS} linear SWE on the Ah staggering (div_ah_sbp_proj_42, grad_ah_sbp_proj_42, "
                        f"coriolis_colocated, co2contra_colocated), FP32, dt {DT:g} s, {NSTEPS} RK4 steps, "
                        "the day workload's Gaussian with the wind at rest",
            "value": world * 6 * N_CELLS ** 2 * NSTEPS / (ms / 1e3), "unit": "cell-updates/s",
            "ms_total": ms, "mass_rel_drift": (m1 - m0) / abs(m0), "energy_rel_drift": (e1 - e0) / abs(e0),
            "with_diffusion": {
                "what": "each RK4 step followed by one explicit_Eul1 step of " + AH_DIFF["hordiff_uv_name"] + " (uv "
                        f"coefficient {AH_DIFF['uv_diff_coeff']}) and " + AH_DIFF["hordiff_h_name"] +
                        f" (h coefficient {AH_DIFF['h_diff_coeff']}), captured with the RK4 stages",
                "value": world * 6 * N_CELLS ** 2 * NSTEPS / (msd / 1e3), "unit": "cell-updates/s",
                "ms_total": msd, "mass_rel_drift": (md1 - md0) / abs(md0)}}


def run_serving(args, torch):
    """Config 5: continuous batching of a Poisson request stream."""
    from ch_swe_b200 import serve
    reqs = serve.poisson_stream(SRV_REQUESTS, rate=SRV_RATE, seed=SRV_SEED)
    for r in reqs:
        r.ic   # generate the initial states before the clock starts
    srv = serve.Server(hbm_budget_bytes=SRV_BUDGET, max_tick=16, grouped=True)
    # tuning is a one-time cost per pool shape: done before the stream starts
    srv.pretune({(r.N, r.precision, r.operator) for r in reqs})
    stats = srv.run(reqs, realtime=True)
    srv.close()
    group_ticks = srv.group_ticks
    # the same stream with every pool ticking on its own stream (no group launches)
    reqs_u = serve.poisson_stream(SRV_REQUESTS, rate=SRV_RATE, seed=SRV_SEED)
    for r in reqs_u:
        r.ic
    srv = serve.Server(hbm_budget_bytes=SRV_BUDGET, max_tick=16)
    srv.pretune({(r.N, r.precision, r.operator) for r in reqs_u})
    su = srv.run(reqs_u, realtime=True)
    srv.close()
    # FP32 requests against the same request in FP64 (the FP64 path is pinned to the
    # oracle at 1e-12): a bounded sample of the smaller cubes
    errs = []
    for r in [r for r in reqs if r.precision == "fp32" and r.N <= 96][:8]:
        import copy
        r64 = copy.copy(r)
        r64.precision = "fp64"
        ref = serve.run_alone(r64)
        errs.append({"rid": r.rid, "N": r.N, "steps": r.nsteps, "operator": r.operator,
                     **{f"{nm}_rel_l2": float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
                        for nm, a, b in zip("huv", r.result, ref)}})
    by_size = {}
    for N in serve.SIZES:
        lat = [r.latency * 1e3 for r in reqs if r.N == N]
        if lat:
            by_size[f"C{N}"] = {"n": len(lat), "p50_ms": float(np.percentile(lat, 50)),
                                "p99_ms": float(np.percentile(lat, 99))}
    seq_s = sequential_seconds(reqs)
    # the stream below capacity
    low = serve.poisson_stream(SRV_LOW_REQUESTS, rate=SRV_LOW_RATE, seed=SRV_LOW_SEED)
    for r in low:
        r.ic
    srv = serve.Server(hbm_budget_bytes=SRV_BUDGET, max_tick=16, grouped=True)
    srv.pretune({(r.N, r.precision, r.operator) for r in low})
    ls = srv.run(low, realtime=True)
    srv.close()
    offered = sum(r.cell_updates for r in low) / max(low[-1].arrival, 1e-9)
    return {
        "workload": f"{SRV_REQUESTS} requests, Poisson {SRV_RATE:g}/s (seed {SRV_SEED}), N in {list(serve.SIZES)}, "
                    "24-576 RK4 steps, FP32/FP64 50/50, linear/advective operator 50/50, 1-4 seeded Gaussians",
        "grouped": {"what": "the linear pools of each precision up to C96 tick together: one grid per kernel "
                               "over their cube sizes (swe_group_rk4_steps_members), 12 launches per RK4 step; "
                               "C192 and C384 pools on their own streams and autotuned configurations",
                    "group_ticks": group_ticks},
        "requests": stats.n, "makespan_s": stats.makespan_s, "p50_ms": stats.p50_ms, "p99_ms": stats.p99_ms,
        "mean_ms": stats.mean_ms, "requests_per_s": stats.requests_per_s,
        "cell_updates_per_s": stats.cell_updates_per_s, "hbm_budget_bytes": SRV_BUDGET,
        "peak_pool_bytes": stats.peak_bytes, "pools": stats.pools, "latency_by_size": by_size,
        "service_p50_ms": stats.service_p50_ms, "service_p99_ms": stats.service_p99_ms,
        "wait_p50_ms": stats.wait_p50_ms, "wait_p99_ms": stats.wait_p99_ms,
        "offered_cell_updates_per_s": sum(r.cell_updates for r in reqs) / max(reqs[-1].arrival, 1e-9),
        "sequential": {"what": "the same requests one after another, each in a single-member context "
                               "(created before the clock) with its upload and download",
                       "seconds": seq_s, "cell_updates_per_s": sum(r.cell_updates for r in reqs) / seq_s,
                       "served_over_sequential": (sum(r.cell_updates for r in reqs) / stats.makespan_s) /
                                                 (sum(r.cell_updates for r in reqs) / seq_s)},
        "ungrouped": {"what": "the same stream, every pool ticking on its own stream",
                      "makespan_s": su.makespan_s, "cell_updates_per_s": su.cell_updates_per_s,
                      "p50_ms": su.p50_ms, "p99_ms": su.p99_ms, "service_p50_ms": su.service_p50_ms,
                      "service_p99_ms": su.service_p99_ms},
        "below_capacity": {
            "workload": f"{SRV_LOW_REQUESTS} requests, Poisson {SRV_LOW_RATE:g}/s (seed {SRV_LOW_SEED}), same mix",
            "offered_cell_updates_per_s": offered, "makespan_s": ls.makespan_s,
            "cell_updates_per_s": ls.cell_updates_per_s, "p50_ms": ls.p50_ms, "p99_ms": ls.p99_ms,
            "service_p50_ms": ls.service_p50_ms, "service_p99_ms": ls.service_p99_ms,
            "wait_p50_ms": ls.wait_p50_ms, "wait_p99_ms": ls.wait_p99_ms},
        "fp32_vs_fp64_sample": errs,
    }


def sequential_seconds(reqs):
    """Wall time of the requests run one after another without batching: one
    single-member context per (N, precision, operator), created and autotuned before
    the clock; each request uploads its state, integrates and downloads."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_timescheme, serve
    doms = {}
    for key in sorted({(r.N, r.precision, r.operator) for r in reqs}):
        dom = create_domain(key[0], precision=key[1], operator=key[2])
        dom.autotune(nreps=8)
        op = serve._operator(dom, key[2])
        st = create_stvec_swm(dom)
        doms[key] = (dom, op, st, create_timescheme(st, "rk4"))
    total = 0.0
    for r in reqs:
        dom, op, st, ts = doms[(r.N, r.precision, r.operator)]
        if r.operator == "linear":
            op.set_member_h_mean(0, r.h_mean)
        t0 = time.perf_counter()
        st.upload(*r.initial_state())
        ts.steps_members(st, op, [r.dt], r.nsteps)
        st.download()
        total += time.perf_counter() - t0
    for dom, _, _, _ in doms.values():
        dom.destroy()
    return total


def run_ensemble(args, torch, dist, world):
    """Batched ensemble (all members in one context) vs the same members one by one."""
    from ch_swe_b200 import create_timescheme, ensemble, create_domain, create_stvec_swm, create_swm_operator
    stream = torch.cuda.current_stream()
    dom, op, st, params = ensemble.create_ensemble(ENS_N, ENS_M, ENS_SEED, precision="fp32")
    dom.set_stream(stream.cuda_stream)
    tune = set_tile(dom, args)
    ic_dev = create_stvec_swm(dom)
    ic_dev.assign(1.0, st)
    rk = create_timescheme(st, "rk4")
    for _ in range(max(1, args.warmup)):
        st.assign(1.0, ic_dev)
        rk.steps(st, op, dom, ENS_DT, ENS_STEPS)
    torch.cuda.synchronize()
    reps = 2
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    batched_ms = 0.0
    for _ in range(reps):
        st.assign(1.0, ic_dev)
        a.record(stream)
        rk.steps(st, op, dom, ENS_DT, ENS_STEPS)
        b.record(stream)
        torch.cuda.synchronize()
        batched_ms += a.elapsed_time(b)
    batched_ms /= reps
    # sequential: one single-member context, the members one after another
    h0, u0, v0 = ensemble.initial_states(ENS_N, params)
    d1 = create_domain(ENS_N, precision="fp32", h_mean=params[0][0])
    d1.set_stream(stream.cuda_stream)
    set_tile(d1, args)
    op1 = create_swm_operator(d1.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": params[0][0]}, d1)
    s1 = create_stvec_swm(d1)
    rk1 = create_timescheme(s1, "rk4")
    s1.upload(h0[0], u0[0], v0[0])
    rk1.steps(s1, op1, d1, ENS_DT, ENS_STEPS)
    torch.cuda.synchronize()
    seq_ms = 0.0
    for k in range(ENS_M):
        s1.upload(h0[k], u0[k], v0[k])
        op1.set_member_h_mean(0, params[k][0])
        a.record(stream)
        rk1.steps(s1, op1, d1, ENS_DT, ENS_STEPS)
        b.record(stream)
        torch.cuda.synchronize()
        seq_ms += a.elapsed_time(b)
    # spot check: the last member alone equals its slot in the batch
    st.assign(1.0, ic_dev)
    rk.steps(st, op, dom, ENS_DT, ENS_STEPS)
    got = st.download(member=ENS_M - 1)
    alone = s1.download()
    diff = max(float(np.abs(g - r).max() / max(np.abs(r).max(), 1e-30)) for g, r in zip(got, alone))
    cells = 6 * ENS_N * ENS_N * ENS_STEPS * ENS_M
    if world > 1:
        from ch_swe_b200 import replicas
        batched_ms = replicas.max_over_ranks(batched_ms, dist, device="cuda")
        seq_ms = replicas.max_over_ranks(seq_ms, dist, device="cuda")
    out = {
        "workload": f"{ENS_M} members x C{ENS_N} linear SWE, dt {ENS_DT:g} s, {ENS_STEPS} RK4 steps, FP32 "
                    "(FP64 metric and reductions, Kahan state), H ~ U[500,2000] m, 1-4 seeded Gaussians",
        "value": world * cells / (batched_ms / 1e3), "unit": "cell-updates/s", "ms_batched": batched_ms,
        "sequential_value": world * cells / (seq_ms / 1e3), "ms_sequential": seq_ms,
        "batched_over_sequential": seq_ms / batched_ms, "tile": dom.tile, "tune_ms_per_rk4_step": tune,
        "last_member_batched_vs_alone_rel_max": diff,
    }
    dom.destroy()
    d1.destroy()
    return out


def run_ours(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        from ch_swe_b200 import replicas
        dist = replicas.init("nccl", local)
    cpu = cpu_baseline() if (rank == 0 and world == 1 and not args.no_cpu) else None
    from ch_swe_b200 import build
    build.build()
    ic, (lam0, phi0) = workload_ic()
    res = {}
    stream = torch.cuda.Stream()   # a real (non-default) stream shared by torch events and the library
    with ClockSampler(local) as clk, torch.cuda.stream(stream):
        for prec in ("fp32", "fp64"):
            res[prec] = run_precision(prec, ic, args, torch, dist, world)
        ens = None if args.no_ensemble else run_ensemble(args, torch, dist, world)
        srv = None if (args.no_serving or world > 1) else run_serving(args, torch)
        nl = None if args.no_nonlinear else run_nonlinear(args, torch, dist, world)
        ah = None if args.no_ah else run_ah(args, torch, dist, world)
    clocks = clk.summary()

    K = args.steps
    r32, r64 = res["fp32"], res["fp64"]
    v32 = world * cells_per_step(N_CELLS) * K / (r32["total_ms"] / 1e3)
    v64 = world * cells_per_step(N_CELLS) * K / (r64["total_ms"] / 1e3)
    errs = {}
    for name, a, b in zip("huv", r32["final"], r64["final"]):
        errs[name] = {"rel_l2": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                      "rel_max": float(np.abs(a - b).max() / np.abs(b).max())}
    peaks, src = measured_peaks()
    D = dof(N_CELLS)
    # algorithmic bytes of one fused stage launch, per DOF and RK4 step: S1 reads the
    # state and writes Y1, ACC (3 words); S2, S3 read Y, V0, ACC and write Y, ACC (5
    # each); S4 reads Y3, V0, ACC and writes V0 (4); FP32 adds the Kahan compensation
    # read and write in S4 (2): 19 words of 4 B per step, 19/4 per launch
    alg_bytes_32 = D * 4 * (19 / 4)
    achieved = alg_bytes_32 / (r32["ms_stage"] / 1e3) / 1e9
    # the stage kernel of the configuration the autotuner chose: the split k_stage (its
    # contravariant components from k_co2contra) or the fused k_fstage (TMA tiles, the
    # contravariant components computed in the tile, edge strips from k_strip)
    fused32 = r32["kernel_config"][2] == 2
    kn = ("k_strip", "k_edge", "k_fstage") if fused32 else ("k_co2contra", "k_edge", "k_stage")
    peak = float(peaks.get("hbm_gbs", 6650.0))
    line = {
        "metric": "C192 RK4 cell-updates/s", "value": v32, "unit": "cell-updates/s", "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": r32["total_ms"] / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"C{N_CELLS} linear SWE (Ch staggering, SBP 4-2), 1 simulated day = {NSTEPS} RK4 "
                               f"steps of dt {DT:g} s per bench step, cube-corner Gaussian (seeded jitter)",
                   "N": N_CELLS, "cells": 6 * N_CELLS ** 2, "dof": D, "dt": DT, "rk4_steps_per_step": NSTEPS,
                   "h_mean": H_MEAN, "gaussian_centre": [lam0, phi0], "parallelism": f"replicas x{world}",
                   "l2_between_steps": "flushed (512 MiB device write) before every timed step"},
        "fp64": {"value": v64, "ms_per_step": r64["total_ms"] / K, "ms_stage_kernel": r64["ms_stage"],
                 "ms_co2contra_kernel": r64["ms_co2contra"], "ms_edge_kernel": r64["ms_edge"], "tile": r64["tile"],
                 "tune_ms_per_rk4_step": r64["tune_ms_per_rk4_step"]},
        "fp32_tile": r32["tile"], "fp32_kernel_config": r32["kernel_config"],
        "fp64_kernel_config": r64["kernel_config"], "fp32_tune_ms_per_rk4_step": r32["tune_ms_per_rk4_step"],
        "fp32_kernel_ms": {kn[0]: r32["ms_co2contra"], kn[1]: r32["ms_edge"], kn[2]: r32["ms_stage"]},
        "fp32_over_fp64": v32 / v64,
        "fp32_vs_fp64_after_one_day": errs,
        "e2e": {"value": r32["e2e_value"], "unit": "cell-updates/s", "h2d_bytes_per_step": r32["e2e_bytes"],
                "d2h_bytes_per_step": r32["e2e_bytes"],
                "path": "ch_swe_b200.swm -> libchswe.so C ABI: upload (pinned staging), 576 RK4 steps, download"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": profile_traffic("fp32_fused" if fused32 else "fp32"), "kernel": kn[2] + "<float>",
                     "peak_source": src, "ms_per_launch": r32["ms_stage"],
                     "alg_bytes_per_launch": alg_bytes_32},
        "gpu_launches": r32["launches"],
        "clocks": clocks,
    }
    if ens is not None:
        line["ensemble"] = ens
    if srv is not None:
        line["serving"] = srv
    if nl is not None:
        line["nonlinear"] = nl
    if ah is not None:
        line["ah"] = ah
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    for r in res.values():
        r["dom"].destroy()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_profile_leg(args):
    """A few RK4 steps of one workload and nothing else: the command the ncu
    summaries under profiles/ are taken from (never a bench value)."""
    import torch
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme, ensemble, testcases
    tile = None if args.tile == "auto" else int(args.tile)
    if args.profile_leg == "ensemble":
        dom, op, st, _ = ensemble.create_ensemble(ENS_N, ENS_M, ENS_SEED, precision="fp32")
        dt = ENS_DT
    elif args.profile_leg == "nonlinear":
        axis = (np.sin(0.7), 0.0, np.cos(0.7))
        dom = create_domain(NL_N, precision="fp32", operator="advective", rotation_axis=axis)
        op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom)
        st = create_stvec_swm(dom).upload(*testcases.williamson2(NL_N, axis=axis))
        dt = NL_DT
    elif args.profile_leg in ("ah", "ah_diffusion"):
        dom = create_domain(N_CELLS, precision="fp32", h_mean=H_MEAN, horizontal_staggering="Ah")
        op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": H_MEAN}, dom)
        h = workload_ic()[0][0]
        st = create_stvec_swm(dom).upload(h, np.zeros_like(h), np.zeros_like(h))
        dt = DT
        if args.profile_leg == "ah_diffusion":
            from ch_swe_b200 import create_swm_diff_operator
            dom.set_diffusion(create_swm_diff_operator(AH_DIFF, dom))
    else:
        dom = create_domain(N_CELLS, precision="fp32", h_mean=H_MEAN)
        op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": H_MEAN}, dom)
        st = create_stvec_swm(dom).upload(*workload_ic()[0])
        dt = DT
    if args.kernel_config:
        dom.kernel_config = tuple(int(x) for x in args.kernel_config.split(","))
    elif tile:
        dom.tile = tile
    rk = create_timescheme(st, "rk4")
    for _ in range(args.rk4_steps):
        rk.step(st, op, dom, dt)
    torch.cuda.synchronize()
    dom_cfg = dom.kernel_config
    dom.destroy()
    print(f"profile leg {args.profile_leg}: {args.rk4_steps} RK4 steps, kernel config {dom_cfg}", flush=True)
    return 0


def main():
    global NSTEPS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the served-workload leg")
    ap.add_argument("--no-nonlinear", action="store_true", help="skip the nonlinear (C384 Williamson 2) leg")
    ap.add_argument("--tile", default="auto", choices=["auto", "17", "25", "33"],
                    help="stage-kernel tile size (default: autotuned per precision)")
    ap.add_argument("--kernel-config", default=None,
                    help="stage-kernel configuration 'tile,blocks_per_sm,runs' (overrides --tile and autotuning)")
    ap.add_argument("--rk4-steps", type=int, default=NSTEPS,
                    help="RK4 steps per bench step (default: one day = 576; shorter only for profiling runs)")
    ap.add_argument("--no-ah", action="store_true", help="skip the Ah-staggering leg")
    ap.add_argument("--profile-leg", choices=["day", "ensemble", "nonlinear", "ah", "ah_diffusion"], default=None,
                    help="run --rk4-steps steps of one workload only (for ncu captures; prints no bench line)")
    args = ap.parse_args()
    if args.profile_leg:
        return run_profile_leg(args)
    NSTEPS = args.rk4_steps
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
