"""Benchmark of the heatbath + Wilson-flow hot path on the 32^4 precision workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step"): a 32^4 lattice, Haar hot start from seed 7, 500 checkerboard
Cabibbo-Marinari heatbath sweeps at beta = 6.0 (N_hits = 1), then Wilson flow to t = 4
(200 RK3 steps of eps = 0.02) with clover Q/E recorded every 10 steps; links stored as FP32
12-real, reductions in FP64.  The 32^4 FP32 field is 201 MB, larger than the 126 MB L2, so
no L2 flush is needed between timed iterations.

`value` is heatbath link-updates/s over the timed steps (CUDA events on the library's
stream, max over ranks); the flow rate, the FP64 path, the FP32-vs-FP64 errors and the
roofline of the dominant kernel are reported beside it.  `e2e` repeats the step through
the C ABI from a pinned host buffer of FP64 links (set_links) with results read back.

--impl reference times the reference algorithm on the host cores: the oracle's CPU
restatement (the reference itself cannot be built: no MPI, Eigen or c-lime) with the
reference schedule (frozen links, random shifts, lexicographic sweeps), one process per
core on 16^4 blocks as the reference's 2^4-rank decomposition of 32^4 would run.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "ecmc-qncb_b200"))

from qcb import replicas  # noqa: E402  (host-side helpers only; the library loads lazily)

L = 32
BETA = 6.0
SEED = 7
SWEEPS = 500
FLOW_EPS = 0.02
FLOW_RECORDS, FLOW_RK = 20, 10          # 200 RK3 steps, Q/E every 10
METRIC = "HB link-updates/s; flow site-steps/s; FP32 vs FP64 @|ΔQ|<1e-4; p99 latency"

# Algorithmic bytes (compulsory HBM traffic) per unit, by storage (bytes per link b):
# heatbath pass: read all 4V links once + write the V/2 updated ones = 9 b per link-update;
# flow: 24 link records + 16 su(3) records (8 reals) per site-step.
HB_BYTES = {("fp32", 12): 9 * 48, ("fp32", 18): 9 * 72, ("fp64", 18): 9 * 144}
FLOW_BYTES = {("fp32", 12): 24 * 48 + 16 * 32, ("fp64", 18): 24 * 144 + 16 * 64}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def fp32_roof(units_per_s, flop_per_unit, peak_tflops, bytes_per_unit=None, hbm_gbs=None):
    """FP32 operation rate of a kernel from its ncu-counted operations per unit.  With the
    algorithmic bytes per unit and the HBM peak it also gives the ceiling that the FP32 peak
    puts on the HBM roofline fraction: units/s at the FP32 peak x bytes per unit / HBM peak."""
    if not flop_per_unit:
        return None
    achieved = units_per_s * flop_per_unit / 1e12
    out = {"achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s", "frac": achieved / peak_tflops,
           "peak_kind": "nominal", "flop_per_unit": flop_per_unit}
    if bytes_per_unit and hbm_gbs:
        ceiling = peak_tflops * 1e12 / flop_per_unit
        out["ceiling"] = {"units_per_s_at_fp32_peak": ceiling,
                          "hbm_frac_at_fp32_peak": ceiling * bytes_per_unit / 1e9 / hbm_gbs}
    return out


def ncu_traffic():
    """DRAM bytes per launch of the dominant kernels from the committed ncu summaries."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"qcb_clocks_{os.getpid()}.csv"

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not self.path.exists():
            return None
        rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.count(",") >= 8]
        try:
            self.path.unlink()
        except OSError:
            pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------------------
def run_ours(args, rank: int, world: int, local_rank: int, dist):
    import numpy as np
    import torch

    import qcb
    from qcb import _lib

    torch.cuda.set_device(local_rank)
    ctx = qcb.Context(local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local_rank))
    lib = _lib.lib()
    dims = (L, L, L, L)
    V = L ** 4
    seed = replicas.replica_seed(SEED, rank)  # independent replicas per rank

    f32 = qcb.GaugeField(ctx, dims, "fp32", 12)
    gf = qcb.GradientFlow(FLOW_EPS)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def step(field, hb_ev=None):
        field.hot_start(seed)
        if hb_ev:
            hb_ev[0].record(stream)
        _lib.check(lib.qcb_heatbath(field.h, BETA, SWEEPS, 1, seed, 0))
        if hb_ev:
            hb_ev[1].record(stream)
        return qcb.observables.topo_charge_flowed(field, gf, FLOW_RECORDS, FLOW_RK)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, dist, device="cuda")

    for _ in range(args.warmup):
        step(f32)
    ctx.sync()

    # ---- timed region: K steps -------------------------------------------------------
    hb_events = [(ev(), ev()) for _ in range(args.steps)]
    t0, t1 = ev(), ev()
    launches0 = ctx.launches()
    barrier()
    with Clocks(local_rank) as clk:
        t0.record(stream)
        for k in range(args.steps):
            step(f32, hb_events[k])
        t1.record(stream)
        barrier()
    ctx.sync()
    launches = ctx.launches() - launches0
    total_ms = t0.elapsed_time(t1)
    hb_ms = sum(a.elapsed_time(b) for a, b in hb_events)
    flow_ms = total_ms - hb_ms  # hot start + flow + measurements
    total_ms = max_over_ranks(total_ms)
    hb_ms = max_over_ranks(hb_ms)
    flow_ms = max_over_ranks(flow_ms)
    updates = world * args.steps * SWEEPS * 4 * V
    site_steps = world * args.steps * FLOW_RECORDS * FLOW_RK * V
    hb_rate = updates / (hb_ms / 1e3)
    flow_rate = site_steps / (flow_ms / 1e3)

    # ---- per-launch durations of the dominant kernels (roofline) --------------------------
    def per_launch(fn, n):
        evs = [(ev(), ev()) for _ in range(n)]
        for a, b in evs:
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return statistics.mean(a.elapsed_time(b) for a, b in evs)

    f32.hot_start(seed)
    # one heatbath sweep = 8 pass launches
    hb_sweep_ms = per_launch(lambda: _lib.check(lib.qcb_heatbath(f32.h, BETA, 1, 1, seed, 0)), 20)
    hb_pass_ms = hb_sweep_ms / 8
    rk3_ms = per_launch(lambda: _lib.check(lib.qcb_flow_steps(f32.h, FLOW_EPS, 1)), 10)
    peak, peak_kind = peaks()
    hb_bytes_launch = HB_BYTES[("fp32", 12)] * V / 2
    hb_achieved = hb_bytes_launch / (hb_pass_ms / 1e3) / 1e9
    flow_achieved = FLOW_BYTES[("fp32", 12)] * V / (rk3_ms / 1e3) / 1e9
    traffic = ncu_traffic()
    # FP32 compute roofline beside the HBM one: ncu-counted FP32 operations per unit times
    # the measured rate, against the nominal FP32 peak (148 SMs x 128 lanes x 2 x max clock;
    # no FP32 peak is measured on this pool).
    fp32_peak = 148 * 128 * 2 * float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text()).get(
        "sm_max_mhz", 1965.0)) * 1e6 / 1e12 if (ROOT / "MEASURED_PEAKS.json").exists() else 74.4

    # ---- FP64 path (same workload, one untimed-for-value step) ---------------------------
    f64 = qcb.GaugeField(ctx, dims, "fp64", 18)
    e64 = (ev(), ev())
    a64, b64 = ev(), ev()
    a64.record(stream)
    step(f64, e64)
    b64.record(stream)
    ctx.sync()
    hb64_ms = e64[0].elapsed_time(e64[1])
    flow64_ms = a64.elapsed_time(b64) - hb64_ms
    hb64_rate = SWEEPS * 4 * V / (hb64_ms / 1e3)
    flow64_rate = FLOW_RECORDS * FLOW_RK * V / (flow64_ms / 1e3)

    # ---- precision: FP32-12 flow vs FP64-18 flow of the same FP64 heatbath output ----------
    f64.hot_start(seed)
    _lib.check(lib.qcb_heatbath(f64.h, BETA, SWEEPS, 1, seed, 0))
    f32.copy_from(f64)
    p64 = qcb.observables.mean_plaquette_global(f64)
    p32 = qcb.observables.mean_plaquette_global(f32)
    r64 = qcb.observables.topo_charge_flowed(f64, gf, 21, 10).reshape(-1, 3)
    r32 = qcb.observables.topo_charge_flowed(f32, gf, 21, 10).reshape(-1, 3)
    precision = {"dP": abs(p32 - p64), "dQ_max": float(np.abs(r32[:, 1] - r64[:, 1]).max()),
                 "dE_rel_max": float((np.abs(r32[:, 2] - r64[:, 2]) / np.abs(r64[:, 2])).max()),
                 "Q_t4_fp64": float(r64[-1, 1]), "E_t4_fp64": float(r64[-1, 2]), "plaquette_fp64": p64,
                 "same_input": "FP64 heatbath output, flowed in FP32-12 and in FP64-18"}

    # ---- e2e through the C ABI with host buffers ------------------------------------------
    # Heatbath e2e step: upload the FP64 links from a pinned host buffer (qcb_set_links),
    # 500 sweeps, mean plaquette read back.  Flow e2e step: upload, flow to t = 4 with the
    # (t, Q, E) records read back.
    host = torch.empty(V * 72, dtype=torch.float64).pin_memory()
    host.copy_(torch.from_numpy(f64.get_links().view(np.float64).reshape(-1)))

    def e2e(body):
        times = []
        for k in range(args.warmup + args.steps):
            barrier()
            a, b = ev(), ev()
            a.record(stream)
            f32.set_links_ptr(host.data_ptr())
            body()
            b.record(stream)
            b.synchronize()
            if k >= args.warmup:
                times.append(a.elapsed_time(b))
        return max_over_ranks(statistics.mean(times))

    plaq_box, tqe_box = [], []

    def hb_body():
        # 500 sweeps with the final plaquette summed inside the last sweep (one call)
        out = ctypes.c_double()
        _lib.check(lib.qcb_heatbath_plaquette(f32.h, BETA, SWEEPS, 1, seed, 0, ctypes.byref(out)))
        plaq_box.append(out.value)

    e2e_hb_ms = e2e(hb_body)
    e2e_fl_ms = e2e(lambda: tqe_box.append(qcb.observables.topo_charge_flowed(f32, gf, FLOW_RECORDS, FLOW_RK)))
    e2e_rate = world * SWEEPS * 4 * V / (e2e_hb_ms / 1e3)
    e2e_flow = world * FLOW_RECORDS * FLOW_RK * V / (e2e_fl_ms / 1e3)
    assert np.isfinite(plaq_box[-1]) and np.all(np.isfinite(tqe_box[-1]))

    result = {
        "metric": METRIC, "value": hb_rate, "unit": "link-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 links, f64 reductions", "data": "synthetic",
        "config": {"workload": "precision 32^4: Haar hot start seed 7, 500 CM heatbath sweeps beta=6.0, "
                               "flow to t=4 (200 RK3 eps=0.02, Q/E every 10)",
                   "lattice": [L, L, L, L], "storage": "fp32-12", "sweeps": SWEEPS, "n_hits": 1,
                   "flow_steps": FLOW_RECORDS * FLOW_RK, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (201 MB field vs 126 MB L2); no flush"},
        "flow": {"value": flow_rate, "unit": "site-steps/s", "ms_per_rk3": rk3_ms,
                 "e2e": {"value": e2e_flow, "unit": "site-steps/s", "ms_per_step": e2e_fl_ms,
                         "h2d_bytes_per_step": V * 72 * 8, "d2h_bytes_per_step": 3 * FLOW_RECORDS * 8},
                 "roofline": {"bound": "hbm", "achieved": flow_achieved, "peak": peak, "unit": "GB/s",
                              "frac": flow_achieved / peak, "peak_kind": peak_kind,
                              "traffic": traffic.get("flow_stage_fp32r12_per_rk3")},
                 "fp32_compute": fp32_roof(V / (rk3_ms / 1e3), traffic.get("flow_fp32r12_fp32_flop_per_site_step"),
                                           fp32_peak, FLOW_BYTES[("fp32", 12)], peak)},
        "fp64": {"hb_value": hb64_rate, "flow_value": flow64_rate, "storage": "fp64-18",
                 "hb_speedup_fp32": hb_rate / world / hb64_rate, "flow_speedup_fp32": flow_rate / world / flow64_rate},
        "precision": precision,
        "roofline": {"bound": "hbm", "kernel": "k_hb_pass<float,12>", "achieved": hb_achieved, "peak": peak,
                     "unit": "GB/s", "frac": hb_achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic.get("hb_pass_fp32r12_per_launch"),
                     "algorithmic_bytes_per_launch": hb_bytes_launch, "launch_ms": hb_pass_ms,
                     "fp32_compute": fp32_roof(V / 2 / (hb_pass_ms / 1e3),
                                               traffic.get("hb_pass_fp32r12_fp32_flop_per_link_update"), fp32_peak,
                                               HB_BYTES[("fp32", 12)], peak)},
        "e2e": {"value": e2e_rate, "unit": "link-updates/s", "ms_per_step": e2e_hb_ms,
                "h2d_bytes_per_step": V * 72 * 8, "d2h_bytes_per_step": 8,
                "step": "qcb_set_links from pinned host FP64 links + 500 sweeps + plaquette to host"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if not args.no_extra and world == 1:
        result["batch"] = batch_section(ctx, lib, stream)
        result["serving"] = serving_section(ctx)
        result["latency"] = {"p50_s": result["serving"]["p50_s"], "p99_s": result["serving"]["p99_s"],
                             "workload": "serving stream (config 4)"}
        # The 20 req/s stream offers about three times the work the GPU completes per second,
        # so its latency is set by the queue.  The same job mix at 80% of the measured job
        # throughput shows the latency of a server that keeps up.
        cap = result["serving"]["throughput_jobs_per_s"]
        result["serving_80pct_load"] = serving_section(ctx, n_requests=40, rate=0.8 * cap)
        # p50 / p99 against the offered rate, below and above the measured job capacity
        curve = []
        for frac in (0.5, 1.2, 2.0):
            r = serving_section(ctx, n_requests=40, rate=frac * cap)
            curve.append({"offered_req_per_s": frac * cap, "offered_over_capacity": frac, "p50_s": r["p50_s"],
                          "p99_s": r["p99_s"], "throughput_jobs_per_s": r["throughput_jobs_per_s"]})
        s80 = result["serving_80pct_load"]
        curve.append({"offered_req_per_s": 0.8 * cap, "offered_over_capacity": 0.8, "p50_s": s80["p50_s"],
                      "p99_s": s80["p99_s"], "throughput_jobs_per_s": s80["throughput_jobs_per_s"]})
        curve.append({"offered_req_per_s": 20.0, "offered_over_capacity": 20.0 / cap,
                      "p50_s": result["serving"]["p50_s"], "p99_s": result["serving"]["p99_s"],
                      "throughput_jobs_per_s": cap})
        result["serving_curve"] = {"capacity_jobs_per_s": cap, "requests_per_point": 40,
                                   "points": sorted(curve, key=lambda c: c["offered_req_per_s"])}
        result["plain"] = plain_section()
        result["ecmc"] = ecmc_section(ctx, cpu=not args.no_cpu_baseline)
        result["large"] = large_workload()
    return result


def profile_steps(args) -> int:
    """warmup + steps of the workload only, nothing else; prints the kernel launch counts so
    that an ncu capture can skip the warm-up launches (-s) and take one step (-c)."""
    import qcb
    from qcb import _lib

    ctx = qcb.Context(0)
    prec, nr = ("fp32", 12) if args.storage == "fp32-12" else ("fp64", 18)
    f = qcb.GaugeField(ctx, (L, L, L, L), prec, nr)
    gf = qcb.GradientFlow(FLOW_EPS)
    counts = []
    for _ in range(args.warmup + args.steps):
        n0 = ctx.launches()
        f.hot_start(SEED)
        _lib.check(_lib.lib().qcb_heatbath(f.h, BETA, SWEEPS, 1, SEED, 0))
        qcb.observables.topo_charge_flowed(f, gf, FLOW_RECORDS, FLOW_RK)
        ctx.sync()
        counts.append(ctx.launches() - n0)
    print(json.dumps({"profile": args.storage, "launches_per_step": counts}))
    return 0


# ---------------------------------------------------------------------------------------
def batch_section(ctx, lib, stream):
    """Batching workload: 64 independent lattices, sizes uniform over {8,12,16,20,24}^4,
    beta uniform over {5.7, 5.85, 6.0, 6.2} (host seed 2024), alternating hot and cold
    starts, 100 heatbath sweeps then the flow to t = 2 (100 RK3 steps, Q/E every 0.2), FP32
    12-real with FP64 reductions; one graph-captured persistent plan; tiles autotuned."""
    import numpy as np
    import torch

    import qcb

    rng = np.random.default_rng(2024)
    n = 64
    sizes = rng.choice([8, 12, 16, 20, 24], size=n)
    betas = rng.choice([5.7, 5.85, 6.0, 6.2], size=n)
    seeds = [3000 + k for k in range(n)]
    fields = []
    for k in range(n):
        f = qcb.GaugeField(ctx, (int(sizes[k]),) * 4, "fp32", 12)
        if k % 2 == 0:
            f.hot_start(seeds[k])
        fields.append(f)
    vols = [int(L) ** 4 for L in sizes]
    batch = qcb.Batch(ctx, fields)
    t0 = time.perf_counter()
    batch.autotune(os.path.join(os.environ.get("TMPDIR", "/tmp"), "qcb_tune.json"))
    tune_s = time.perf_counter() - t0
    hb_tiles, flow_tiles = batch.tiles()

    def timed(fn, reps=2):
        fn()  # capture / warm
        ctx.sync()
        best = 1e30
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out = fn()
            b.record(stream)
            b.synchronize()
            best = min(best, a.elapsed_time(b))
        return best, out

    offs = [0] * n
    hb_ms, _ = timed(lambda: batch.run(betas, seeds, offs, n_sweeps=100, n_groups=0, rk_per_group=0))
    fl_ms, _ = timed(lambda: batch.run(betas, seeds, offs, n_sweeps=0, eps=0.02, n_groups=10, rk_per_group=10))
    all_ms, (plaq, rec, used) = timed(lambda: batch.run(betas, seeds, offs, n_sweeps=100, eps=0.02, n_groups=10,
                                                         rk_per_group=10))
    updates = 100 * 4 * sum(vols)
    site_steps = 100 * sum(vols)
    # the same heatbath work through per-lattice calls (one launch per pass and lattice)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for k, f in enumerate(fields):
        qcb._lib.check(lib.qcb_heatbath(f.h, float(betas[k]), 100, 1, seeds[k], 0))
    b.record(stream)
    b.synchronize()
    single_ms = a.elapsed_time(b)
    batch.close()
    return {"workload": "64 lattices {8..24}^4 x {5.7..6.2}, 100 sweeps + flow to t=2, fp32-12", "graph": used,
            "total_volume": sum(vols), "ms_per_plan": all_ms,
            "hb": {"value": updates / (hb_ms / 1e3), "unit": "link-updates/s", "ms": hb_ms},
            "flow": {"value": site_steps / (fl_ms / 1e3), "unit": "site-steps/s", "ms": fl_ms},
            "unbatched_hb": {"value": updates / (single_ms / 1e3), "unit": "link-updates/s", "ms": single_ms,
                             "launches": 64 * 800},
            "autotune_s": tune_s, "tiles": {"hb": sorted(set(hb_tiles)), "flow": sorted(set(flow_tiles))},
            "mean_plaquette": float(np.mean(plaq)), "mean_E_t2": float(np.mean(rec[:, -1, 2]))}


ECMC_L, ECMC_LCORE, ECMC_THETA = 64, 4, 100.0
FP64_NOMINAL_TFLOPS = 37.0  # B200 FP64 (non-tensor), NVIDIA's nominal figure; not measured here


def _ecmc_cpu_worker(args):
    """One host core as one rank of the reference: the oracle's restatement of
    sample_persistant with the reference's own generator (std::mt19937_64, std::
    distributions, the rank's set regenerated per call) on a 4^4 block with frozen faces,
    random_shift + one sample call per shift (theta_sample 100), for `budget` seconds."""
    seed, budget = args
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.select_build("fast")
    p = dict(beta=BETA, theta_sample=ECMC_THETA, theta_refresh_site=50.0, theta_refresh_R=15.0, epsilon_set=0.15,
             poisson=0)
    run = oracle.EcmcRefRun(ECMC_LCORE, seed, False, p)
    run.run(5)
    events0 = run.run(0)[1][0]
    t = time.perf_counter()
    events = events0
    while time.perf_counter() - t < budget:
        events = run.run(20)[1][0]
    return events - events0, time.perf_counter() - t


def ecmc_cpu_reference(budget_s: float = 8.0) -> dict:
    """The reference's event-chain algorithm with its own generator on the host cores, one
    process per core as one rank each (see _ecmc_cpu_worker)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.build_fast()
    cores = min(64, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1))
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_ecmc_cpu_worker, [(500 + r, budget_s) for r in range(cores)])
    return {"value": sum(r[0] for r in res) / max(r[1] for r in res), "unit": "events/s", "cores": cores,
            "kind": "port",
            "sample": f"{cores} processes, each one rank of the reference (one chain on a {ECMC_LCORE}^4 block, the "
                      f"reference's std::mt19937_64 generator and per-call set), theta_sample {ECMC_THETA:g} calls "
                      f"for {budget_s:g} s; oracle built -O3 -march=native -fcx-limited-range"}


def ecmc_section(ctx, steps=5, warmup=3, cpu_budget_s=8.0, cpu=True):
    """Event-chain Monte Carlo: a 64^4 FP64 lattice as 16^4 blocks of 4^4 (65536 chains, one
    per block, as 65536 ranks of the reference would run), beta = 6.0, from a Haar hot start
    (seed 7) plus 20 heatbath sweeps, with the reference's default budgets (theta_sample 100,
    refresh site 50, refresh R 15, epsilon_set 0.15).  One step = one random translation and
    one sample call of every chain (the links packed to the FP64 array-of-structures copy, the
    set drawn, the chains run, the links unpacked); CUDA events on the library's stream."""
    import numpy as np
    import torch

    import qcb

    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    dims = (ECMC_L,) * 4
    f = qcb.GaugeField(ctx, dims, "fp64", 18)
    f.hot_start(SEED)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, BETA, 20, 1, SEED, 0))
    ch = qcb.EventChains(f, qcb.ecmc.params(beta=BETA, theta_sample=ECMC_THETA, l_core=ECMC_LCORE), SEED)
    rng = np.random.default_rng(11)
    cum = np.zeros(4, int)

    def shift():
        nonlocal cum
        cum = (cum + rng.integers(0, ECMC_LCORE, 4)) % ECMC_L
        ch.sample(cum)

    for _ in range(warmup):
        shift()
    ch.counters(reset=True)
    launches0 = ctx.launches()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        shift()
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b)
    launches = ctx.launches() - launches0
    events, lifts, revs = ch.counters(reset=True)
    rate = events / (ms / 1e3)
    # end to end through the C ABI, the links resident: one shift + the plaquette to the host
    t = time.perf_counter()
    for _ in range(steps):
        shift()
        plaq = qcb.observables.mean_plaquette_global(f)
    e2e_s = (time.perf_counter() - t) / steps
    e_ev, _, _ = ch.counters(reset=True)
    traffic = ncu_traffic()
    flop_per_event = traffic.get("ecmc_fp64_flop_per_event")
    flop = flop_per_event * rate / 1e12 if flop_per_event else None
    out = {"metric": "ECMC events/s (one link update each)", "value": rate, "unit": "events/s",
           "workload": f"{ECMC_L}^4 fp64, {ch.n_chains} chains of {ECMC_LCORE}^4 blocks, beta={BETA}, theta_sample="
                       f"{ECMC_THETA:g}, refresh 50/15, epsilon_set 0.15",
           "lanes_per_chain": ch.lanes,
           "ms_per_step": ms / steps, "events_per_chain_per_step": events / steps / ch.n_chains,
           "lambda": ECMC_THETA * ch.n_chains * steps / lifts, "same_site_lift_frac": revs / lifts,
           "plaquette": plaq, "gpu_launches": launches,
           "e2e": {"value": e_ev / (e2e_s * steps), "unit": "events/s", "s_per_step": e2e_s,
                   "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 8,
                   "step": "random translation + qcb_ecmc_sample + qcb_plaquette to host, links resident"},
           "roofline": {"bound": "fp64 (latency and register bound in practice)", "achieved": flop,
                        "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                        "frac": flop / FP64_NOMINAL_TFLOPS if flop else None,
                        "peak_kind": "nominal (no FP64 peak is measured)", "flop_per_event": flop_per_event,
                        "dram_bytes_per_event_ncu": traffic.get("ecmc_dram_bytes_per_event")}}
    ch.close()
    f.close()
    if cpu:
        out["cpu_baseline"] = ecmc_cpu_reference(cpu_budget_s)
    return out


def ecmc_profile_case(ctx, lanes=3):
    """The small case an ncu capture of k_ecmc_sample runs on (a few GB on the device): a 42^4
    FP64 lattice as 14^4 blocks of 3^4 (38416 chains), Haar hot start + 5 heatbath sweeps, two
    sample calls (capture the second: -s 1 -c 1).  Three lanes per chain is the kernel shape the
    library picks for the 64^4 workload's 65536 chains; with one, the thread counters count each
    operation of the algorithm once (the chains take the same events at any lane count)."""
    import qcb

    f = qcb.GaugeField(ctx, (42,) * 4, "fp64", 18)
    f.hot_start(1)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, BETA, 5, 1, 3, 0))
    ch = qcb.EventChains(f, qcb.ecmc.params(beta=BETA, theta_sample=ECMC_THETA, l_core=3), 7)
    ch.lanes = lanes
    ch.sample((0, 1, 2, 0))
    ch.counters(reset=True)
    ch.sample((1, 1, 0, 2))
    events, lifts, revs = ch.counters(reset=True)
    out = {"case": "ecmc 42^4 l_core 3", "chains": ch.n_chains, "lanes_per_chain": ch.lanes,
           "events_second_call": events, "lifts": lifts}
    ch.close()
    f.close()
    return out


def serving_section(ctx, n_requests=100, rate=20.0, quantum_sweeps=2, quantum_steps=4):
    """Serving workload: a Poisson stream (mean `rate` req/s, stream seed 77) of 70% Wilson-flow
    measurements to t ~ U[1, 6] and 30% generate-N-sweeps jobs with N ~ U[10, 200]; sizes
    16^4 (0.4), 24^4 (0.3), 32^4 (0.2), 48^4 (0.1); beta ~ U[5.8, 6.3]; FP32 12-real.  The
    inputs are pre-thermalised on the device from per-request seeds before the stream starts
    (untimed setup) and stay resident.  Latency = completion - arrival on the server clock."""
    import threading

    import numpy as np

    import qcb

    rng = np.random.default_rng(77)
    gaps = rng.exponential(1.0 / rate, size=n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    kinds = rng.random(n_requests) < 0.7
    sizes = rng.choice([16, 24, 32, 48], p=[0.4, 0.3, 0.2, 0.1], size=n_requests)
    betas = rng.uniform(5.8, 6.3, size=n_requests)
    tflow = rng.uniform(1.0, 6.0, size=n_requests)
    nsw = rng.integers(10, 201, size=n_requests)
    lib = qcb._lib.lib()
    fields = []
    for k in range(n_requests):
        f = qcb.GaugeField(ctx, (int(sizes[k]),) * 4, "fp32", 12)
        f.hot_start(7000 + k)
        qcb._lib.check(lib.qcb_heatbath(f.h, float(betas[k]), 20, 1, 7000 + k, 0))
        fields.append(f)
    ctx.sync()
    srv = qcb.Server(ctx, "fp32", 12, hbm_budget=48 << 30, quantum_sweeps=quantum_sweeps, quantum_steps=quantum_steps)
    submit_t = {}

    def feeder():
        t_start = time.perf_counter()
        for k in range(n_requests):
            wait = arrivals[k] - (time.perf_counter() - t_start)
            if wait > 0:
                time.sleep(wait)
            if kinds[k]:
                jid = srv.submit_flow(fields[k], 0.02, int(round(tflow[k] / 0.02)))
            else:
                jid = srv.submit_sweeps(fields[k], float(betas[k]), int(nsw[k]), seed=7000 + k, sweep_offset=20)
            submit_t[jid] = k

    th = threading.Thread(target=feeder)
    th.start()
    th.join()
    srv.drain(3600)
    res = srv.poll(n_requests + 10)
    stats = srv.stats()
    srv.close()
    lat = np.array([r.finish_s - r.submit_s for r in res])
    wait = np.array([r.admit_s - r.submit_s for r in res])
    ok = all(r.status == 0 for r in res)
    span = max(r.finish_s for r in res) - min(r.submit_s for r in res)
    work_sites = sum((round(tflow[k] / 0.02) if kinds[k] else 0) * int(sizes[k]) ** 4 for k in range(n_requests))
    work_upd = sum((0 if kinds[k] else int(nsw[k])) * 4 * int(sizes[k]) ** 4 for k in range(n_requests))
    return {"workload": f"Poisson {rate} req/s, {n_requests} requests, 70% flow t~U[1,6], 30% N~U[10,200] sweeps, "
                        "sizes 16/24/32/48^4 (0.4/0.3/0.2/0.1), beta~U[5.8,6.3], fp32-12",
            "quantum": {"sweeps": quantum_sweeps, "rk3_steps": quantum_steps},
            "all_ok": ok, "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "admission_wait_p99_s": float(np.percentile(wait, 99)),
            "throughput_jobs_per_s": len(res) / span, "span_s": span,
            "flow_site_steps_per_s": work_sites / span, "hb_link_updates_per_s": work_upd / span,
            "offered_flow_site_steps": work_sites, "offered_link_updates": work_upd,
            "ticks": stats["ticks"], "max_active": stats["max_active"], "arena_peak_bytes": stats["arena_peak"]}


# ---------------------------------------------------------------------------------------
def large_workload(out_path=None) -> dict:
    """Large single lattice: 64^4 (67M links) at beta = 6.3, Haar hot start from seed 99,
    200 heatbath sweeps, then the flow to t = 6 (300 RK3 steps of 0.02) with Q/E every step,
    in FP32 12-real storage (3.2 GB) and in FP64 18-real storage (9.7 GB).  The FP32 flow
    runs on the FP64 heatbath output, so its Q/E errors against the FP64 flow are the
    precision of the FP32 flow alone.  Per-kernel HBM GB/s are algorithmic bytes over
    CUDA-event time per launch."""
    import numpy as np
    import torch

    import qcb
    from qcb import _lib

    Lg, beta, seed, sweeps, n_flow, eps = 64, 6.3, 99, 200, 300, 0.02
    dims, V = (Lg,) * 4, Lg ** 4
    ctx = qcb.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    lib = _lib.lib()
    gf = qcb.GradientFlow(eps)
    peak, peak_kind = peaks()

    def timed(fn, n=1, warm=0):
        for _ in range(warm):
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / n

    out = {"workload": "64^4 beta=6.3 hot start seed 99, 200 CM sweeps, flow to t=6 (300 RK3 eps=0.02, "
                       "Q/E every step)", "lattice": list(dims), "kernels": {}}
    res = {}
    fields = {}
    with Clocks(0) as clk:
        for prec, nr in (("fp64", 18), ("fp32", 12)):
            tag = f"{prec}-{nr}"
            f = qcb.GaugeField(ctx, dims, prec, nr)
            fields[tag] = f
            f.hot_start(seed)
            hb_ms = timed(lambda: _lib.check(lib.qcb_heatbath(f.h, beta, sweeps, 1, seed, 0)))
            plaq = qcb.observables.mean_plaquette_global(f)
            pass_ms = hb_ms / (8 * sweeps)
            hb_gbs = HB_BYTES[(prec, nr)] * V / 2 / (pass_ms / 1e3) / 1e9
            res[tag] = {"hb_total_s": hb_ms / 1e3, "hb_link_updates_per_s": sweeps * 4 * V / (hb_ms / 1e3),
                        "plaquette_after_hb": plaq, "device_bytes": f.device_bytes()}
            out["kernels"][f"hb_pass {tag}"] = {"ms_per_launch": pass_ms, "GB/s": hb_gbs, "frac": hb_gbs / peak}
        # the same configuration flowed in both storages
        fields["fp32-12"].copy_from(fields["fp64-18"])
        rec = {}
        for tag, f in fields.items():
            prec, nr = tag.split("-")
            nr = int(nr)
            scratch = qcb.GaugeField(ctx, dims, prec, nr)
            scratch.copy_from(f)
            rk3_ms = timed(lambda: _lib.check(lib.qcb_flow_steps(scratch.h, eps, 1)), 5, warm=2)
            qe_ms = timed(lambda: qcb.observables.topo_q_e_clover_global(scratch), 3, warm=1)
            scratch.close()
            qcb.observables.topo_charge_flowed(f, gf, 1, 1)  # allocates the flow work space untimed
            fl_gbs = FLOW_BYTES[(prec, nr)] * V / (rk3_ms / 1e3) / 1e9
            out["kernels"][f"flow RK3 step {tag}"] = {"ms_per_step": rk3_ms, "GB/s": fl_gbs, "frac": fl_gbs / peak}
            out["kernels"][f"clover Q/E {tag}"] = {"ms_per_measurement": qe_ms}
            t_ms = timed(lambda: rec.__setitem__(tag, qcb.observables.topo_charge_flowed(f, gf, n_flow, 1)))
            res[tag]["flow_total_s"] = t_ms / 1e3
            res[tag]["flow_site_steps_per_s"] = n_flow * V / (t_ms / 1e3)
            res[tag]["Q_t6"] = float(rec[tag][-2])
            res[tag]["E_t6"] = float(rec[tag][-1])
    r64, r32 = rec["fp64-18"].reshape(-1, 3), rec["fp32-12"].reshape(-1, 3)
    out["results"] = res
    out["precision"] = {"dQ_max": float(np.abs(r32[:, 1] - r64[:, 1]).max()),
                        "dE_rel_max": float((np.abs(r32[:, 2] - r64[:, 2]) / np.abs(r64[:, 2])).max()),
                        "same_input": "FP64 heatbath output, flowed in FP32-12 and in FP64-18"}
    out["speedup_fp32_over_fp64"] = {
        "hb": res["fp32-12"]["hb_link_updates_per_s"] / res["fp64-18"]["hb_link_updates_per_s"],
        "flow_with_qe": res["fp32-12"]["flow_site_steps_per_s"] / res["fp64-18"]["flow_site_steps_per_s"]}
    out["peak"] = {"hbm_gbs": peak, "kind": peak_kind}
    out["clocks"] = clk.summary()
    for f in fields.values():
        f.close()
    ctx.close()
    if out_path:
        Path(out_path).write_text(json.dumps(out, indent=1) + "\n")
    return out


# ---------------------------------------------------------------------------------------
PLAIN_INPUT = """L_core=8
n_core_dims=1
cold_start=true
seed=1234
N_shift_therm = 0
N_shift=200
N_switch_eo=1
beta = 6.0
N_sweeps = 1
N_hits = 1
N_shift_plaquette = 1
topo = false
run_name = plain8
run_dir = {run_dir}
save_each_shifts = 1000
"""


def _plain_cpu(_):
    """The plain-method workload with the reference schedule on one host core: 200 shifts of
    one sweep with the plaquette each, then 50 RK3 flow steps (N_rk_steps = 1) with Q/E."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.select_build("fast")
    t = time.perf_counter()
    chain = oracle.RefChain(8, 1234, True)
    chain.run(6.0, 200, 1, 1)
    oracle.flow_measure(chain.links(), (8, 8, 8, 8), 0.02, 50, 1)
    return time.perf_counter() - t


def plain_section():
    """Plain method (8^4, beta = 6.0, cold start, seed 1234, 200 sweeps with the plaquette each,
    then the flow on the final configuration, eps = 0.02, 50 steps, FP64) end to end through the
    drop-in driver gauge_hb_ncb (process start, parsing, device work, the output files), and
    the same workload with the reference schedule on one host core (the oracle port)."""
    import tempfile

    driver = ROOT / "ecmc-qncb_b200" / "bin" / "gauge_hb_ncb"
    with tempfile.TemporaryDirectory() as d:
        inp = Path(d) / "in.txt"
        inp.write_text(PLAIN_INPUT.format(run_dir=Path(d) / "data"))
        t = time.perf_counter()
        r = subprocess.run([str(driver), str(inp)], capture_output=True, text=True, timeout=600)
        t_drv = time.perf_counter() - t
        ok = r.returncode == 0
        # the flow on the saved configuration, through the library (t = 0 .. 0.98)
        import qcb

        ctx = qcb.Context(0)
        f = qcb.GaugeField(ctx, (8, 8, 8, 8))
        f.load_ildg(Path(d) / "data" / "plain8" / "plain8")
        t = time.perf_counter()
        tqe = qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), 50, 1)
        t_flow = time.perf_counter() - t
        f.close()
        ctx.close()
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.build_fast()
    with mp.get_context("spawn").Pool(1) as pool:
        t_cpu = pool.map(_plain_cpu, [0])[0]
    return {"workload": "8^4 beta=6.0 cold start seed 1234, 200 sweeps + plaquette each; flow eps=0.02, 50 steps",
            "driver_ok": ok, "driver_wall_s": t_drv, "flow_wall_s": t_flow, "Q_final": float(tqe[-2]),
            "cpu_reference_schedule_1core_s": t_cpu,
            "note": "driver wall time includes process start, CUDA context creation and the output files"}


# ---------------------------------------------------------------------------------------
def _ref_worker(args):
    """One 'rank' of the reference schedule on a block of edge lb: sweeps then flow."""
    lb, sweeps, rk3, seed = args
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.select_build("fast")
    chain = oracle.RefChain(lb, seed, False)
    t = time.perf_counter()
    chain.run(BETA, sweeps, 1, 1)  # shift + sweep + plaquette per shift
    t_hb = time.perf_counter() - t
    dims = (lb,) * 4
    u = chain.links()
    t = time.perf_counter()
    oracle.flow_steps(u, dims, FLOW_EPS, rk3)
    t_flow = time.perf_counter() - t
    return t_hb, chain.updates_per_sweep() * sweeps, t_flow, lb ** 4 * rk3


def cpu_baseline(sweeps: int = 1, rk3: int = 1, block: int = 16):
    """Reference algorithm on the host cores: one process per hardware thread (the reference
    runs one MPI rank per core), each on a 16^4 block as in the reference's 2^4-rank
    decomposition of 32^4; the rates are summed over the processes.  The oracle runs as its
    timing build: -O3 for the host's instruction set (the reference's release flags,
    CMakeLists.txt:88-102), complex products without __muldc3, and a neighbour table as the
    reference keeps one (GeometryCB.cpp:10-31)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.build_fast()
    cores = min(64, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1))
    with mp.get_context("spawn").Pool(cores) as pool:
        t = time.perf_counter()
        res = pool.map(_ref_worker, [(block, sweeps, rk3, 100 + r) for r in range(cores)])
        wall = time.perf_counter() - t
    hb_rate = sum(r[1] for r in res) / max(r[0] for r in res)
    flow_rate = sum(r[3] for r in res) / max(r[2] for r in res)
    return {"value": hb_rate, "unit": "link-updates/s", "cores": cores, "kind": "port",
            "flow_value": flow_rate, "flow_unit": "site-steps/s", "wall_s": wall,
            "sample": f"{cores} processes x ({sweeps} reference shift+sweep on a {block}^4 block with frozen "
                      f"links, then {rk3} RK3 flow step); link-updates counted as 4L(L-1)^3 per sweep; "
                      f"oracle built -O3 -march=native -fcx-limited-range with a neighbour table"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the batching and serving sections")
    ap.add_argument("--profile", action="store_true",
                    help="run only warmup + steps of the workload (for ncu); print launch counts")
    ap.add_argument("--storage", choices=["fp32-12", "fp64-18"], default="fp32-12")
    ap.add_argument("--ecmc-lanes", type=int, choices=[1, 3, 6], default=3,
                    help="lanes per chain of the event-chain profile case (1: no lane repeats the "
                         "chain's serial work, so thread counters count the algorithm's operations)")
    ap.add_argument("--workload", choices=["precision", "large", "batch", "ecmc"], default="precision",
                    help="large: the 64^4 single-lattice workload; batch: the 64-lattice batching workload "
                         "alone; ecmc: the event-chain workload alone; each printed as its own JSON object")
    ap.add_argument("--out", default=None, help="also write the large-workload JSON to this path")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank, world, local_rank = replicas.env_rank()

    if args.impl == "reference":
        if rank != 0:
            return 0
        runs = []
        for _ in range(args.warmup + args.steps):
            runs.append(cpu_baseline())
        timed = runs[args.warmup:]
        v = statistics.mean(r["value"] for r in timed)
        cb = dict(timed[0])
        cb["value"] = v
        out = {"impl": "reference", "metric": METRIC, "value": v, "unit": "link-updates/s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": "precision 32^4 (reference schedule, 16^4 blocks per core), beta=6.0, "
                                      "hot start; sweep and RK3 flow rates", "lattice": [L, L, L, L]},
               "flow": {"value": statistics.mean(r["flow_value"] for r in timed), "unit": "site-steps/s"},
               "ecmc": ecmc_cpu_reference(),
               "cpu_baseline": cb,
               "e2e": {"value": v, "unit": "link-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return 0

    if args.workload == "large":
        if rank == 0:
            print(json.dumps(large_workload(args.out)))
        return 0
    if args.workload == "batch":
        if rank == 0:
            import torch

            import qcb
            from qcb import _lib

            ctx = qcb.Context(0)
            stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
            print(json.dumps(batch_section(ctx, _lib.lib(), stream)))
            ctx.close()
        return 0
    if args.workload == "ecmc":
        if rank == 0:
            import qcb

            ctx = qcb.Context(0)
            if args.profile:
                print(json.dumps(ecmc_profile_case(ctx, args.ecmc_lanes)))
            else:
                print(json.dumps(ecmc_section(ctx, steps=args.steps, warmup=args.warmup,
                                              cpu=not args.no_cpu_baseline)))
            ctx.close()
        return 0
    dist = replicas.init("nccl", timeout_s=300)
    if args.profile:
        return profile_steps(args)
    try:
        res = run_ours(args, rank, world, local_rank, dist)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline()
        if rank == 0:
            print(json.dumps(res))
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
