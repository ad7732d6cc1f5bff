"""Benchmark of the B200 patch-update path (cell-updates/s), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dam|dam-uniform|swirl|shockbubble] [--precision fp64|fp32wave]
                    [--pstar pvrs|mlp]

Default workload (the configuration the metric is quoted on): 2D shallow water,
radial dam break on [-1,1]^2, adaptive quadtree levels 3-7, 16x16 patches, mbc=2,
Roe solver with Harten-Hyman fix, MC limiter, subcycled levels, time sync on,
regrid every 4 coarse steps (refine where |grad h| dx > 0.01, coarsen below
0.002).  Synthetic initial data of the reference app (no dataset is involved).
One "step" is one coarse step (fclaw2d_advance_all_levels: every level
subcycled, ghost fill, update, time sync), replayed as one CUDA graph per forest.
The regrid every 4 coarse steps runs between timed steps: its host wall time is
reported separately and excluded from the device time, while the graph capture of
the new forest falls inside the next timed step.

value      : interior cell updates of all ranks / max over ranks of the device time
             of the timed steps (CUDA events on the solver's stream).  L2 (126 MB)
             is flushed between timed steps by writing a 512 MB buffer.
e2e        : the same metric through the C ABI with host buffers: per step
             fc2d_b200_set_q from pinned host memory, fc2d_b200_advance,
             fc2d_b200_get_q back to pinned host memory (wall clock).
roofline   : the fused update kernel, algorithmic bytes per interior cell
             8*(2*meqn + maux) over its event-timed launch durations, against the
             measured HBM copy bandwidth in MEASURED_PEAKS.json.
cpu_baseline: the FP64 CPU oracle (OpenMP over patches, all host cores) on a bounded
             sample of the same workload.
--impl reference times the reference's CPU implementation of the path: the
reference's Fortran cannot be compiled here, so it is the C restatement (oracle)
with all host threads, on the same config.
Multi-GPU (torchrun): every rank runs its own instance of the workload
(independent simulations, weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "dam": dict(name="radialdam_sw_amr_l3-7_16x16", mx=16, my=16, minlevel=3, maxlevel=7, subcycle=1,
                time_sync=1, regrid_interval=4, spinup=16),
    "dam-uniform": dict(name="radialdam_sw_uniform_l7_16x16", mx=16, my=16, minlevel=7, maxlevel=7, subcycle=0,
                        time_sync=0, regrid_interval=0, spinup=2),
    "swirl": dict(name="swirl_advection_uniform_l4_32x32", mx=32, my=32, minlevel=4, maxlevel=4, subcycle=0,
                  time_sync=0, regrid_interval=0, spinup=0),
    "shockbubble": dict(name="euler_shockbubble_amr_l4-8_16x16", mx=16, my=16, minlevel=4, maxlevel=8, subcycle=1,
                        time_sync=1, regrid_interval=4, spinup=8),
}


def _peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per interior
# cell-update of the fused update kernel, from one ncu --set full capture of a
# 16384-patch launch (radial dam, uniform level 7, 16x16 patches, mbc 2); the
# summaries are profiles/step2_sw_roe_16x16_<precision>.md.  A launch of n
# patches moves n * 256 times this.
DRAM_BYTES_PER_CELL = {
    ("sw_roe_16x16", "fp32wave"): (158.340352e6 + 89.620224e6) / (16384 * 256),
    ("sw_roe_16x16", "fp64"): (159.835648e6 + 243.607808e6) / (16384 * 256),
}


def _traffic_per_launch(wl: dict, precision: str, cells_per_launch: float):
    if wl["name"].startswith("swirl") or wl["mx"] != 16:
        return None
    b = DRAM_BYTES_PER_CELL.get(("sw_roe_16x16", precision))
    return None if b is None else b * cells_per_launch


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms (GPU selected by UUID)."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) > 8:
                for k, n in enumerate(names):
                    if r[5 + k] == "Active":
                        reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _preset(wl: dict):
    from forestclaw_b200 import problems
    if wl["name"].startswith("swirl"):
        return problems.SWIRL
    if wl["name"].startswith("euler"):
        return problems.SHOCKBUBBLE
    return problems.DAM


def _options(wl: dict, precision: str):
    import forestclaw_b200 as fb
    from forestclaw_b200 import problems
    kw = {k: wl[k] for k in ("mx", "my", "minlevel", "maxlevel", "subcycle", "time_sync")}
    gc = problems.options(_preset(wl), **kw)
    gc.precision = fb.PREC_FP32WAVE if precision == "fp32wave" else fb.PREC_FP64
    return _preset(wl), gc


def _initial_dt(wl: dict, prob) -> float:
    from forestclaw_b200.problems import SHOCKBUBBLE, SWIRL, swirl_dt
    if prob is SWIRL:
        return swirl_dt(wl["mx"], wl["minlevel"])
    if prob is SHOCKBUBBLE:
        # CFL ~0.8 for the fastest initial wave, the sound speed sqrt(1.4/0.138) = 3.19
        # inside the bubble, on the coarsest level
        return 0.8 * (1.0 / (wl["mx"] << wl["minlevel"])) / 3.2
    # coarse-level dt for CFL ~0.9 at the initial state (max speed sqrt(g*2))
    dx = 2.0 / (wl["mx"] << wl["minlevel"])
    return 0.9 * dx / (2.0 ** 0.5 * 1.5)


def cpu_sample(wl: dict, precision: str, max_seconds: float = 20.0, threads: int = 0):
    """Time the FP64 CPU oracle on the workload's initial forest for a bounded number of steps."""
    from oracle import pyoracle as po
    from tests.cases import DAM, SHOCKBUBBLE, SWIRL, make
    prob = _preset(wl)
    kw = {k: wl[k] for k in ("mx", "my", "minlevel", "maxlevel", "subcycle", "time_sync")}
    case = SWIRL if wl["name"].startswith("swirl") else SHOCKBUBBLE if wl["name"].startswith("euler") else DAM
    oc, _ = make(case, nthreads=threads, **kw)
    s = po.OracleSim(oc)
    s.initialize()
    dt = _initial_dt(wl, prob)
    t, steps = 0.0, 0
    c0 = s.cell_updates
    t0 = time.perf_counter()
    while True:
        cfl = s.advance(t, dt)
        t += dt
        steps += 1
        if wl["time_sync"]:
            dt *= 0.9 / cfl
        if time.perf_counter() - t0 > max_seconds or steps >= 200:
            break
    el = time.perf_counter() - t0
    cells = s.cell_updates - c0
    ncores = threads or os.cpu_count()
    return {"value": cells / el, "unit": "cell-updates/s", "cores": ncores, "kind": "port",
            "sample": f"{steps} coarse steps of {wl['name']} from the initial refinement "
                      f"({s.num_patches} patches, {cells:.3e} cell updates, {el:.1f} s, FP64 C oracle, OpenMP)"}


def run_reference(args, wl, rank, world):
    if rank != 0:
        return 0
    cpu = cpu_sample(wl, args.precision, max_seconds=max(5.0, 25.0 / max(args.steps, 1)), threads=0)
    line = {
        "metric": "cell-updates/s", "value": cpu["value"], "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["name"], "l2": "n/a (CPU)"}, "impl": "reference",
        "cpu_baseline": cpu,
        "e2e": {"value": cpu["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def train_pstar_mlp(wl, prob, device, nsamples, epochs):
    """Sample interface states uniformly from the FP64 run of the workload over
    its spin-up steps (seed 0), train the p*-seed network on the GPU on the
    states its gate selects, and return it with a summary (not timed)."""
    import forestclaw_b200 as fb
    from forestclaw_b200 import problems
    kw = {k: wl[k] for k in ("mx", "my", "minlevel", "maxlevel", "subcycle", "time_sync")}
    g = fb.Solver(problems.options(prob, device=device, **kw))
    g.initialize()
    t0 = time.perf_counter()
    t, dt = 0.0, _initial_dt(wl, prob)
    snaps = max(wl["spinup"], 1)
    per = max(nsamples // snaps, 1)
    parts = []
    for n in range(snaps):
        parts.append(g.sample_interfaces(per, seed=n))
        cfl = g.advance(t, dt)
        t += dt
        dt *= 0.9 / cfl
        if wl["regrid_interval"] and (n + 1) % wl["regrid_interval"] == 0:
            g.regrid()
    g.close()
    prim = np.concatenate(parts)
    rl, ul, pl, rr, ur, pr = prim.T
    pb, rb = 0.5 * (pl + pr), 0.5 * (rl + rr)
    strength = np.abs(pr - pl) / pb + np.abs(ur - ul) / np.sqrt(pb / rb)
    strong = prim[strength > 0.2]
    m = fb.PStarMLP(device=device, seed=0)
    info = {"samples": int(len(prim)), "gated_samples": int(len(strong)), "epochs": epochs}
    if len(strong) >= 256:
        m.set_data(strong, gamma=1.4, tol=1e-10)
        h0 = m.newton_histogram(False)
        info["loss"] = m.train(epochs=epochs, batch=4096, lr=2e-3, seed=0)
        h1 = m.newton_histogram(True)
        mean = lambda h: float((np.arange(32) * h).sum() / max(h.sum(), 1))
        info["gated_newton_mean_pvrs"] = mean(h0)
        info["gated_newton_mean_mlp"] = mean(h1)
    info["train_s"] = time.perf_counter() - t0
    return m, info


def error_vs_fp64(wl, prob, device, mlp, steps=8):
    """Relative L1 error per field of the FP32-wave run against the FP64 run
    (bitwise equal to the CPU oracle) from the same initial forest, no regrid."""
    import forestclaw_b200 as fb
    from forestclaw_b200 import problems
    kw = {k: wl[k] for k in ("mx", "my", "minlevel", "maxlevel", "subcycle", "time_sync")}
    a = fb.Solver(problems.options(prob, device=device, **kw))
    b = fb.Solver(problems.options(prob, device=device, precision=fb.PREC_FP32WAVE, **kw))
    a.initialize(); b.initialize()
    if mlp is not None:
        b.set_pstar_seed(mlp)
    t, dt = 0.0, _initial_dt(wl, prob)
    for _ in range(steps):
        ca = a.advance(t, dt)
        b.advance(t, dt)
        t += dt
        dt *= 0.9 / ca
    qa, qb = a.get_q()[:, :, 2:-2, 2:-2], b.get_q()[:, :, 2:-2, 2:-2]
    a.close(); b.close()
    out = []
    for m in range(qa.shape[1]):
        den = np.abs(qa[:, m]).sum() if np.abs(qa[:, m]).sum() > 0 else np.abs(qa[:, 0]).sum()
        out.append(float(np.abs(qa[:, m] - qb[:, m]).sum() / den))
    return {"steps": steps, "l1_rel_per_field": out}


def run_ours(args, wl, rank, world, local_rank):
    import torch
    import forestclaw_b200 as fb
    torch.cuda.set_device(local_rank)
    prob, gc = _options(wl, args.precision)
    gc.device = local_rank
    mlp, mlp_info = None, None
    if args.pstar == "mlp":
        mlp, mlp_info = train_pstar_mlp(wl, prob, local_rank, args.mlp_samples, args.mlp_epochs)
    g = fb.Solver(gc)
    g.initialize()
    if mlp is not None:
        g.set_pstar_seed(mlp)
    dt = _initial_dt(wl, prob)
    t = 0.0
    # spin-up with regrid so the timed forest is representative (not timed)
    regrid_ms = []
    for n in range(wl["spinup"]):
        cfl = g.advance(t, dt)
        t += dt
        if wl["time_sync"]:
            dt *= 0.9 / cfl
        if wl["regrid_interval"] and (n + 1) % wl["regrid_interval"] == 0:
            t0 = time.perf_counter()
            g.regrid()
            regrid_ms.append((time.perf_counter() - t0) * 1e3)
    for _ in range(args.warmup):
        cfl = g.advance(t, dt)
        t += dt
        if wl["time_sync"]:
            dt *= 0.9 / cfl
    g.synchronize()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # timed steps: each coarse step replays the CUDA graph of the current forest;
    # the regrid every regrid_interval steps runs between timed steps (host wall
    # clock, reported separately), and the first step on a new forest includes
    # its graph capture
    g.set_timing(False)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    props = torch.cuda.get_device_properties(local_rank)
    clk = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local_rank))
    if rank == 0:
        clk.start()
    step_ms, cells, launches, timed_regrid_ms = [], 0.0, 0, []
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        c0 = g.cell_updates
        g.event_record(0)
        cfl = g.advance(t, dt)
        g.event_record(1)
        step_ms.append(g.event_elapsed(0, 1))
        cells += g.cell_updates - c0
        launches += g.last_update_stats()["total_launches"]
        t += dt
        if wl["time_sync"]:
            dt *= 0.9 / cfl
        if wl["regrid_interval"] and (k + 1) % wl["regrid_interval"] == 0:
            t0 = time.perf_counter()
            g.regrid()
            timed_regrid_ms.append((time.perf_counter() - t0) * 1e3)
    torch.cuda.synchronize()
    clocks = clk.stop() if rank == 0 else None
    # roofline pass (not part of the timed steps): the same steps launched
    # eagerly with a CUDA event pair around every update launch
    g.set_timing(True)
    upd_ms, upd_bytes, upd_launches = 0.0, 0.0, 0
    for k in range(max(2, min(args.steps, 4))):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        g.advance(t, dt)
        st = g.last_update_stats()
        upd_ms += st["update_ms"]
        upd_bytes += st["update_bytes"]
        upd_launches += st["update_launches"]
        t += dt
    g.set_timing(False)
    total_ms = float(np.sum(step_ms))
    if world > 1:
        tt = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(tt.item())
        cc = torch.tensor([cells], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(cc, op=torch.distributed.ReduceOp.SUM)
        cells_all = float(cc.item())
    else:
        cells_all = cells
    value = cells_all / (total_ms * 1e-3)
    # ---- end to end through the C ABI with pinned host buffers ----
    nq = g.num_patches * gc.meqn * (gc.mx + 2 * gc.mbc) * (gc.my + 2 * gc.mbc)
    hq = torch.empty(nq, dtype=torch.float64, pin_memory=True)
    g.get_q_ptr(hq.data_ptr())
    e2e_steps = max(2, min(args.steps, 10))
    torch.cuda.synchronize()
    te0 = time.perf_counter()
    e2e_cells = 0.0
    for _ in range(e2e_steps):
        c0 = g.cell_updates
        g.set_q_ptr(hq.data_ptr())
        g.advance(t, dt)
        g.get_q_ptr(hq.data_ptr())
        e2e_cells += g.cell_updates - c0
        t += dt
    e2e_s = time.perf_counter() - te0
    if world > 1:
        te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(te.item())
        e2e_cells *= world
    e2e = {"value": e2e_cells / e2e_s, "unit": "cell-updates/s", "h2d_bytes_per_step": nq * 8,
           "d2h_bytes_per_step": nq * 8}
    if rank != 0:
        return 0
    peaks = _peaks()
    achieved = upd_bytes / (upd_ms * 1e-3) / 1e9 if upd_ms > 0 else None
    per_launch_bytes = upd_bytes / max(upd_launches, 1)
    traffic = _traffic_per_launch(wl, args.precision, per_launch_bytes / (8 * (2 * gc.meqn + gc.maux)))
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": (achieved / peaks["hbm_gbs"]) if achieved else None, "traffic": traffic,
                "peak_source": peaks["source"], "kernel": "step2 fused update",
                "algorithmic_bytes_per_launch": per_launch_bytes,
                "bytes_per_cell_update": 8 * (2 * gc.meqn + gc.maux),
                "avg_launch_ms": upd_ms / max(upd_launches, 1)}
    cpu = cpu_sample(wl, args.precision, max_seconds=args.cpu_seconds) if args.cpu_seconds > 0 else None
    err = error_vs_fp64(wl, prob, local_rank, mlp) if args.precision == "fp32wave" else None
    newton = None
    if wl["name"].startswith("euler"):
        h = g.newton_histogram()
        newton = {"mean_iterations": float((np.arange(32) * h).sum() / max(h.sum(), 1)),
                  "histogram": [int(v) for v in h[:12]], "pstar_start": args.pstar, "mlp": mlp_info}
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-waves/f64-q",
        "data": "synthetic (reference app initial data)",
        "config": {"workload": wl["name"], "patches": g.num_patches, "precision": args.precision,
                   "cells_per_step": cells / args.steps,
                   "l2": "flushed between timed steps (512 MB write)",
                   "launch": "CUDA graph per coarse step (captured once per forest)",
                   "regrid": (f"every {wl['regrid_interval']} coarse steps between timed steps, excluded from "
                              "the device time" if wl["regrid_interval"] else "none"),
                   "regrids_in_timed_loop": len(timed_regrid_ms),
                   "regrid_ms_median": float(np.median(regrid_ms + timed_regrid_ms)) if regrid_ms else None},
        "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
        "error_vs_fp64": err, "newton": newton,
        "gpu_launches": launches, "update_launches": upd_launches,
    }
    print(json.dumps(line), flush=True)
    g.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dam", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32wave"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--pstar", default="pvrs", choices=["pvrs", "mlp"],
                    help="Euler: Newton start of the exact solver (mlp: trained on the FP64 run first)")
    ap.add_argument("--mlp-samples", type=int, default=1_000_000)
    ap.add_argument("--mlp-epochs", type=int, default=20)
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, wl, rank, world)
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return run_ours(args, wl, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
