"""Benchmark of the B200 patch-update path (cell-updates/s), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dam|dam-uniform|swirl|shockbubble|batch] [--precision fp32wave|fp64]
                    [--pstar pvrs|mlp] [--no-fp64-compare] [--no-autotune] [--variant V]

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

The FP32-wave form (FP32 waves and limiter, FP64 q, fluxes and registers) is the
default; the same run times the plain FP64 kernel (bitwise equal to the CPU
oracle) on the same workload and protocol ("fp64_kernel", with the speed-up) and
states the FP32 error against FP64 ("error_vs_fp64").  After the spin-up the
autotuner picks the patch-to-CTA variant of each arm ("patch_to_cta").
Workload "batch": 64 seeded tsunami instances (f-waves with bathymetry), one
solver per patch size (8x8, 16x16), both stepping concurrently on their own streams.

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
Multi-GPU (torchrun): a single-forest workload is one forest partitioned over the
ranks along the space-filling curve (fc2d_b200_set_partition: each rank updates
its own patches, a halo of q, qlast and registers moves over NCCL before each ghost
update, the CFL number, regrid tags and mass are reduced; strong scaling), or with
--no-partition one replica per rank (weak scaling).  The batch workload gives each
rank its own instances (weak scaling, no data-path collective).
e2e, per step: set_q from pinned host memory, advance, get_q back; every
regrid_interval steps the regrid (and a get_q of the new forest) inside the
wall-clock region.
error_vs_oracle: the FP32-wave run against the FP64 CPU oracle from the same
initial forest (per-field relative L1 and Linf, mass).
The default line carries a second measurement under "secondary": the shock-bubble
(Euler, exact solver) with the learned p* start (--no-secondary skips it).
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
    "sphere": dict(name="sphere_advection_cubed_l4-9_32x32", mx=32, my=32, minlevel=4, maxlevel=9, subcycle=1,
                   time_sync=0, adapt_dt=1, regrid_interval=4, spinup=4, cpu_maxlevel=6),
    "batch": dict(name="tsunami_batch_64_instances_8x8_16x16", batch=True, instances=64, mx=16, my=16,
                  minlevel=0, maxlevel=0, subcycle=1, time_sync=1, regrid_interval=4, spinup=8),
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
    if wl["name"].startswith("sphere"):
        return problems.SPHERE
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
    from forestclaw_b200.problems import SHOCKBUBBLE, SPHERE, SWIRL, swirl_dt
    if prob is SWIRL:
        return swirl_dt(wl["mx"], wl["minlevel"])
    if prob is SPHERE:
        # CFL ~0.45 on the coarsest level: speed omega R = 2 pi, cells of (pi/2)/(mx 2^l)
        # radians at a face centre, about half that near the cube corners
        return 0.9 * 0.5 * (0.5 * np.pi / (wl["mx"] << wl["minlevel"])) / (2.0 * np.pi)
    if prob is SHOCKBUBBLE:
        # CFL ~0.8 for the fastest initial wave, the sound speed sqrt(1.4/0.138) = 3.19
        # inside the bubble, on the coarsest level
        return 0.8 * (1.0 / (wl["mx"] << wl["minlevel"])) / 3.2
    # coarse-level dt for CFL ~0.9 at the initial state (max speed sqrt(g*2))
    dx = 2.0 / (wl["mx"] << wl["minlevel"])
    return 0.9 * dx / (2.0 ** 0.5 * 1.5)


def cpu_sample(wl: dict, precision: str, max_seconds: float = 20.0, threads: int = 0, steps: int = 200,
               warmup: int = 0):
    """The FP64 CPU oracle on the workload after the GPU arm's spin-up protocol (spinup
    coarse steps with a regrid every regrid_interval, untimed), then `warmup` untimed and
    up to `steps` timed coarse steps on the spun-up forest, stopping early once
    max_seconds of timed work are done.  Timed: fclaw2d_advance_all_levels only; the
    regrids between timed steps are excluded, as in the GPU arm."""
    from oracle import pyoracle as po
    from tests.cases import DAM, SHOCKBUBBLE, SWIRL, make
    from tests.cases import SPHERE
    prob = _preset(wl)
    kw = {k: wl[k] for k in ("mx", "my", "minlevel", "maxlevel", "subcycle", "time_sync")}
    if "cpu_maxlevel" in wl:
        kw["maxlevel"] = wl["cpu_maxlevel"]
    case = (SWIRL if wl["name"].startswith("swirl") else SHOCKBUBBLE if wl["name"].startswith("euler")
            else SPHERE if wl["name"].startswith("sphere") else DAM)
    oc, _ = make(case, nthreads=threads, **kw)
    s = po.OracleSim(oc)
    s.initialize()
    adapt = wl.get("adapt_dt", wl["time_sync"])
    ri = wl["regrid_interval"]
    t, dt = 0.0, _initial_dt(wl, prob)
    ts0 = time.perf_counter()
    for n in range(wl["spinup"]):
        cfl = s.advance(t, dt)
        t += dt
        if adapt:
            dt *= 0.9 / cfl
        if ri and (n + 1) % ri == 0:
            s.regrid()
    for _ in range(warmup):
        cfl = s.advance(t, dt)
        t += dt
        if adapt:
            dt *= 0.9 / cfl
    spin_s = time.perf_counter() - ts0
    step_s, cells = [], 0.0
    for k in range(steps):
        c0 = s.cell_updates
        t0 = time.perf_counter()
        cfl = s.advance(t, dt)
        step_s.append(time.perf_counter() - t0)
        cells += s.cell_updates - c0
        t += dt
        if adapt:
            dt *= 0.9 / cfl
        if sum(step_s) > max_seconds:
            break
        if ri and (k + 1) % ri == 0:
            s.regrid()
    el = sum(step_s)
    ncores = threads or os.cpu_count()
    return {"value": cells / el, "unit": "cell-updates/s", "cores": ncores, "kind": "port",
            "ms_per_step": 1e3 * el / len(step_s), "steps_timed": len(step_s),
            "sample": f"{len(step_s)} timed coarse steps of {wl['name']}"
                      + (f" with maxlevel {wl['cpu_maxlevel']} (the host metric at the full maxlevel is too slow)"
                         if "cpu_maxlevel" in wl else "")
                      + f" after the GPU arm's spin-up ({wl['spinup']} steps, regrid every {ri}; {spin_s:.1f} s, "
                        f"untimed), regrid between timed steps excluded ({s.num_patches} patches at the end, "
                        f"{cells:.3e} cell updates in {el:.1f} s, FP64 C oracle, OpenMP)"}


def run_reference(args, wl, rank, world):
    if rank != 0:
        return 0
    if wl.get("batch"):
        cpu = cpu_sample_batch(wl, max_seconds=max(5.0, 25.0 / max(args.steps, 1)), threads=0)
        steps, ms = args.steps, None
    else:
        # the same forest protocol as the GPU arm, bounded to ~90 s of timed CPU work
        cpu = cpu_sample(wl, args.precision, max_seconds=90.0, threads=0, steps=args.steps, warmup=args.warmup)
        steps, ms = cpu["steps_timed"], cpu["ms_per_step"]
    line = {
        "metric": "cell-updates/s", "value": cpu["value"], "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": steps, "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True,
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
        # momenta are relative to the density (depth): they vanish where the flow is at rest
        mom = qa.shape[1] >= 3 and m in (1, 2)
        den = np.abs(qa[:, 0 if mom else m]).sum()
        out.append(float(np.abs(qa[:, m] - qb[:, m]).sum() / den))
    return {"steps": steps, "l1_rel_per_field": out,
            "normalisation": "sum |q_m| per field; momenta by the sum of the density (depth)"}


def error_vs_oracle(wl, prob, device, mlp, steps=8):
    """Per-field error of the FP32-wave run against the FP64 CPU oracle from the same
    initial forest: `steps` coarse steps with the oracle's CFL setting both dt
    schedules, no regrid.  Relative L1 = sum |dq| area / sum |q| area and relative
    Linf = max |dq| / max |q| over interior cells (momenta normalised by the depth or
    density, which vanish nowhere), and the relative difference of the mass (field 0)."""
    import forestclaw_b200 as fb
    from forestclaw_b200 import problems
    from oracle import pyoracle as po
    from tests.cases import DAM, SHOCKBUBBLE, make
    case = SHOCKBUBBLE if wl["name"].startswith("euler") else DAM
    kw = {k: wl[k] for k in ("mx", "my", "minlevel", "maxlevel", "subcycle", "time_sync")}
    oc, _ = make(case, **kw)
    o = po.OracleSim(oc)
    o.initialize()
    b = fb.Solver(problems.options(prob, device=device, precision=fb.PREC_FP32WAVE, **kw))
    b.initialize()
    if mlp is not None:
        b.set_pstar_seed(mlp)
    t, dt = 0.0, _initial_dt(wl, prob)
    for _ in range(steps):
        co = o.advance(t, dt)
        b.advance(t, dt)
        t += dt
        dt *= 0.9 / co
    qo, qb = o.get_q()[:, :, 2:-2, 2:-2], b.get_q()[:, :, 2:-2, 2:-2]
    mo, mb = o.mass(), b.mass()
    lev = o.patch_info()[:, 0]
    b.close()
    area = ((prob["bx"] - prob["ax"]) / (wl["mx"] * (prob.get("mi", 1) * 2.0 ** lev))) * \
           ((prob["by"] - prob["ay"]) / (wl["my"] * (prob.get("mj", 1) * 2.0 ** lev)))
    w = area[:, None, None]
    l1, linf = [], []
    for m in range(qo.shape[1]):
        mom = qo.shape[1] >= 3 and m in (1, 2)
        ref = qo[:, 0 if mom else m]
        d = np.abs(qo[:, m] - qb[:, m])
        l1.append(float((d * w).sum() / (np.abs(ref) * w).sum()))
        linf.append(float(d.max() / np.abs(ref).max()))
    return {"against": "FP64 CPU oracle", "steps": steps, "patches": int(len(lev)), "l1_rel_per_field": l1,
            "linf_rel_per_field": linf, "mass_rel_diff": float(abs(mb[0] - mo[0]) / abs(mo[0])),
            "normalisation": "per field sum |q_m| area (L1) and max |q_m| (Linf); momenta by the depth/density"}


def _spinup(g, wl, t, dt, steps):
    """Untimed coarse steps with the workload's regrid interval; returns (t, dt, regrid ms list)."""
    regrid_ms = []
    for n in range(steps):
        cfl = g.advance(t, dt)
        t += dt
        if wl.get("adapt_dt", wl["time_sync"]):
            dt *= 0.9 / cfl
        if wl["regrid_interval"] and (n + 1) % wl["regrid_interval"] == 0:
            t0 = time.perf_counter()
            g.regrid()
            regrid_ms.append((time.perf_counter() - t0) * 1e3)
    return t, dt, regrid_ms


def _timed_steps(g, wl, steps, t, dt, flush):
    """The timed coarse steps: L2 flushed before each, CUDA events on the solver's
    stream around each advance (graph replay); the regrid every regrid_interval
    steps runs between timed steps and is reported separately."""
    import torch
    step_ms, cells, launches, regrid_ms, phases = [], 0.0, 0, [], []
    for k in range(steps):
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
        if wl.get("adapt_dt", wl["time_sync"]):
            dt *= 0.9 / cfl
        if wl["regrid_interval"] and (k + 1) % wl["regrid_interval"] == 0:
            t0 = time.perf_counter()
            g.regrid()
            regrid_ms.append((time.perf_counter() - t0) * 1e3)
            phases.append(g.last_regrid_stats())
    return dict(step_ms=step_ms, cells=cells, launches=launches, regrid_ms=regrid_ms, t=t, dt=dt,
                regrid_phases=phases)


def _roofline_pass(solvers, t_dt, flush, steps, wl=None):
    """Eager run of `steps` steps with a CUDA event pair around every update launch:
    (update ms, algorithmic bytes, launches) of the fused update kernel.  With `wl`
    (one forest) the steps follow the workload's dt rule and regrids, as the timed
    loop does; without it each solver takes steps of its fixed dt."""
    import torch
    ms, by, nl = 0.0, 0.0, 0
    for g in solvers:
        g.set_timing(True)
    for k in range(steps):
        for i, g in enumerate(solvers):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            t, dt = t_dt[i]
            if getattr(g, "ninst", 0):
                g.advance_instances(dt)
            elif wl is not None:
                cfl = g.advance(t, dt)
                dt1 = dt * 0.9 / cfl if wl.get("adapt_dt", wl["time_sync"]) else dt
                t_dt[i] = (t + dt, dt1)
            else:
                g.advance(t + k * dt, dt)
            st = g.last_update_stats()
            ms += st["update_ms"]
            by += st["update_bytes"]
            nl += st["update_launches"]
            if wl is not None and wl["regrid_interval"] and (k + 1) % wl["regrid_interval"] == 0:
                g.regrid()
    for g in solvers:
        g.set_timing(False)
    return ms, by, nl


def _tune(g, enabled, variant=None):
    if variant is not None:                       # a fixed patch-to-CTA variant, no tuning
        g.set_variant(variant)
        return {"variant": g.variant, "autotuned": False, **g.variants()[g.variant]}
    if not enabled:
        return {"variant": g.variant, "autotuned": False, **g.variants()[g.variant]}
    best, ms = g.autotune(reps=3)
    v = g.variants()
    lev = sorted(set(int(x) for x in g.patch_info()[:, 0]))
    per_level = g.level_variants()
    return {"variant": best, "autotuned": True, **v[best],
            "per_level": {str(l): int(per_level[l]) for l in lev if 0 <= l < 33},
            "candidates": [dict(ms_per_pass=round(float(m), 4), **x) for m, x in zip(ms, v)]}


def _roofline_dict(upd_ms, upd_bytes, upd_launches, traffic, bytes_per_cell):
    peaks = _peaks()
    achieved = upd_bytes / (upd_ms * 1e-3) / 1e9 if upd_ms > 0 else None
    return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": (achieved / peaks["hbm_gbs"]) if achieved else None, "traffic": traffic,
            "peak_source": peaks["source"], "kernel": "step2 fused update",
            "algorithmic_bytes_per_launch": upd_bytes / max(upd_launches, 1),
            "bytes_per_cell_update": bytes_per_cell, "avg_launch_ms": upd_ms / max(upd_launches, 1)}


def _fp64_kernel_arm(args, wl, prob, local_rank, flush):
    """The plain FP64 B200 kernel (bitwise equal to the CPU oracle) on the same
    workload and the same timing protocol: the comparator of the metric."""
    import forestclaw_b200 as fb
    _, gc = _options(wl, "fp64")
    gc.device = local_rank
    g = fb.Solver(gc)
    _maybe_partition(g, args, local_rank)
    g.initialize()
    t, dt, _ = _spinup(g, wl, 0.0, _initial_dt(wl, prob), wl["spinup"])
    tune = _tune(g, not args.no_autotune)         # --variant names a variant of the main arm
    t, dt, _ = _spinup(g, dict(wl, regrid_interval=0), t, dt, args.warmup)
    g.synchronize()
    _bracket()
    r = _timed_steps(g, wl, args.steps, t, dt, flush)
    _bracket()
    g.close()
    from forestclaw_b200 import ranks
    total_ms, _, value = ranks.aggregate(float(np.sum(r["step_ms"])), r["cells"], "cuda")
    return {"value": value, "ms_per_step": total_ms / args.steps,
            "variant": {k: tune[k] for k in ("variant", "threads", "min_blocks", "reg")}}


def _partitioned(args) -> bool:
    import torch.distributed as dist
    return bool(getattr(args, "partition", False)) and dist.is_available() and dist.is_initialized() \
        and dist.get_world_size() > 1


def _maybe_partition(g, args, local_rank):
    """With several ranks (and --partition, the default), the one forest is split
    over them along the space-filling curve with a halo exchange per ghost update
    (NCCL, device to device)."""
    if _partitioned(args):
        from forestclaw_b200 import partition as pt
        pt.partition(g, pt.TorchComm(device=local_rank))


def _bracket():
    """Both sides of a timed region: every rank's device idle, then a barrier."""
    import torch
    torch.cuda.synchronize()
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.barrier()


def _twin(gc, wl, prob, args, local_rank, mlp, variant, level_variants, start):
    """A second solver brought to the timed loop's first state: the same spin-up,
    regrids and variants, then the warm-up steps."""
    import forestclaw_b200 as fb
    g = fb.Solver(gc)
    _maybe_partition(g, args, local_rank)
    g.initialize()
    if mlp is not None:
        g.set_pstar_seed(mlp)
    t, dt, _ = _spinup(g, wl, 0.0, _initial_dt(wl, prob), wl["spinup"])
    g.set_variant(variant)
    g.set_level_variants(level_variants)
    t, dt = _spinup(g, dict(wl, regrid_interval=0), t, dt, args.warmup)[:2]
    if (t, dt) != start:
        raise SystemExit("a second solver did not reach the timed loop's first state")
    return g, t, dt


def run_ours(args, wl, rank, world, local_rank):
    """The measurement of one single-forest workload; the JSON dict on rank 0, else None."""
    import torch
    import forestclaw_b200 as fb
    if wl.get("batch"):
        return run_batch(args, wl, rank, world, local_rank)
    torch.cuda.set_device(local_rank)
    prob, gc = _options(wl, args.precision)
    gc.device = local_rank
    mlp, mlp_info = None, None
    if args.pstar == "mlp":
        mlp, mlp_info = train_pstar_mlp(wl, prob, local_rank, args.mlp_samples, args.mlp_epochs)
    g = fb.Solver(gc)
    _maybe_partition(g, args, local_rank)
    g.initialize()
    if mlp is not None:
        g.set_pstar_seed(mlp)
    # spin-up with regrid so the timed forest is representative (not timed),
    # then the autotuner picks the patch-to-CTA variant on that forest
    t, dt, regrid_ms = _spinup(g, wl, 0.0, _initial_dt(wl, prob), wl["spinup"])
    tune = _tune(g, not args.no_autotune, args.variant)
    t_start, dt_start = _spinup(g, dict(wl, regrid_interval=0), t, dt, args.warmup)[:2]
    t, dt = t_start, dt_start
    g.synchronize()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    g.set_timing(False)
    props = torch.cuda.get_device_properties(local_rank)
    clk = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local_rank))
    _bracket()
    if rank == 0:
        clk.start()
    r = _timed_steps(g, wl, args.steps, t, dt, flush)
    _bracket()
    clocks = clk.stop() if rank == 0 else None
    step_ms, cells, launches, timed_regrid_ms, t, dt = (r["step_ms"], r["cells"], r["launches"], r["regrid_ms"],
                                                         r["t"], r["dt"])
    from forestclaw_b200 import ranks
    total_ms, cells_all, value = ranks.aggregate(float(np.sum(step_ms)), cells, "cuda")
    newton = None
    if wl["name"].startswith("euler"):
        h = g.newton_histogram()
        newton = {"mean_iterations": float((np.arange(32) * h).sum() / max(h.sum(), 1)),
                  "histogram": [int(v) for v in h[:12]], "pstar_start": args.pstar, "mlp": mlp_info}
    npatch = g.num_patches
    level_variants = g.level_variants()
    g.close()
    twin = lambda: _twin(gc, wl, prob, args, local_rank, mlp, tune["variant"], level_variants, (t_start, dt_start))
    # ---- roofline: every update launch event-timed over the timed loop's K steps ----
    g, t, dt = twin()
    upd_ms, upd_bytes, upd_launches = _roofline_pass([g], [(t, dt)], flush, args.steps, wl)
    g.close()
    # ---- end to end through the C ABI with pinned host buffers, regrids included ----
    # the same K coarse steps as the timed loop, from its first state
    g, t, dt = twin()
    per_patch = gc.meqn * (gc.mx + 2 * gc.mbc) * (gc.my + 2 * gc.mbc)
    cap = 2 * g.num_patches * per_patch
    hq = torch.empty(cap, dtype=torch.float64, pin_memory=True)
    g.get_q_ptr(hq.data_ptr())
    e2e_steps = args.steps
    torch.cuda.synchronize()
    te0 = time.perf_counter()
    e2e_cells, e2e_h2d, e2e_d2h, e2e_regrids = 0.0, 0.0, 0.0, 0
    ph = {"set_q": 0.0, "advance": 0.0, "advance_after_regrid": 0.0, "get_q": 0.0, "regrid": 0.0}
    after_regrid = False
    for k in range(e2e_steps):
        c0 = g.cell_updates
        nq = g.num_patches * per_patch
        if nq > cap:                       # the forest outgrew the pinned buffer
            cap = 2 * nq
            hq = torch.empty(cap, dtype=torch.float64, pin_memory=True)
        p0 = time.perf_counter()
        g.set_q_ptr(hq.data_ptr())
        p1 = time.perf_counter()
        cfl = g.advance(t, dt)
        p2 = time.perf_counter()
        g.get_q_ptr(hq.data_ptr())
        p3 = time.perf_counter()
        ph["set_q"] += p1 - p0
        ph["advance_after_regrid" if after_regrid else "advance"] += p2 - p1
        ph["get_q"] += p3 - p2
        after_regrid = False
        e2e_cells += g.cell_updates - c0
        e2e_h2d += nq * 8
        e2e_d2h += nq * 8
        t += dt
        if wl.get("adapt_dt", wl["time_sync"]):
            dt *= 0.9 / cfl
        if wl["regrid_interval"] and (k + 1) % wl["regrid_interval"] == 0:
            p4 = time.perf_counter()
            g.regrid()
            e2e_regrids += 1
            after_regrid = True
            # the new forest's data back to the host copy (counted with the step's d2h bytes)
            nq = g.num_patches * per_patch
            if nq > cap:
                cap = 2 * nq
                hq = torch.empty(cap, dtype=torch.float64, pin_memory=True)
            g.get_q_ptr(hq.data_ptr())
            e2e_d2h += nq * 8
            ph["regrid"] += time.perf_counter() - p4
    e2e_s = time.perf_counter() - te0
    e2e_s = ranks.max_over_ranks(e2e_s, "cuda")
    e2e_cells = ranks.sum_over_ranks(e2e_cells, "cuda")
    e2e = {"value": e2e_cells / e2e_s, "unit": "cell-updates/s",
           "h2d_bytes_per_step": int(e2e_h2d / e2e_steps), "d2h_bytes_per_step": int(e2e_d2h / e2e_steps),
           "steps": e2e_steps, "regrids": e2e_regrids,
           "wall_ms_per_step": {k: round(v * 1e3 / e2e_steps, 4) for k, v in ph.items()},
           "protocol": "per coarse step: set_q from pinned host memory, advance, get_q to pinned host memory; "
                       "the workload's regrid (host tree edit, device repopulation, graph recapture) inside "
                       "the wall-clock region; the same coarse steps as the device-timed loop, from the same "
                       "state (a second solver spun up the same way)",
           "cells_match_timed_loop": bool(e2e_cells == cells_all),
           "graphs": g.graph_stats()}
    g.close()
    fp64 = None
    if args.precision != "fp64" and not args.no_fp64_compare:
        fp64 = _fp64_kernel_arm(args, wl, prob, local_rank, flush)
        fp64["speedup"] = value / fp64["value"] if world == 1 else None
    if rank != 0:
        return None
    bpc = 8 * (2 * gc.meqn + gc.maux)
    traffic = _traffic_per_launch(wl, args.precision, upd_bytes / max(upd_launches, 1) / bpc)
    roofline = _roofline_dict(upd_ms, upd_bytes, upd_launches, traffic, bpc)
    cpu = (cpu_sample(wl, args.precision, max_seconds=args.cpu_seconds, steps=args.steps)
           if args.cpu_seconds > 0 else None)
    err = None
    if args.precision == "fp32wave":
        oracle_ok = wl["name"].startswith(("radialdam", "euler"))
        err = (error_vs_oracle(wl, prob, local_rank, mlp) if oracle_ok
               else error_vs_fp64(wl, prob, local_rank, mlp))
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "strong" if _partitioned(args) else "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-waves/f64-q",
        "data": "synthetic (reference app initial data)",
        "config": {"workload": wl["name"], "patches": npatch, "precision": args.precision,
                   "multi_gpu": ("one forest partitioned along the space-filling curve, halo exchange per ghost "
                                 "update over NCCL" if _partitioned(args) else
                                 ("one replica of the forest per rank" if world > 1 else "one GPU")),
                   "cells_per_step": cells / args.steps,
                   "l2": "flushed between timed steps (512 MB write)",
                   "launch": "CUDA graph per coarse step (captured once per forest)",
                   "regrid": (f"every {wl['regrid_interval']} coarse steps between timed steps, excluded from "
                              "the device time" if wl["regrid_interval"] else "none"),
                   "regrids_in_timed_loop": len(timed_regrid_ms),
                   "regrid_ms_median": float(np.median(regrid_ms + timed_regrid_ms)) if regrid_ms else None,
                   "regrid_phase_ms_median": ({k: round(float(np.median([p[k] for p in r["regrid_phases"]])), 3)
                                               for k in r["regrid_phases"][0]} if r.get("regrid_phases") else None),
                   "patch_to_cta": tune},
        "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
        "fp64_kernel": fp64, ("error_vs_oracle" if err and "against" in err else "error_vs_fp64"): err,
        "newton": newton, "gpu_launches": launches, "update_launches": upd_launches,
    }
    return line


def _batch_groups(precision, device, n=64, seed=None):
    """The batched workload: n seeded tsunami instances, one solver per patch size
    (all instances of a size share every level launch)."""
    import forestclaw_b200 as fb
    from forestclaw_b200 import problems, ranks
    if seed is None:
        # each rank runs its own n instances (disjoint seeds): weak scaling, no exchange
        seed = ranks.instance_seed_base(ranks.rank_world()[0], n)
    insts, sizes = problems.tsunami_instances(n, seed)
    by = {}
    for k, (inst, mx) in enumerate(zip(insts, sizes)):
        by.setdefault(mx, []).append((k, inst))
    groups = []
    for mx in sorted(by):
        gc = problems.options(problems.TSUNAMI, mx=mx, my=mx, minlevel=0, maxlevel=0, subcycle=1, time_sync=1,
                              device=device)
        gc.precision = fb.PREC_FP32WAVE if precision == "fp32wave" else fb.PREC_FP64
        g = fb.Solver(gc)
        g.set_instances([x for _, x in by[mx]])
        g.initialize()
        # coarse dt for CFL ~0.9 at the initial state (max speed ~ sqrt(g * 2))
        dt = np.array([0.9 * (2.0 / (mx << x["minlevel"])) / 1.5 for _, x in by[mx]])
        groups.append({"g": g, "dt": dt, "mx": mx, "ids": [k for k, _ in by[mx]]})
    return groups


def _batch_step(groups, events=None):
    """One coarse step of every instance: all groups launched, then all waited for."""
    import torch
    if events is not None:
        start, ends = events
        start.record()
    for k, G in enumerate(groups):
        if events is not None:
            ext = torch.cuda.ExternalStream(G["g"].stream_handle())
            ext.wait_event(start)
        G["g"].advance_instances_begin(G["dt"])
        if events is not None:
            ends[k].record(ext)
    cfl = [G["g"].advance_instances_end() for G in groups]
    for G, c in zip(groups, cfl):
        G["dt"] = G["dt"] * 0.9 / c
    return cfl


def _batch_run(groups, steps, regrid_interval, flush=None, timed=False):
    import torch
    step_ms, cells, launches, regrid_ms = [], 0.0, 0, []
    for k in range(steps):
        ev = None
        if timed:
            flush.fill_(float(k))
            torch.cuda.synchronize()
            ev = (torch.cuda.Event(enable_timing=True), [torch.cuda.Event(enable_timing=True) for _ in groups])
        c0 = sum(G["g"].cell_updates for G in groups)
        _batch_step(groups, ev)
        if timed:
            torch.cuda.synchronize()
            step_ms.append(max(ev[0].elapsed_time(e) for e in ev[1]))
            launches += sum(G["g"].last_update_stats()["total_launches"] for G in groups)
        cells += sum(G["g"].cell_updates for G in groups) - c0
        if regrid_interval and (k + 1) % regrid_interval == 0:
            t0 = time.perf_counter()
            for G in groups:
                G["g"].regrid()
            regrid_ms.append((time.perf_counter() - t0) * 1e3)
    return dict(step_ms=step_ms, cells=cells, launches=launches, regrid_ms=regrid_ms)


def _batch_timed_arm(args, wl, precision, local_rank, flush, tune_on, clk=None):
    import torch
    groups = _batch_groups(precision, local_rank, wl["instances"])
    _batch_run(groups, wl["spinup"], wl["regrid_interval"])
    tunes = {str(G["mx"]): _tune(G["g"], tune_on) for G in groups}
    _batch_run(groups, args.warmup, 0)
    _bracket()
    if clk is not None:
        clk.start()
    r = _batch_run(groups, args.steps, wl["regrid_interval"], flush, timed=True)
    _bracket()
    r["clocks"] = clk.stop() if clk is not None else None
    return groups, tunes, r


def _batch_error(local_rank, n, steps=8):
    """Per-instance relative L1 error of h of the FP32-wave batch against the
    FP64 batch (bitwise equal to standalone oracle runs) from the same initial
    forests, the FP64 CFL setting both dt schedules, and the relative difference
    of each instance's mass (the instances have outflow boundaries, so mass
    itself changes in both)."""
    a = _batch_groups("fp64", local_rank, n)
    b = _batch_groups("fp32wave", local_rank, n)
    for k in range(steps):
        for A, B in zip(a, b):
            B["dt"] = A["dt"].copy()
        _batch_step(a)
        _batch_step(b)
    errs, dmass = [], []
    for A, B in zip(a, b):
        qa, qb = A["g"].get_q(), B["g"].get_q()
        ia, ib = A["g"].patch_instance(), B["g"].patch_instance()
        ma, mb = A["g"].mass_instances(), B["g"].mass_instances()
        for i in range(len(A["ids"])):
            xa, xb = qa[ia == i][:, 0, 2:-2, 2:-2], qb[ib == i][:, 0, 2:-2, 2:-2]
            errs.append(float(np.abs(xa - xb).sum() / np.abs(xa).sum()))
            dmass.append(float(abs(mb[i, 0] - ma[i, 0]) / abs(ma[i, 0])))
        A["g"].close()
        B["g"].close()
    return {"steps": steps, "l1_rel_h_max": max(errs), "l1_rel_h_median": float(np.median(errs)),
            "mass_rel_diff_vs_fp64_max": max(dmass), "instances": len(errs)}


def cpu_sample_batch(wl, max_seconds=15.0, threads=0):
    """The FP64 CPU oracle on the batch's instances, one after another (each a
    standalone forest), for a bounded time."""
    from oracle import pyoracle as po
    from forestclaw_b200 import problems
    from tests.cases import TSUNAMI, make
    insts, sizes = problems.tsunami_instances(wl["instances"], 0)
    t0 = time.perf_counter()
    cells, steps, used = 0.0, 0, 0
    for inst, mx in zip(insts, sizes):
        kw = {k: inst[k] for k in ("minlevel", "maxlevel", "pdata")}
        oc, _ = make(TSUNAMI, mx=mx, my=mx, subcycle=1, time_sync=1, nthreads=threads, **kw)
        o = po.OracleSim(oc)
        o.initialize()
        dt = 0.9 * (2.0 / (mx << inst["minlevel"])) / 1.5
        c0, t = o.cell_updates, 0.0
        for n in range(4):
            cfl = o.advance(t, dt)
            t += dt
            dt *= 0.9 / cfl
            steps += 1
        cells += o.cell_updates - c0
        used += 1
        if time.perf_counter() - t0 > max_seconds:
            break
    el = time.perf_counter() - t0
    return {"value": cells / el, "unit": "cell-updates/s", "cores": threads or os.cpu_count(), "kind": "port",
            "sample": f"4 coarse steps of each of the first {used} instances of {wl['name']}, standalone "
                      f"({cells:.3e} cell updates, {el:.1f} s, FP64 C oracle, OpenMP; setup included)"}


def run_batch(args, wl, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    props = torch.cuda.get_device_properties(local_rank)
    clk = ClockSampler(f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local_rank))
    if world > 1:
        torch.distributed.barrier()
    groups, tunes, r = _batch_timed_arm(args, wl, args.precision, local_rank, flush, not args.no_autotune,
                                        clk if rank == 0 else None)
    clocks = r["clocks"]
    from forestclaw_b200 import ranks
    cells = r["cells"]
    total_ms, cells_all, value = ranks.aggregate(float(np.sum(r["step_ms"])), cells, "cuda")
    nroof = max(2, min(args.steps, 4))
    upd_ms, upd_bytes, upd_launches = _roofline_pass([G["g"] for G in groups], [(0.0, G["dt"]) for G in groups],
                                                     flush, nroof)
    # ---- end to end: q of every group from pinned host memory and back, every step, the
    # ---- regrids inside (every regrid_interval steps, as in the timed loop) ----
    def qlen(g):
        o = g.opts
        return g.num_patches * o.meqn * (o.mx + 2 * o.mbc) * (o.my + 2 * o.mbc)
    # pinned buffers with room for twice the current forest (a regrid may grow it)
    bufs = [torch.empty(2 * qlen(G["g"]), dtype=torch.float64, pin_memory=True) for G in groups]
    for G, hq in zip(groups, bufs):
        G["g"].get_q_ptr(hq.data_ptr())
    interval = wl["regrid_interval"]
    e2e_steps = max(interval, min(args.steps, 3 * interval))
    torch.cuda.synchronize()
    te0 = time.perf_counter()
    e2e_cells, nbytes, nbytes_d2h, e2e_regrids = 0.0, 0, 0, 0
    for k in range(e2e_steps):
        c0 = sum(G["g"].cell_updates for G in groups)
        for G, hq in zip(groups, bufs):
            G["g"].set_q_ptr(hq.data_ptr())
        _batch_step(groups)
        for G, hq in zip(groups, bufs):
            G["g"].get_q_ptr(hq.data_ptr())
            nbytes += 8 * qlen(G["g"])
        e2e_cells += sum(G["g"].cell_updates for G in groups) - c0
        if (k + 1) % interval == 0:
            for j, G in enumerate(groups):
                G["g"].regrid()
                # the new forest's data back to the host copy (counted with the step's d2h bytes)
                if qlen(G["g"]) > bufs[j].numel():      # the forest outgrew the pinned buffer
                    bufs[j] = torch.empty(2 * qlen(G["g"]), dtype=torch.float64, pin_memory=True)
                G["g"].get_q_ptr(bufs[j].data_ptr())
                nbytes_d2h += 8 * qlen(G["g"])
            e2e_regrids += 1
    e2e_s = ranks.max_over_ranks(time.perf_counter() - te0, "cuda")
    e2e_cells = ranks.sum_over_ranks(e2e_cells, "cuda")
    e2e = {"value": e2e_cells / e2e_s, "unit": "cell-updates/s", "h2d_bytes_per_step": nbytes // e2e_steps,
           "d2h_bytes_per_step": (nbytes + nbytes_d2h) // e2e_steps, "steps": e2e_steps, "regrids": e2e_regrids,
           "protocol": "per coarse step: set_q of every group from pinned host memory, the step, get_q to "
                       "pinned host memory; the regrid every regrid_interval steps inside the wall-clock "
                       "region, continuing from the device-timed loop's last state"}
    info = {str(G["mx"]): {"instances": len(G["ids"]), "patches": G["g"].num_patches} for G in groups}
    for G in groups:
        G["g"].close()
    fp64 = None
    if args.precision != "fp64" and not args.no_fp64_compare:
        g64, tune64, r64 = _batch_timed_arm(args, wl, "fp64", local_rank, flush, not args.no_autotune)
        ms64, _, v64 = ranks.aggregate(float(np.sum(r64["step_ms"])), r64["cells"], "cuda")
        fp64 = {"value": v64, "ms_per_step": ms64 / args.steps,
                "variants": {k: {x: v[x] for x in ("variant", "threads", "min_blocks", "reg")}
                             for k, v in tune64.items()}}
        fp64["speedup"] = value / fp64["value"] if world == 1 else None
        for G in g64:
            G["g"].close()
    if rank != 0:
        return None
    roofline = _roofline_dict(upd_ms, upd_bytes, upd_launches, None, 8 * (2 * 3 + 1))
    cpu = cpu_sample_batch(wl, max_seconds=args.cpu_seconds) if args.cpu_seconds > 0 else None
    err = _batch_error(local_rank, wl["instances"]) if args.precision == "fp32wave" else None
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-waves/f64-q",
        "data": "synthetic (seeded instances: xoshiro256** per instance)",
        "config": {"workload": wl["name"], "instances": wl["instances"], "groups": info,
                   "precision": args.precision, "cells_per_step": cells / args.steps,
                   "l2": "flushed between timed steps (512 MB write)",
                   "launch": "one CUDA graph per patch-size group and coarse step (captured once per forest), "
                             "the groups on their own streams; step time = max over groups of events "
                             "from a common start",
                   "regrid": f"every {wl['regrid_interval']} coarse steps between timed steps, excluded",
                   "regrids_in_timed_loop": len(r["regrid_ms"]),
                   "regrid_ms_median": float(np.median(r["regrid_ms"])) if r["regrid_ms"] else None,
                   "patch_to_cta": tunes},
        "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
        "fp64_kernel": fp64, "error_vs_fp64": err,
        "gpu_launches": r["launches"], "update_launches": upd_launches,
    }
    return line


def launch_profile(args, wl):
    """The workload after its spin-up, then args.steps untimed coarse steps (graph replay):
    the launches of the last step are the last entries of an ncu launch list of this run."""
    import forestclaw_b200 as fb
    if wl.get("batch"):
        raise SystemExit("--launch-profile covers single-forest workloads")
    prob, gc = _options(wl, args.precision)
    g = fb.Solver(gc)
    g.initialize()
    t, dt, _ = _spinup(g, wl, 0.0, _initial_dt(wl, prob), wl["spinup"])
    for _ in range(args.steps):
        c = g.advance(t, dt)
        t += dt
        if wl.get("adapt_dt", wl["time_sync"]):
            dt *= 0.9 / c
    g.synchronize()
    lev = g.patch_info()[:, 0]
    print(json.dumps({"launch_profile": wl["name"], "steps": args.steps,
                      "patches_per_level": {str(int(l)): int((lev == l).sum()) for l in sorted(set(lev.tolist()))},
                      "last_step": g.last_update_stats()}), flush=True)
    g.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dam", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp32wave", choices=["fp64", "fp32wave"])
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="skip the timed run of the plain FP64 kernel on the same workload")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default patch-to-CTA variant")
    ap.add_argument("--variant", type=int, default=None,
                    help="use this patch-to-CTA variant (index into Solver.variants()), no autotuning")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--pstar", default="pvrs", choices=["pvrs", "mlp"],
                    help="Euler: Newton start of the exact solver (mlp: trained on the FP64 run first)")
    ap.add_argument("--mlp-samples", type=int, default=1_000_000)
    ap.add_argument("--mlp-epochs", type=int, default=20)
    ap.add_argument("--no-partition", dest="partition", action="store_false",
                    help="with several ranks, run one replica of a single-forest workload per rank instead of "
                         "partitioning the one forest over them")
    ap.add_argument("--no-secondary", dest="secondary", action="store_false",
                    help="skip the second measurement (shock-bubble with the learned p* start) of the default line")
    ap.add_argument("--secondary-steps", type=int, default=20)
    ap.add_argument("--launch-profile", action="store_true",
                    help="profiling aid, no timing: spin up the workload, run --steps coarse steps, print the "
                         "patches per level and the launches of the last step (for an ncu launch list)")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, wl, rank, world)
    if args.launch_profile:
        return launch_profile(args, wl)
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        line = run_ours(args, wl, rank, world, local_rank)
        if args.secondary and args.workload == "dam" and world == 1:
            # the Euler configuration with the learned p* start, as a second key of the line
            sargs = argparse.Namespace(**vars(args))
            sargs.steps, sargs.pstar, sargs.cpu_seconds = args.secondary_steps, "mlp", min(args.cpu_seconds, 10.0)
            sec = run_ours(sargs, WORKLOADS["shockbubble"], rank, world, local_rank)
            if line is not None and sec is not None:
                line["secondary"] = {"shockbubble_mlp": sec}
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
