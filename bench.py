"""Benchmark: photons/s of the MCML photon walk on one B200 (or one run sharded over N GPUs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload skin5|slab_n14] [--impl b200|reference]

A step is one full run of the workload: 'skin5' (default; five-layer skin stack, 1e8 photons,
nr=500 x nz=400 A(r,z), 30 exit-angle bins) or 'slab_n14' (one slab, 1e6 photons). `value` times
the walk kernel (with its tally zeroing) on the device with CUDA events on the launching stream,
L2 flushed between steps; `e2e` times the public C-ABI call tmc_b200_run with host buffers (the
run description goes in through the kernel parameters, the fixed-point tallies come back to host
memory and are decoded) by the host clock. `cpu_baseline` and `--impl reference` time the
reference's own multithreaded CPU engine (oracle/_ref/tissuemc, built from TissueMC's sources) on
a bounded sample of the same workload on this host's cores.

Under torchrun (N > 1) a step is ONE run of N times the workload's photons, sharded by photon id:
each rank walks its contiguous share (tmc_b200_run_device_range; the same Philox streams and
batches as on one GPU), then one NCCL all-reduce of the int64 fixed-point tally buffer (1.85 MB
for skin5) leaves the whole run's tallies on every rank, bit for bit those of a one-GPU run. Work
per GPU is fixed (weak scaling); the slowest rank's time is reported.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SWEEP_DESC = ("4096 configurations drawn by tmc_b200_sweep_sample(master seed 1): 1-3 layers, "
              "mua logU[0.01,10], mus' logU[1,50], g U[0.7,0.95], n U[1.33,1.5], d logU[0.01,1] cm, "
              "photons logU[1e4,1e6] (9.07e8 in all); grid nr=nz=64, dr=dz=0.01 cm, na=1; 10 batches each")
WORKLOADS = {
    "skin5": "five-layer skin stack (n=1.4 in air; 1e8 photons; dr=0.002 cm x 500, dz=0.001 cm x 400, na=30)",
    "slab_n14": "single slab n=1.4 in air (mua=5, mus=95, g=0.8, d=0.05 cm; 1e6 photons; 50x20 grid, na=30)",
    "sweep": SWEEP_DESC,
    "surrogate": "learned surrogate trained on sweep solves; gated serving and inverse fits",
    "serve": "fused ensemble inference: 4 members of 13(64) -> 4x512 GELU -> 66(128), gate on the R_d spread",
    "train": "surrogate training: 4 members, batch 4096 each, Adam + Polyak averaging, synthetic targets",
}
TRAIN_FLOP_PER_SAMPLE = 3 * 2 * (64 * 512 + 3 * 512 * 512 + 512 * 128)  # forward + two backward products
SERVE_FLOP_PER_QUERY = 4 * 2 * (64 * 512 + 3 * 512 * 512 + 512 * 128)  # 7.08 MFLOP (padded shapes)
METRIC = "photons/s on 1 B200 (plain MC)"
# DRAM bytes (read + write) of one walk launch, from one ncu capture of the full skin5 launch
# (1e8 photons; dram__bytes_read.sum 2.41 / 2.71 MB over two launches, dram__bytes_write.sum 0):
# the tally buffer's compulsory reads; the tallies stay in shared memory and L2, so the traffic
# does not grow with the photons.
WALK_DRAM_BYTES = {"skin5": 2.56e6}

# Algorithmic work of the walk, counted from the reference's step (include/tissuemc/physics.hpp
# :148-193 and :101-144 with the scoring) and frozen here: FP32 operations and SFU operations
# (log, sqrt, rsqrt, sin, cos, reciprocal of a division) per interaction step and per boundary
# step. The issue roofline of one SM is 128 FP32 lanes and 16 SFU lanes per clock.
F_INT, S_INT = 61, 12
F_BND, S_BND = 25, 3
# Interaction and boundary steps per photon, measured with the float64 oracle (seed 1).
STEPS_PER_PHOTON = {"skin5": (604.20, 14.30), "slab_n14": (19.71, 2.03)}


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="skin5", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--batches", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--photons", type=int, default=0,
                    help="override the workload's photon count (for profiling captures only)")
    ap.add_argument("--autotune", action="store_true", help="sweep: pick the launch shape first")
    ap.add_argument("--scale", type=float, default=1.0, help="surrogate: fraction of the full data and query counts")
    ap.add_argument("--epochs", type=int, default=300, help="surrogate: training epochs")
    ap.add_argument("--queries", type=int, default=1 << 20, help="serve: queries per step")
    ap.add_argument("--configs", type=int, default=4096, help="sweep: configurations")
    ap.add_argument("--photon-scale", type=float, default=1.0, help="sweep: scale every configuration's photons "
                    "(diagnostic)")
    ap.add_argument("--no-loop", action="store_true", help="sweep: skip the single-run loop baseline (diagnostic)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="walk: use the planner's default launch and tile plan instead of autotuning it")
    ap.add_argument("--tile-tz", type=int, default=None,
                    help="walk: the depth of the shared core tile (-1: none), instead of autotuning the plan "
                         "(for profiling one plan)")
    ap.add_argument("--threads", type=int, default=0,
                    help="walk: threads per block of the plan given by --tile-tz (0: the planner's 256)")
    ap.add_argument("--no-extras", action="store_true",
                    help="default line only: skip the sweep, serve and reference-GPU sub-measurements")
    ap.add_argument("--no-profiles", action="store_true",
                    help="diagnostic: skip the profile tallies (rung 6 without profiles); not a result")
    return ap.parse_args()


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


def _peak(key: str, fallback: float) -> tuple[float, str]:
    """A roofline denominator: `key` of MEASURED_PEAKS.json (searched through nested objects) when
    the file has it, else `fallback` (an earlier measurement on B200s of the same kind); returns the
    value and a note saying which."""

    def find(obj):
        if isinstance(obj, dict):
            v = obj.get(key)
            if isinstance(v, (int, float)) and not isinstance(v, bool):
                return float(v)
            for sub in obj.values():
                got = find(sub)
                if got is not None:
                    return got
        return None

    v = find(_peaks())
    if v is not None:
        return v, f"{key} of MEASURED_PEAKS.json (measured)"
    return fallback, f"fallback {fallback:g} (MEASURED_PEAKS.json has no {key})"


class Clocks:
    """nvidia-smi sampling during the timed region (SM clock and throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9], strict=False):
                if v.lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _cpu_info() -> tuple[str, int]:
    model = "unknown"
    try:
        m = re.search(r"model name\s*:\s*(.+)", Path("/proc/cpuinfo").read_text())
        model = m.group(1).strip() if m else model
    except OSError:
        pass
    return model, os.cpu_count() or 1


def reference_cpu_sample(workload: str, target_s: float = 12.0) -> dict:
    """Time the reference's own CPU engine (all host threads) on a bounded sample of the workload:
    a short pilot sizes the sample to about `target_s` seconds."""
    import oracle

    if not oracle.reference_available():
        raise RuntimeError("oracle/_ref/tissuemc is missing (built by `make -C oracle` where the reference sources are)")
    text = (ROOT / "tissuemc_b200" / "configs" / f"{workload}.mci").read_text()
    model, cores = _cpu_info()
    batches = max(10, 4 * cores)
    pilot = 20 * batches if workload == "skin5" else 2000 * batches
    r = oracle.run_reference(text, pilot, batches, 1, "float64", threads=0)
    rate = r["photons"] / max(r["wall_seconds"], 1e-3)
    n = max(batches, int(rate * target_s) // batches * batches)
    r = oracle.run_reference(text, n, batches, 1, "float64", threads=0)
    return {"value": r["photons"] / r["wall_seconds"], "unit": "photons/s", "cores": r["threads"],
            "kind": "reference", "seconds": r["wall_seconds"],
            "sample": f"{n} photons of {workload} ({batches} batches, float64, reference CPU engine "
                      f"oracle/_ref/tissuemc, {r['threads']} threads on {model})"}


REF_GPU_BIN = ROOT / "baseline" / "_ref" / "tissuemc_cuda"


def reference_gpu_run(workload: str, photons: int, batches: int, rung: int = 7, repeats: int = 2) -> dict:
    """The reference's own CUDA engine (TissueMC's src/cuda/engine.cu at rung `rung`, compiled
    unchanged for sm_100a into baseline/_ref/tissuemc_cuda by baseline/Makefile) on the same
    workload, photons, batches and seed on this GPU, timed by its own kernel_seconds (CUDA events
    around its kernels, src/cuda/engine.cu:209-275); the mean of `repeats` runs after one warm-up."""
    import tempfile

    if not REF_GPU_BIN.exists():
        return {"unavailable": "baseline/_ref/tissuemc_cuda is not built (make -C baseline needs the TissueMC sources)"}
    mci = ROOT / "tissuemc_b200" / "configs" / f"{workload}.mci"
    ks, ws = [], []
    with tempfile.TemporaryDirectory() as tmp:
        out = Path(tmp) / "ref.json"
        for i in range(repeats + 1):
            p = subprocess.run([str(REF_GPU_BIN), "run", str(mci), "--engine", "cuda", "--rung", str(rung),
                                "--photons", str(photons), "--batches", str(batches), "--seed", "1",
                                "--output", str(out)], capture_output=True, text=True, timeout=900)
            if p.returncode != 0:
                return {"unavailable": f"the reference's CUDA engine exited {p.returncode}: {p.stderr.strip()[:200]}"}
            r = json.loads(out.read_text())["runs"][0]
            if i:
                ks.append(float(r["kernel_seconds"]))
                ws.append(float(r["wall_seconds"]))
    k = sum(ks) / len(ks)
    return {"value": photons / k, "unit": "photons/s", "rung": rung, "kernel_seconds": k,
            "wall_seconds": sum(ws) / len(ws), "photons": photons, "batches": batches, "repeats": repeats,
            "what": f"TissueMC's own CUDA engine, rung {rung}, compiled unchanged for sm_100a "
                    "(baseline/_ref/tissuemc_cuda), its kernel_seconds on this GPU"}


def run_reference_arm(a) -> None:
    rank, world, _ = _dist()
    if rank != 0:
        return
    vals, secs = [], []
    for _ in range(a.warmup):
        reference_cpu_sample(a.workload, target_s=3.0)
    for _ in range(a.steps):
        s = reference_cpu_sample(a.workload, target_s=8.0)
        vals.append(s["value"])
        secs.append(s["seconds"])
    v = sum(vals) / len(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "photons/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the workload's .mci; seeded Philox photons)",
            "config": {"workload": f"{a.workload}: {WORKLOADS[a.workload]}", "photons_per_step": "bounded sample"},
            "cpu_baseline": {k: s[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": v, "unit": "photons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line["cpu_baseline"]["value"] = v
    print(json.dumps(line), flush=True)


# Interaction and boundary steps per photon of the 4096-configuration sweep workload, weighted by
# the configurations' photon counts (float64 oracle, 128 photons of each configuration).
SWEEP_STEPS_PER_PHOTON = (141.1, 3.8)


def issue_roofline(steps: tuple[float, float], n_sm: int, f_mhz: float) -> tuple[float, str, float, float]:
    """Photons/s of the FP32/SFU issue roofline for a photon of `steps` (interaction, boundary)
    steps: N_SM x f / max(F / 128, S / 16) with the frozen per-step counts F_*, S_*; returns the
    bound, which term binds, and F, S per photon."""
    f_tot = steps[0] * F_INT + steps[1] * F_BND
    s_tot = steps[0] * S_INT + steps[1] * S_BND
    clocks_per_photon = max(f_tot / 128.0, s_tot / 16.0) / n_sm
    return f_mhz * 1e6 / clocks_per_photon, ("sfu" if s_tot / 16.0 >= f_tot / 128.0 else "fp32"), f_tot, s_tot


def measure_sweep(configs: int, steps: int, warmup: int, device: int, seed: int = 1, autotune: bool = False,
                  photon_scale: float = 1.0, loop: bool = True) -> dict:
    """Batched sweep: solves/s of the graph-captured persistent launch (CUDA events around the sweep
    kernel, tmc_b200_sweep_run's kernel_seconds) and end to end (host clock around the call: table
    upload, the launch, the summary download), beside a loop of single-run launches over the same
    configurations (equal total photons)."""
    import tissuemc_b200 as tmc

    cfgs = tmc.sweep_sample(seed, configs)
    if photon_scale != 1.0:  # diagnostic: a shorter sweep over the same configurations
        for c in cfgs:
            c.photons = max(1, int(c.photons * photon_scale))
    opt = tmc.sweep_options(device=device)
    tuned = None
    if autotune:
        # the launch shape and per-warp tile, timed on this sweep itself (tmc_b200_sweep_autotune;
        # samples of fewer photons picked shapes that were slower at full size); the results do not
        # depend on them
        sample = cfgs
        t_default = min(tmc.sweep_run(sample, opt).seconds for _ in range(2))
        opt, t_best = tmc.sweep_autotune(sample, opt)
        tuned = {"sample": "the workload itself",
                 "sample_seconds_default": t_default, "sample_seconds_chosen": t_best,
                 "options": {k: int(getattr(opt, k)) for k in ("threads_per_block", "item_photons", "tile_r",
                                                                "tile_z")}}
    for _ in range(warmup):
        tmc.sweep_run(cfgs, opt)
    with Clocks(device) as clk:
        kern, wall = [], []
        for _ in range(steps):
            t0 = time.perf_counter()
            r = tmc.sweep_run(cfgs, opt)
            wall.append(time.perf_counter() - t0)
            kern.append(r.seconds)
    loop_s = tmc.sweep_run_loop(cfgs, opt).seconds if loop else None
    n = len(cfgs)
    ks, ws = sum(kern) / len(kern), sum(wall) / len(wall)
    photons = sum(int(c.photons) for c in cfgs)
    import torch

    n_sm = torch.cuda.get_device_properties(device).multi_processor_count
    f_mhz, f_note = _peak("sm_max_mhz", 1965.0)
    peak, bound, f_tot, s_tot = issue_roofline(SWEEP_STEPS_PER_PHOTON, n_sm, f_mhz)
    return {
        "metric": "solves/s on 1 B200 (batched sweep)", "value": n / ks, "unit": "solves/s",
        "ms_per_step": 1e3 * ks, "steps": steps, "warmup": warmup,
        "config": {"workload": f"sweep: {SWEEP_DESC}", "configs": n, "photon_scale": photon_scale,
                   "threads_per_block": opt.threads_per_block, "item_photons": opt.item_photons,
                   "tile_r": opt.tile_r, "tile_z": opt.tile_z, "autotuned": bool(autotune)},
        "autotune": tuned,
        "e2e": {"value": n / ws, "unit": "solves/s",
                "h2d_bytes_per_step": n * 48 + n * 4 + sum(c.num_layers for c in cfgs) * 96,
                "d2h_bytes_per_step": n * (opt.nr + 3) * 8},
        "loop_baseline": None if loop_s is None else {
            "value": n / loop_s, "unit": "solves/s", "seconds": loop_s,
            "what": "one single-run walk launch per configuration, back to back on one stream"},
        "speedup_vs_loop": None if loop_s is None else loop_s / ks,
        "photons_per_s": photons / ks,
        "roofline": {"bound": bound, "achieved": photons / ks / 1e9, "peak": peak / 1e9, "unit": "Gphotons/s",
                     "frac": photons / ks / peak,
                     "peak_source": f"issue roofline: {n_sm} SMs x {f_mhz:.0f} MHz ({f_note}) / max(F/128, S/16), "
                                    f"F={f_tot:.0f} FP32 and S={s_tot:.0f} SFU ops per photon"},
        "gpu_launches": steps * 2, "clocks": clk.summary(),
    }


def run_sweep(a) -> None:
    rank, world, local = _dist()
    m = measure_sweep(a.configs, a.steps, a.warmup, local, seed=1 + rank, autotune=a.autotune,
                      photon_scale=a.photon_scale, loop=not a.no_loop)
    if rank == 0:
        line = {"metric": m["metric"], "value": world * m["value"], "unit": "solves/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 transport, u64 fixed-point tallies",
                "data": "synthetic (seeded configurations)"}
        line.update({k: v for k, v in m.items() if k not in line})
        print(json.dumps(line), flush=True)


def run_surrogate(a) -> None:
    """The learned surrogate end to end (training data from the batched sweep, training, accuracy
    against high-photon MC, gated serving, inverse fits); one JSON line of its measurements."""
    from tissuemc_b200 import surrogate

    rank, world, local = _dist()
    res = surrogate.pipeline(scale=a.scale, epochs=a.epochs, log=lambda m: print(m, file=sys.stderr, flush=True))
    if rank == 0:
        s = res["serving"]
        print(json.dumps({
            "metric": "gated surrogate queries/s on 1 B200", "value": s["gated_queries_per_s"], "unit": "queries/s",
            "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 GEMMs, fp32 accumulation", "data": "synthetic (sweep-generated)",
            "config": {"workload": "surrogate: 12+1 -> 4x512 GELU -> 66 MLP, 4 members, batch 4096", "scale": a.scale},
            "speedup_vs_plain_mc": s["speedup_vs_plain_mc"], "details": res}), flush=True)


def measure_serve(queries: int, steps: int, warmup: int, device: int, seed: int = 3000) -> dict:
    """Surrogate serving throughput: one fused tcgen05 launch (tmc_b200_nn_ensemble_infer) per step
    over `queries` feature vectors drawn from the sweep distribution. The weights are random (the
    kernel's work does not depend on their values). value = queries / CUDA-event time of the launch,
    L2 flushed between steps; e2e = queries / host time of FusedServer (pinned host features in,
    host outputs, mean R_d and route flags out)."""
    import numpy as np
    import torch

    import tissuemc_b200 as tmc
    from tissuemc_b200 import surrogate as S

    torch.cuda.set_device(device)
    n = queries
    ens = S.Ensemble(members=4, batch=4096, seed=0, device=f"cuda:{device}")
    ens.norm = S.Norm(np.zeros(S.N_FEAT), np.ones(S.N_FEAT), np.full(S.N_OUT, -2.0), np.full(S.N_OUT, 0.3))
    q = S.features(tmc.sweep_sample(seed, n))
    q = (q - q.mean(0)) / np.maximum(q.std(0), 1e-6)
    fs = S.FusedServer(ens)
    fs._reserve(n)
    fs.d_feats[:n].copy_(torch.from_numpy(q.astype(np.float32)))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")
    stream = torch.cuda.current_stream()

    def step() -> float:
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fs.launch(fs.d_feats, n, fs.d_out, fs.d_rd, fs.d_spread, fs.d_route, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(warmup):
        step()
    with Clocks(device) as clk:
        times = [step() for _ in range(steps)]
    if tmc.lib().tmc_b200_nn_status(1):
        raise RuntimeError("a tensor-core wait gave up in the fused ensemble kernel")
    ms = sum(times) / len(times)
    # end to end: features already in pinned host memory, results back in pinned host memory
    h_q = torch.from_numpy(q.astype(np.float32)).pin_memory()
    e2e_t = []
    for i in range(steps + 1):
        t0 = time.perf_counter()
        fs(h_q, copy=False)
        if i:
            e2e_t.append(time.perf_counter() - t0)
    e2e_s = sum(e2e_t) / len(e2e_t)
    peak, peak_note = _peak("bf16_tflops", 1590.0)
    achieved = n * SERVE_FLOP_PER_QUERY / (ms * 1e-3) / 1e12
    del flush
    return {
        "metric": "surrogate queries/s on 1 B200 (fused ensemble kernel)", "value": n / (ms * 1e-3),
        "unit": "queries/s", "ms_per_step": ms, "steps": steps, "warmup": warmup,
        "dtype": "bf16 operands, fp32 accumulation",
        "config": {"workload": f"serve: {WORKLOADS['serve']}", "queries_per_step": n,
                   "l2": "flushed between steps (256 MB write)"},
        "e2e": {"value": n / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": n * S.N_FEAT * 4,
                "d2h_bytes_per_step": n * (S.N_OUT * 4 + 4 + 1)},
        "gpu_launches": steps,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": f"bf16 burst peak: {peak_note}; algorithmic FLOPs of the "
                                    "padded layers, 7.08 MFLOP per query"},
        "clocks": clk.summary(),
    }


def run_serve(a) -> None:
    rank, world, local = _dist()
    m = measure_serve(a.queries, a.steps, a.warmup, local, seed=3000 + rank)
    if rank == 0:
        line = {"metric": m["metric"], "value": m["value"], "unit": "queries/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "data": "synthetic (sweep-distribution queries, random weights)"}
        line.update({k: v for k, v in m.items() if k not in line})
        print(json.dumps(line), flush=True)


def run_train(a) -> None:
    """Surrogate training throughput: --steps optimiser steps of the 4-member ensemble (forward,
    backward, Adam, averaging: every product on the tcgen05 kernels) on synthetic samples;
    value = samples per second over all members, CUDA events around the steps that replay the
    captured step graph (the first step of the call, launched from the host while the graph is
    captured, is not timed)."""
    import numpy as np
    import torch

    from tissuemc_b200 import surrogate as S

    rank, world, local = _dist()
    torch.cuda.set_device(local)
    rng = np.random.default_rng(rank)
    X, Y = rng.normal(size=(65536, S.N_FEAT)), rng.normal(size=(65536, S.N_OUT))
    ens = S.Ensemble(members=4, batch=4096, seed=0, device=f"cuda:{local}")
    ens.train(X[:4096 * max(1, a.warmup)], Y[:4096 * max(1, a.warmup)], epochs=1, lr=1e-3, ema=0.999)
    steps = max(1, a.steps)
    n = 4096 * steps
    Xs, Ys = np.resize(X, (n, S.N_FEAT)), np.resize(Y, (n, S.N_OUT))
    with Clocks(local) as clk:
        ens.train(Xs, Ys, epochs=1, lr=1e-3, ema=0.999)
    ms = ens.last_step_ms  # CUDA events around the replayed optimiser steps (data upload and setup excluded)
    if rank == 0:
        peak, peak_note = _peak("bf16_tflops_sustained", 1400.0)
        achieved = 4 * 4096 * TRAIN_FLOP_PER_SAMPLE / (ms * 1e-3) / 1e12
        print(json.dumps({
            "metric": "surrogate training samples/s on 1 B200 (4-member ensemble)",
            "value": 4 * 4096 / (ms * 1e-3), "unit": "samples/s", "n_gpus": world, "steps": steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 operands, fp32 accumulation and master weights", "data": "synthetic (random samples)",
            "config": {"workload": f"train: {WORKLOADS['train']}"},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "peak_source": f"bf16 sustained peak (a seconds-long training loop): {peak_note}; "
                                        "3 x forward FLOPs per sample"},
            "clocks": clk.summary(),
        }), flush=True)


def main() -> None:
    a = _args()
    if a.impl == "reference":
        run_reference_arm(a)
        return
    if a.workload == "surrogate":
        run_surrogate(a)
        return
    if a.workload == "sweep":
        run_sweep(a)
        return
    if a.workload == "serve":
        run_serve(a)
        return
    if a.workload == "train":
        run_train(a)
        return
    import ctypes

    import torch

    import numpy as np

    import tissuemc_b200 as tmc

    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    spec = tmc.workload(a.workload)
    if a.photons:
        spec.photons = a.photons
    photons = spec.photons  # per GPU
    # With N GPUs the job is ONE run of N x photons, sharded by photon id: each rank walks its
    # contiguous share (the same streams and batches as on one GPU) and one NCCL all-reduce of the
    # int64 tally buffer gives every rank the whole run's tallies, bit for bit a 1-GPU run's.
    spec.photons = photons * world
    first, count = tmc.shard_range(spec.photons, rank, world)
    opt = tmc.options(batches=a.batches, seed=1, device=local, rung=6 if a.no_profiles else 0,
                      profiles=not a.no_profiles, tile_tz=a.tile_tz or 0)
    if a.tile_tz is not None:
        opt.threads_per_block = a.threads
    tuning = None
    if not a.no_autotune and a.tile_tz is None:
        # the launch and tally-tile plan, picked by timing candidates on a 2e7-photon sample of
        # this run (tmc_b200_autotune); the results do not depend on it
        opt, plan, t_default, t_best = tmc.autotune(spec, opt, sample_photons=min(spec.photons, 20_000_000))
        tuning = {"plan": plan, "sample_photons": min(spec.photons, 20_000_000),
                  "sample_seconds_default_plan": t_default, "sample_seconds_chosen_plan": t_best,
                  "options": {k: int(getattr(opt, k)) for k in ("threads_per_block", "blocks_per_sm", "tile_tz",
                                                                 "tile_ra_rows", "tile_cross")}}
    sizes = tmc.query_sizes(spec, opt)
    words = int(sizes.tally_words)
    # the tallies, then the launch's photon-claim counter (device_words = tally_words + 1)
    d_tally = torch.empty(int(sizes.device_words), dtype=torch.int64, device=f"cuda:{local}")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    stream = torch.cuda.Stream(device=local)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            torch.cuda.synchronize()

    def walk() -> None:
        """This rank's share of the run, then (N > 1) the all-reduce, on `stream`."""
        if world == 1:
            tmc.run_device(spec, opt, d_tally.data_ptr(), stream.cuda_stream)
        else:
            import torch.distributed as dist

            tmc.run_device_range(spec, opt, first, count, d_tally.data_ptr(), stream.cuda_stream)
            dist.all_reduce(d_tally)  # unsigned 64-bit sums are int64 two's-complement sums

    def step() -> float:
        with torch.cuda.stream(stream):
            flush.fill_(1.0)  # evict L2 between steps (outside the timed events)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            walk()
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(a.warmup):
        step()
    barrier()
    with Clocks(local) as clk:
        times = [step() for _ in range(a.steps)]
        barrier()
    total_ms = sum(times)
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([total_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / a.steps
    value = spec.photons / (ms / 1e3)

    # end to end through the public API with host buffers: on one GPU tmc.run (the C ABI's
    # tmc_b200_run); on N, each rank's shard, the all-reduce, the copy back and the decode
    e2e_times = []
    sz = tmc.query_sizes(spec, opt)
    for i in range(a.steps + 1):
        t0 = time.perf_counter()
        if world == 1:
            res = tmc.run(spec, opt)
        else:
            with torch.cuda.stream(stream):
                walk()
            stream.synchronize()  # the walk and the all-reduce ran on `stream`, not the current one
            host = d_tally[:words].cpu()
            res = tmc.decode(spec, opt, host.numpy().view(np.uint64))
            res.device = torch.cuda.get_device_name(local)
        if i:  # the first call is a warm-up
            e2e_times.append(time.perf_counter() - t0)
    e2e_s = sum(e2e_times) / len(e2e_times)
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": spec.photons / e2e_s, "unit": "photons/s",
           "h2d_bytes_per_step": int(ctypes.sizeof(tmc.CRunSpec) + ctypes.sizeof(tmc.COptions)),
           "d2h_bytes_per_step": int(sz.tally_words) * 8}

    if rank == 0:
        f_mhz, f_note = _peak("sm_max_mhz", 1965.0)
        n_sm = torch.cuda.get_device_properties(local).multi_processor_count
        peak, bound, f_tot, s_tot = issue_roofline(STEPS_PER_PHOTON[a.workload], n_sm, f_mhz)
        achieved = photons / (ms / 1e3)
        line = {
            "metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 transport, u64 fixed-point tallies",
            "data": "synthetic (the workload's .mci; seeded Philox photons)",
            "config": {"workload": f"{a.workload}: {WORKLOADS[a.workload]}", "photons_per_step": spec.photons, "photons_per_gpu": photons,
                       "batches": a.batches, "l2": "flushed between steps (256 MB write)",
                       "profiles": not a.no_profiles,
                       "parallelism": f"one run sharded by photon id over {world} GPUs + NCCL int64 all-reduce"
                       if world > 1 else "1 GPU"},
            "e2e": e2e,
            "gpu_launches": a.steps,
            "roofline": {
                "bound": bound, "achieved": achieved / 1e9,
                "peak": peak / 1e9, "unit": "Gphotons/s", "frac": achieved / peak,
                "traffic": WALK_DRAM_BYTES.get(a.workload) if not a.photons else None,
                "peak_source": f"issue roofline: {n_sm} SMs x {f_mhz:.0f} MHz ({f_note}) / "
                               f"max(F/128, S/16) with F={f_tot:.0f} FP32 and S={s_tot:.0f} SFU ops per photon",
            },
            "clocks": clk.summary(),
            "kernel_ms_per_step": ms,
            "autotune": tuning,
            "device": res.device,
        }  # fmt: skip
        if not a.no_cpu_baseline and world == 1:
            try:
                line["cpu_baseline"] = reference_cpu_sample(a.workload)
                line["cpu_baseline"].pop("seconds", None)
            except Exception as exc:  # report, never fake
                line["cpu_baseline"] = {"unavailable": str(exc)}
        if world == 1 and not a.no_extras and not a.photons:
            # the other parts of the metric, measured in the same run on the same GPU: the batched
            # sweep (solves/s vs the loop of plain launches), the gated surrogate's serving kernel,
            # and the reference's own CUDA engine on this workload
            ref_gpu = reference_gpu_run(a.workload, spec.photons, a.batches)
            if "value" in ref_gpu:
                ref_gpu["b200_kernel_speedup"] = value / ref_gpu["value"]
            line["reference_gpu"] = ref_gpu
            for key, fn in (("sweep", lambda: measure_sweep(4096, 2, 1, local, autotune=not a.no_autotune)),
                            ("serve", lambda: measure_serve(1 << 20, 5, 3, local))):
                try:
                    line[key] = fn()
                except Exception as exc:  # report, never fake
                    line[key] = {"unavailable": f"{type(exc).__name__}: {exc}"}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
